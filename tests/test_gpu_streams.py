"""Charge calls on two streams at once keep separate device scratch.

Two tubes of different sizes are integrated on two CUDA streams with calls
interleaved and no host synchronisation between them (the second stream's
kernels can run while the first stream's are in flight).  Each result must
match the FP64 oracle; with one shared scratch the second call would
overwrite the first call's checkpoints and launch tables.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-8


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


CASE_A = dict(type_id=(17, 0), num_unitcells=300, num_modes=4, contact_mu=(0.0, -0.4), contact_T=(300.0, 300.0),
              eq_integration_pts=(48, 48, 96), noneq_integration_pts=(200, 400, 200), noneq_percent_intercuts=(30.0, 70.0),
              E_zPlus_imag=1e-3)
CASE_B = dict(type_id=(13, 0), num_unitcells=120, num_modes=5, contact_mu=(-0.3, -0.3), contact_T=(300.0, 300.0),
              eq_integration_pts=(64, 64, 128), E_pole_max=3.0)


def test_two_streams_distinct_tubes_match_oracle(negf_lib, oracle):
    import torch
    from electrostatic_b200.negf import CNT, compute_charge
    from electrostatic_b200.workloads import site_potential

    cases = []
    for i, kw in enumerate((CASE_A, CASE_B)):
        g = CNT(**kw)
        U = site_potential(g.site_positions(), 77 + i)
        g.set_potential(U, (U[0], U[-1]))
        o = oracle.OracleTube(**kw, noneq_percent_intercuts=None) if "noneq_percent_intercuts" not in kw else \
            oracle.OracleTube(**kw)
        o.set_potential(U, (U[0], U[-1]))
        cases.append((g, o.charge(nthreads=8)))
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    QA = torch.zeros(cases[0][0].num_field_sites, dtype=torch.float64, device="cuda")
    QB = torch.zeros(cases[1][0].num_field_sites, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    for _ in range(4):
        with torch.cuda.stream(s1):
            compute_charge([cases[0][0]], out=QA, stream=s1)
        with torch.cuda.stream(s2):
            compute_charge([cases[1][0]], out=QB, stream=s2)
    torch.cuda.synchronize()
    errA = _rel(QA.cpu().numpy(), cases[0][1])
    errB = _rel(QB.cpu().numpy(), cases[1][1])
    assert errA <= FP64_TOL and errB <= FP64_TOL, (errA, errB)


def test_release_scratch_frees_and_next_call_reallocates(negf_lib, oracle):
    """negf_release_scratch hands a stream's scratch back to the device (the
    free memory grows by at least the checkpoint bytes of the last call) and
    the next call on that stream allocates it again and gives the same charge,
    bitwise, with the kernel times of a timed call still readable."""
    import torch
    from electrostatic_b200.negf import CNT, compute_charge, last_stats, release_scratch, set_timing
    from electrostatic_b200.workloads import site_potential

    g = CNT(**CASE_A)
    U = site_potential(g.site_positions(), 91)
    g.set_potential(U, (U[0], U[-1]))
    o = oracle.OracleTube(**CASE_A)
    o.set_potential(U, (U[0], U[-1]))
    Qo = o.charge(nthreads=8)
    s = torch.cuda.Stream()
    Q1 = torch.zeros(g.num_field_sites, dtype=torch.float64, device="cuda")
    Q2 = torch.zeros_like(Q1)
    set_timing(True)
    try:
        compute_charge([g], out=Q1, stream=s)
        scratch = last_stats()["checkpoint_bytes"]
        compute_charge([g], out=Q1, stream=s)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        release_scratch(s)  # the timed call's events go with the workspace
        free_after = torch.cuda.mem_get_info()[0]
        st = last_stats()
    finally:
        set_timing(False)
    assert st["rgf_kernel_ms"] > 0.0
    assert free_after - free_before >= scratch // 2, (free_before, free_after, scratch)
    release_scratch(s)  # nothing left on that stream: a no-op
    compute_charge([g], out=Q2, stream=s)
    torch.cuda.synchronize()
    assert torch.equal(Q1, Q2)
    assert _rel(Q2.cpu().numpy(), Qo) <= FP64_TOL
