"""Parallel-in-length pass 1: the sweeps of every chain split into pieces
(transfer matrices, prefix over the pieces, piece sweeps) give the charge of
the single sweep."""
import pytest

from test_gpu_parity import CASES, _pair, _rel

pytestmark = pytest.mark.gpu


def _with_pieces(tube, P):
    from electrostatic_b200 import _lib
    from electrostatic_b200.negf import last_stats
    L = _lib.load()
    assert L.negf_set_tuning(4, P) == 0
    try:
        Q = tube.Solve_NEGF()
        return Q, last_stats()
    finally:
        L.negf_set_tuning(4, 0)


@pytest.mark.parametrize("case", ["equilibrium_poles", "bias_gl_paths", "window_regular"])
@pytest.mark.parametrize("P", [2, 5, 16])
def test_pieces_equal_single_sweep(oracle, case, P):
    g, o = _pair(oracle, seed=41, **CASES[case])
    Q1, _ = _with_pieces(g, 1)
    QP, st = _with_pieces(g, P)
    assert st["pieces"] == P
    assert _rel(QP, Q1) <= 1e-10, _rel(QP, Q1)
    assert _rel(QP, o.charge(nthreads=8)) <= 1e-8


def test_pieces_mixed_precision_and_decimation(oracle):
    kw = dict(type_id=(17, 0), num_unitcells=40, num_modes=3, contact_mu=(0.0, -0.3), contact_T=(300.0, 320.0),
              eq_integration_pts=(24, 24, 40), noneq_integration_pts=(60,), E_zPlus_imag=2e-3, use_decimation=1,
              precision="mixed")
    g, o = _pair(oracle, seed=42, **kw)
    Q1, _ = _with_pieces(g, 1)
    QP, _ = _with_pieces(g, 7)
    assert _rel(QP, Q1) <= 1e-6
    assert _rel(QP, o.charge(nthreads=8)) <= 1e-5


def test_long_tube_automatic_pieces():
    """A 16000-site tube with few energies: the automatic choice splits it."""
    from electrostatic_b200.negf import CNT
    from electrostatic_b200.workloads import site_potential
    g = CNT(type_id=(17, 0), num_unitcells=4000, num_modes=2, contact_mu=(0.0, -0.2), contact_T=(300.0, 300.0),
            eq_integration_pts=(8, 8, 16), noneq_integration_pts=(32,), E_zPlus_imag=1e-3)
    U = site_potential(g.site_positions(), 7, amp=0.2, ramp=0.2)
    g.set_potential(U, (U[0], U[-1]))
    Qa, st = _with_pieces(g, 0)
    assert st["pieces"] > 1
    Q1, _ = _with_pieces(g, 1)
    assert _rel(Qa, Q1) <= 1e-10, _rel(Qa, Q1)


def _long_tubes():
    from electrostatic_b200.negf import CNT
    from electrostatic_b200.workloads import site_potential
    tubes = []
    for k, (uc, mu) in enumerate([(3000, -0.2), (2000, -0.1)]):
        t = CNT(type_id=(17, 0), num_unitcells=uc, num_modes=2, contact_mu=(0.0, mu), contact_T=(300.0, 300.0),
                eq_integration_pts=(8, 8, 16), noneq_integration_pts=(24,), E_zPlus_imag=1e-3)
        U = site_potential(t.site_positions(), 11 + k, amp=0.2, ramp=0.2)
        t.set_potential(U, (U[0], U[-1]))
        tubes.append(t)
    return tubes


def _plan_charge(tubes, P, autotune=False):
    import torch
    from electrostatic_b200 import _lib
    from electrostatic_b200.negf import ChargePlan
    L = _lib.load()
    assert L.negf_set_tuning(4, P) == 0
    try:
        Q = torch.zeros(sum(t.num_field_sites for t in tubes), dtype=torch.float64, device="cuda")
        plan = ChargePlan(tubes, Q, autotune=autotune)
        plan.launch()
        torch.cuda.synchronize()
        info = plan.info()
        skip = torch.ones(1, dtype=torch.int32, device="cuda")
        Qs = Q.clone()
        plan.launch(skip=skip)  # a set skip flag leaves the charge untouched
        torch.cuda.synchronize()
        assert torch.equal(Q, Qs)
        plan.close()
        return Q.cpu().numpy(), info
    finally:
        L.negf_set_tuning(4, 0)


def test_plan_pieces_equal_single_sweep():
    """Charge plans of long tubes with few energies: the automatic rule and a
    forced piece count split the sweeps, with the charge of the single sweep."""
    tubes = _long_tubes()
    Q1, i1 = _plan_charge(tubes, 1)
    assert i1["pieces"] == 1
    Qa, ia = _plan_charge(tubes, 0)
    assert ia["pieces"] > 1 and ia["pass2_warps_per_block"] > 0
    assert _rel(Qa, Q1) <= 1e-10, _rel(Qa, Q1)
    Q6, i6 = _plan_charge(tubes, 6)
    assert i6["pieces"] == 6
    assert _rel(Q6, Q1) <= 1e-10, _rel(Q6, Q1)


def test_plan_autotune_considers_pieces():
    tubes = _long_tubes()
    Q1, _ = _plan_charge(tubes, 1)
    Qt, it = _plan_charge(tubes, 0, autotune=True)
    assert it["pieces"] >= 1 and it["tuned_ms"] > 0
    if it["pass2_warps_per_block"] == 0:
        assert it["pieces"] == 1
    assert _rel(Qt, Q1) <= 1e-10, _rel(Qt, Q1)
