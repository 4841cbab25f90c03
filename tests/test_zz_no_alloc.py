"""The allocation-free charge entry point, through the C-ABI.

negf_compute_charge_noalloc serves callers that cannot allocate device memory
when they need the induced charge (programs whose device memory comes from
their own pool, plugins that must not grow the host program's footprint).  It
keeps every per-call buffer in one static 32 MiB device array shared by all
calls.  These checks compare it with negf_compute_charge on two calls in a row
(with different potentials, so a stale array would show), with the FP64
oracle, on a mixed-precision tube and on an energy shard (rank 1 of 2, no Rho0
subtraction), and check that an oversized problem is refused.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-8  # norm-wise relative bound used by the FP64 parity tests
MIXED_TOL = 1e-5  # the same bound for the mixed-precision path


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def _potential(y, seed):
    rng = np.random.default_rng(seed)
    U = 0.3 * np.exp(-((y - rng.uniform(y[0], y[-1])) ** 2) / 20.0)
    return U + 0.2 * (y - y[0]) / (y[-1] - y[0]) + rng.uniform(-0.05, 0.05)


def test_noalloc_matches_compute_charge_on_two_calls(negf_lib):
    import torch
    from electrostatic_b200.negf import CNT, compute_charge

    tubes = [
        CNT(type_id=(17, 0), num_unitcells=40, num_modes=3, contact_mu=(0.0, -0.3), contact_T=(300.0, 300.0),
            eq_integration_pts=(24, 24, 40), noneq_integration_pts=(96,)),
        CNT(type_id=(13, 0), num_unitcells=15, num_modes=2, contact_mu=(-0.5, -0.5), contact_T=(300.0, 300.0),
            eq_integration_pts=(32, 32, 32), E_pole_max=3.0),
    ]
    total = sum(t.num_field_sites for t in tubes)
    handles = (C.c_void_p * len(tubes))(*[t.handle for t in tubes])
    out = torch.empty(total, dtype=torch.float64, device="cuda")
    for call, seed in enumerate((1, 2)):
        for t in tubes:
            U = _potential(t.site_positions(), seed * 10 + t.num_field_sites)
            t.set_potential(U, (U[0], U[-1]))
        ref = compute_charge(tubes)  # the allocating entry point, host output
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = negf_lib.negf_compute_charge_noalloc(handles, len(tubes), C.c_void_p(out.data_ptr()), None)
        assert rc == 0, negf_lib.negf_last_error().decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got)), f"call {call}"
        assert _rel(got, ref) <= TOL, (call, _rel(got, ref))


def test_noalloc_refuses_oversized_problem(negf_lib):
    import torch
    from electrostatic_b200.negf import CNT

    big = CNT(type_id=(17, 0), num_unitcells=1000, num_modes=8, contact_mu=(0.0, -0.5), contact_T=(300.0, 300.0),
              eq_integration_pts=(64, 64, 128), E_zPlus_imag=1e-4, realaxis_window=(-1.5, 1.5, 512, 0))
    out = torch.empty(big.num_field_sites, dtype=torch.float64, device="cuda")
    handles = (C.c_void_p * 1)(big.handle)
    rc = negf_lib.negf_compute_charge_noalloc(handles, 1, C.c_void_p(out.data_ptr()), None)
    assert rc == -1  # NEGF_ERR_ARG
    msg = negf_lib.negf_last_error().decode()
    assert "bytes of device scratch" in msg and "33554432" in msg, msg


def _oracle_tube(oracle, kw, U):
    okw = {k: v for k, v in kw.items() if k not in ("precision",)}
    o = oracle.OracleTube(**okw)
    o.set_potential(U, (U[0], U[-1]))
    return o


def test_noalloc_matches_oracle_mixed_and_shard(negf_lib, oracle):
    import torch
    from electrostatic_b200.negf import CNT, compute_charge

    base = dict(type_id=(17, 0), num_unitcells=30, num_modes=3, contact_mu=(0.0, -0.3), contact_T=(300.0, 300.0),
                eq_integration_pts=(24, 24, 40), noneq_integration_pts=(96,))
    g64 = CNT(**base)
    gmx = CNT(**base, precision="mixed")
    gsh = CNT(**base)
    U = _potential(g64.site_positions(), 7)
    for t in (g64, gmx, gsh):
        t.set_potential(U, (U[0], U[-1]))
    gsh.set_energy_shard(1, 2)
    o = _oracle_tube(oracle, base, U)
    Qo = o.charge(nthreads=4)
    N = g64.num_field_sites
    out = torch.empty(N, dtype=torch.float64, device="cuda")

    def run(t):
        out.fill_(float("nan"))
        h = (C.c_void_p * 1)(t.handle)
        rc = negf_lib.negf_compute_charge_noalloc(h, 1, C.c_void_p(out.data_ptr()), None)
        assert rc == 0, negf_lib.negf_last_error().decode()
        torch.cuda.synchronize()
        return out.cpu().numpy()

    q64 = run(g64)
    assert _rel(q64, Qo) <= TOL, _rel(q64, Qo)
    qmx = run(gmx)
    assert _rel(qmx, Qo) <= MIXED_TOL, _rel(qmx, Qo)
    assert _rel(qmx, compute_charge([gmx])) <= TOL
    # shard 1 of 2: the second half of the point list (RhoEq + poles, then NonEq), no Rho0 subtraction
    qsh = run(gsh)
    n_eq = len(o.paths(1)[0]) + len(o.paths(2)[0])
    n_ne = len(o.paths(3)[0])
    lo, hi = (n_eq + n_ne) // 2, n_eq + n_ne
    ref = np.zeros(N)
    if lo < n_eq:
        ref += o.partial(1, lo, n_eq)
    ref += o.partial(3, max(lo, n_eq) - n_eq, hi - n_eq)
    assert _rel(qsh, ref) <= TOL, _rel(qsh, ref)
    assert _rel(qsh, compute_charge([gsh])) <= TOL
