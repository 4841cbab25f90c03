"""GPU parity at the benchmarked sizes: the sm_100a kernels (through the
C-ABI) against the FP64 oracle on the exact workloads that bench.py times.

* config 2: (17,0) N = 4000, 8 modes, 1024 contour + 3072 real-axis points
  (eta = 1e-4 eV), seeded potential; FP64 and mixed precision.
* config 3: (13,0), 600 ring blocks of 26 atoms, 2048 contour points + poles,
  real-space ring-block RGF against the dense block-RGF oracle; FP64 and mixed.
* config 4: the full uneven 16-tube batch, one charge pass, FP64 and mixed.

Bars: ||Q_gpu - Q_oracle||_inf / ||Q_oracle||_inf <= 1e-8 (FP64 path) and
<= 1e-5 (mixed path), the same norm-wise bounds as the small-case tests.  The
oracle runs on every host core (its O(N) mode for the mode-space cases).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-8
MIXED_TOL = 1e-5
THREADS = max(1, len(os.sched_getaffinity(0)))


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _oracle_kwargs(kw):
    o = {k: v for k, v in kw.items() if k not in ("precision", "mixed_fp64_band", "mixed_realaxis_fp32")}
    o.setdefault("noneq_percent_intercuts", None)
    return o


@pytest.fixture(scope="module")
def config2(oracle):
    from electrostatic_b200.workloads import SEED_BASE, config2_kwargs, site_potential
    kw = config2_kwargs()
    o = oracle.OracleTube(**_oracle_kwargs(kw))
    from electrostatic_b200.negf import CNT
    g = CNT(**kw)
    U = site_potential(g.site_positions(), SEED_BASE + 2)
    o.set_potential(U, (U[0], U[-1]))
    return kw, U, o.charge(nthreads=THREADS)


def test_config2_fp64_matches_oracle(negf_lib, config2):
    from electrostatic_b200.negf import CNT
    kw, U, Qo = config2
    g = CNT(**kw)
    assert g.num_field_sites == 4000
    Qg = g.Solve_NEGF(U, (U[0], U[-1]))
    err = _rel(Qg, Qo)
    print(f"config 2 FP64: max rel vs oracle {err:.3e}")
    assert err <= FP64_TOL, err


def test_config2_mixed_matches_oracle(negf_lib, config2):
    from electrostatic_b200.negf import CNT
    kw, U, Qo = config2
    g = CNT(**dict(kw, precision="mixed"))
    Qg = g.Solve_NEGF(U, (U[0], U[-1]))
    err = _rel(Qg, Qo)
    print(f"config 2 mixed: max rel vs oracle {err:.3e}")
    assert err <= MIXED_TOL, err


@pytest.fixture(scope="module")
def config3(oracle):
    from electrostatic_b200.negf import CNT
    from electrostatic_b200.workloads import SEED_BASE, config3_kwargs, site_potential
    kw = config3_kwargs()
    g = CNT(**kw)
    U = site_potential(g.site_positions(), SEED_BASE + 3)
    o = oracle.OracleTube(**_oracle_kwargs(kw))
    o.set_potential(U, (U[0], U[-1]))
    return kw, U, o.rs_charge(nthreads=THREADS)


@pytest.mark.parametrize("precision,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
def test_config3_realspace_matches_block_oracle(negf_lib, config3, precision, tol):
    from electrostatic_b200.negf import CNT
    kw, U, Qo = config3
    g = CNT(**dict(kw, precision=precision))
    assert g.num_field_sites == 1200  # 600 blocks of two rings
    g.set_potential(U, (U[0], U[-1]))
    Qg = g.realspace_charge()
    err = _rel(Qg, Qo)
    print(f"config 3 {precision}: max rel vs block oracle {err:.3e}")
    assert err <= tol, err


def test_config3_biased_realspace_matches_mode_space_and_oracle(negf_lib, oracle):
    """The config-3 tube at a 0.3 V drain bias (contacts at -0.8 / -1.1 eV,
    3072 real-axis points at 1e-4 eV broadening, the biased workload bench.py
    times): the real-space pass, whose source and drain columns of G travel
    through 600 ring blocks, equals the mode-space pass over all 7 modes and
    the oracle's mode-space charge (equal for this ring-uniform potential).
    At this broadening the block products on the real axis are differences of
    large terms: a mirrored (assumed symmetric) product tile moved this charge
    by 40x its size, which the small biased cases did not show."""
    from electrostatic_b200.negf import CNT
    from electrostatic_b200.workloads import SEED_BASE, config3_kwargs, site_potential
    kw = config3_kwargs()
    kw.pop("precision")
    kb = dict(kw, contact_mu=(-0.8, -1.1), noneq_integration_pts=(3072,), E_zPlus_imag=1e-4)
    g = CNT(**kb)
    assert g.num_field_sites == 1200
    U = site_potential(g.site_positions(), SEED_BASE + 3)
    g.set_potential(U, (U[0], U[-1]))
    assert g.noneq()
    Qr = g.realspace_charge()
    Qm = g.Solve_NEGF()
    o = oracle.OracleTube(**_oracle_kwargs(kb))
    o.set_potential(U, (U[0], U[-1]))
    Qo = o.charge(nthreads=THREADS)
    err_m, err_o = _rel(Qr, Qm), _rel(Qr, Qo)
    print(f"config 3 biased: real space vs mode space {err_m:.3e}, vs oracle {err_o:.3e}")
    assert err_m <= FP64_TOL and err_o <= FP64_TOL, (err_m, err_o)


@pytest.fixture(scope="module")
def config4(oracle):
    from electrostatic_b200.workloads import SEED_BASE, site_potential, uneven_batch
    descs = uneven_batch(precision="fp64")
    Us, Qs = [], []
    for i, d in enumerate(descs):
        o = oracle.OracleTube(**_oracle_kwargs(d))
        y = _positions(d)
        U = site_potential(y, SEED_BASE + 4 + 100 * i)
        o.set_potential(U, (U[0], U[-1]))
        Us.append(U)
        Qs.append(o.charge(nthreads=THREADS))
    return descs, Us, np.concatenate(Qs)


def _positions(d):
    """Axial ring positions [nm] of a zigzag tube (CNT.cpp:93-132)."""
    acc, uc = 1.42e-10, d["num_unitcells"]
    y0 = -(uc / 2.0) * 3.0 * acc - acc / 2.0
    ring = np.array([acc, 1.5 * acc, 2.5 * acc, 3.0 * acc])
    r = np.arange(4 * uc)
    return (ring[r % 4] + 3 * acc * (r // 4) + y0) / 1e-9


@pytest.mark.parametrize("precision,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
def test_config4_batch_pass_matches_oracle(negf_lib, config4, precision, tol):
    import torch
    from electrostatic_b200.negf import CNT, ChargePlan, compute_charge
    descs, Us, Qo = config4
    tubes = [CNT(**dict(d, precision=precision)) for d in descs]
    for t, U in zip(tubes, Us):
        np.testing.assert_allclose(t.site_positions(), _positions({"num_unitcells": t.num_field_sites // 4}),
                                   rtol=0, atol=1e-12)
        t.set_potential(U, (U[0], U[-1]))
    Qg = compute_charge(tubes)
    err = _rel(Qg, Qo)
    # the charge plan (the launch the SCF loop replays) gives the same charge
    Qp = torch.zeros(len(Qo), dtype=torch.float64, device="cuda")
    plan = ChargePlan(tubes, Qp, autotune=False)
    plan.launch()
    torch.cuda.synchronize()
    errp = _rel(Qp.cpu().numpy(), Qo)
    plan.close()
    print(f"config 4 {precision}: max rel vs oracle {err:.3e} (plan {errp:.3e})")
    assert err <= tol and errp <= tol, (err, errp)
