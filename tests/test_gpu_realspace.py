"""Real-space ring-block RGF on the GPU against the FP64 block-RGF oracle
and against the mode-space engine (a ring-uniform potential decouples the
real-space blocks into the m mode chains)."""
import numpy as np
import pytest

from test_gpu_parity import _pair, _rel

pytestmark = pytest.mark.gpu

TOL = 1e-8


def _eq_kw(m, cells, **extra):
    kw = dict(type_id=(m, 0), num_unitcells=cells, num_modes=m // 2 + 1, contact_mu=(-0.8, -0.8),
              contact_T=(300.0, 300.0), eq_integration_pts=(16, 16, 24), E_pole_max=3.0, E_zPlus_imag=1e-6)
    kw.update(extra)
    return kw


@pytest.mark.parametrize("m,cells", [(13, 4), (7, 3), (16, 2), (3, 3), (4, 2), (10, 2), (15, 2)])
def test_realspace_against_block_oracle(oracle, m, cells):
    g, o = _pair(oracle, seed=31, **_eq_kw(m, cells, num_modes=1))  # the real-space pass uses every atom
    Qg = g.realspace_charge()
    Qo = o.rs_charge(nthreads=8)
    assert _rel(Qg, Qo) <= TOL, _rel(Qg, Qo)
    # the second call reuses the tube's Rho0 (computed by the first): the same charge
    assert np.array_equal(g.realspace_charge(), Qg)


MIXED_TOL = 1e-5


@pytest.mark.parametrize("m,cells", [(13, 6), (8, 4)])
def test_realspace_mixed_against_block_oracle(oracle, m, cells):
    """Mixed mode: contour and pole chains at least mixed_fp64_band above the
    real axis in FP32 with tensor-core products, the rest in FP64."""
    g, o = _pair(oracle, seed=33, **_eq_kw(m, cells, num_modes=1, precision="mixed"))
    E = np.concatenate([g.energy_points(1)[0], g.energy_points(2)[0]])
    assert np.sum(np.abs(E.imag) >= 1e-3) > 0.5 * len(E)  # most chains take the FP32 path
    Qg = g.realspace_charge()
    Qo = o.rs_charge(nthreads=8)
    assert _rel(Qg, Qo) <= MIXED_TOL, _rel(Qg, Qo)


def test_realspace_mixed_long_tube_against_fp64():
    """300 blocks: the FP32 recursion stays within the mixed tolerance of the FP64 pass."""
    from electrostatic_b200.negf import CNT
    from electrostatic_b200.workloads import site_potential
    kw = _eq_kw(13, 150, eq_integration_pts=(64, 64, 96))
    g64, g32 = CNT(**kw), CNT(**kw, precision="mixed")
    U = site_potential(g64.site_positions(), 20261203 + 3)
    for g in (g64, g32):
        g.set_potential(U, (U[0], U[-1]))
    Q64, Q32 = g64.realspace_charge(), g32.realspace_charge()
    assert _rel(Q32, Q64) <= MIXED_TOL, _rel(Q32, Q64)


def test_realspace_per_atom_potential(oracle):
    import torch
    g, o = _pair(oracle, seed=32, **_eq_kw(13, 3))
    rng = np.random.default_rng(4)
    Ua = (np.repeat(np.asarray(g_U(g)), 13) + 0.05 * rng.standard_normal(g.num_field_sites * 13)).reshape(-1, 13)
    Qg = g.realspace_charge(U_atoms=torch.tensor(Ua, device="cuda"))
    Qo = o.rs_charge(Uatoms=Ua, nthreads=8)
    assert _rel(Qg, Qo) <= TOL, _rel(Qg, Qo)


def g_U(g):
    from electrostatic_b200.scf import device_view
    return device_view(g.potential_device_ptr(), g.num_field_sites).cpu().numpy()


def test_realspace_equals_all_modes_mode_space():
    """Full-length check of the invariant: 300 blocks, all 7 modes of (13,0)."""
    from electrostatic_b200.negf import CNT
    from electrostatic_b200.workloads import site_potential
    g = CNT(**_eq_kw(13, 150, eq_integration_pts=(32, 32, 48)))
    U = site_potential(g.site_positions(), 20261203 + 3)
    g.set_potential(U, (U[0], U[-1]))
    Qr = g.realspace_charge()
    Qm = g.Solve_NEGF()
    assert _rel(Qr, Qm) <= TOL, _rel(Qr, Qm)


def test_realspace_rejections():
    from electrostatic_b200._lib import NEGFError
    from electrostatic_b200.negf import CNT
    t = CNT(type_id=(17, 0), num_unitcells=2, num_modes=2, contact_mu=(-0.8, -0.8))
    with pytest.raises(NEGFError, match="at most 32 atoms"):
        t.realspace_charge()


def _bias_kw(m, cells, **extra):
    kw = dict(type_id=(m, 0), num_unitcells=cells, num_modes=1, contact_mu=(0.0, -0.3), contact_T=(300.0, 320.0),
              eq_integration_pts=(16, 16, 24), noneq_integration_pts=(48,), E_pole_max=3.0, E_zPlus_imag=1e-4)
    kw.update(extra)
    return kw


@pytest.mark.parametrize("m,cells", [(13, 4), (7, 3), (16, 2), (4, 3), (10, 2), (1, 3)])
def test_realspace_noneq_against_block_oracle(oracle, m, cells):
    """Biased tubes: the real-axis points add the source and drain spectral
    functions (carried through the sweeps as ring-corner columns) against the
    dense-block oracle (left- and right-connected recursions)."""
    g, o = _pair(oracle, seed=35, **_bias_kw(m, cells))
    assert g.noneq()
    Qg = g.realspace_charge()
    Qo = o.rs_charge(nthreads=8)
    assert _rel(Qg, Qo) <= TOL, _rel(Qg, Qo)


def test_realspace_noneq_per_atom_potential_and_mixed(oracle):
    import torch
    kw = _bias_kw(13, 4, contact_mu=(-0.1, -0.5))
    g, o = _pair(oracle, seed=36, **kw)
    rng = np.random.default_rng(6)
    Ua = (np.repeat(np.asarray(g_U(g)), 13) + 0.05 * rng.standard_normal(g.num_field_sites * 13)).reshape(-1, 13)
    Qo = o.rs_charge(Uatoms=Ua, nthreads=8)
    Qg = g.realspace_charge(U_atoms=torch.tensor(Ua, device="cuda"))
    assert _rel(Qg, Qo) <= TOL, _rel(Qg, Qo)
    gm, _ = _pair(oracle, seed=36, **kw, precision="mixed")
    Qm = gm.realspace_charge(U_atoms=torch.tensor(Ua, device="cuda"))
    assert _rel(Qm, Qo) <= MIXED_TOL, _rel(Qm, Qo)


def test_realspace_noneq_equals_all_modes_mode_space():
    """A biased 300-block (13,0) tube with a ring-uniform potential: the
    real-space charge equals the mode-space charge over all 7 modes."""
    from electrostatic_b200.negf import CNT
    from electrostatic_b200.workloads import site_potential
    g = CNT(**_bias_kw(13, 150, num_modes=7, eq_integration_pts=(32, 32, 48), noneq_integration_pts=(96,)))
    U = site_potential(g.site_positions(), 20261203 + 5)
    g.set_potential(U, (U[0], U[-1]))
    Qr = g.realspace_charge()
    Qm = g.Solve_NEGF()
    assert _rel(Qr, Qm) <= TOL, _rel(Qr, Qm)


def _tiles(negf_lib, which, m, data, count, out_per):
    import ctypes as C
    buf = np.concatenate([[m, count], data.ravel()])
    out = np.zeros(max(len(buf), 2 + out_per * count))
    dp = C.POINTER(C.c_double)
    inp = np.zeros_like(out)
    inp[: len(buf)] = buf
    assert negf_lib.negf_device_selftest(which, len(out), inp.ctypes.data_as(dp), out.ctypes.data_as(dp)) == 0
    r = out[2: 2 + out_per * count].reshape(count, m, m, 2)
    return r[..., 0] + 1j * r[..., 1]


def _cplx_pack(M):
    return np.stack([M.real, M.imag], axis=-1)


@pytest.mark.parametrize("m", [4, 13, 16])
def test_tile_inversion_and_products(negf_lib, m):
    """The chain kernels' m x m primitives: inversion on the diagonal pivots
    with the partial-pivoting fall-back (FP64 and FP32), products on the FP64
    cores and on the TF32 tensor cores (three-multiply complex form with
    high/remainder operand splits), against numpy."""
    rng = np.random.default_rng(m)
    n = 24
    # like E - H - Sigma: complex symmetric, positive definite imaginary part
    A = rng.standard_normal((n, m, m)) + 1j * rng.standard_normal((n, m, m))
    A = 0.3 * (A + np.transpose(A, (0, 2, 1)))
    A += np.eye(m)[None] * (2.0 + 0.5j)
    # matrices whose diagonal pivots are small: the fall-back must pivot
    Bp = rng.standard_normal((8, m, m)) + 0.1j * rng.standard_normal((8, m, m))
    Bp[:, np.arange(m), np.arange(m)] = 1e-5 * (1 + 1j)
    for which, tol in ((2, 1e-12), (3, 2e-4)):
        for M in (A, Bp):
            X = _tiles(negf_lib, which, m, _cplx_pack(M), len(M), 2 * m * m)
            res = np.abs(M @ X - np.eye(m)[None]).max()
            cond = max(np.linalg.cond(Mi) for Mi in M)
            assert res <= tol * max(1.0, cond / 100), (which, res, cond)
    P = rng.standard_normal((n, 2, m, m)) + 1j * rng.standard_normal((n, 2, m, m))
    ref = P[:, 0] @ P[:, 1]
    for which, tol in ((4, 1e-13), (5, 2e-6)):
        Cg = _tiles(negf_lib, which, m, np.stack([_cplx_pack(P[:, 0]), _cplx_pack(P[:, 1])], axis=1), n, 2 * m * m)
        err = np.abs(Cg - ref).max() / np.abs(ref).max()
        assert err <= tol, (which, err)


@pytest.mark.parametrize("bias", [False, True])
def test_realspace_decimation_leads_equal_mode_space(bias):
    """A tube with the reference's decimation leads: the real-space lead
    corners take the same per-mode decimated surface values, so the charge
    equals the mode-space charge over all modes."""
    from electrostatic_b200.negf import CNT
    from electrostatic_b200.workloads import site_potential
    kw = _bias_kw(13, 20, num_modes=7, use_decimation=1) if bias else _eq_kw(13, 20, num_modes=7, use_decimation=1)
    g = CNT(**kw)
    U = site_potential(g.site_positions(), 20261203 + 7, amp=0.2)
    g.set_potential(U, (U[0], U[-1]))
    Qr = g.realspace_charge()
    Qm = g.Solve_NEGF()
    assert _rel(Qr, Qm) <= TOL, _rel(Qr, Qm)
