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
    b = CNT(type_id=(13, 0), num_unitcells=2, num_modes=2, contact_mu=(0.0, -0.3))
    with pytest.raises(NEGFError, match="equilibrium"):
        b.realspace_charge()
