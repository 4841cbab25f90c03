"""GPU parity: the sm_100a kernels (through the C-ABI) against the FP64 oracle.

Bar (FP64 path): ||Q_gpu - Q_oracle||_inf / ||Q_oracle||_inf <= 1e-8.
Bar (mixed path): the same norm-wise relative error <= 1e-5.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-8
MIXED_TOL = 1e-5


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def _potential(N, y_nm, seed, amp=0.4):
    """Seeded sum of 5 Gaussian bumps plus a linear ramp (the benchmark recipe)."""
    rng = np.random.default_rng(seed)
    L = y_nm[-1] - y_nm[0]
    U = np.zeros(N)
    for _ in range(5):
        A = rng.uniform(-amp, amp)
        w = rng.uniform(2.0, 10.0)
        c = rng.uniform(y_nm[0], y_nm[-1])
        U += A * np.exp(-((y_nm - c) ** 2) / (2 * w * w))
    U += 0.5 * (y_nm - y_nm[0]) / L
    return U


def _pair(oracle, seed=0, U=None, Uc=None, **kw):
    from electrostatic_b200.negf import CNT
    g = CNT(**kw)
    okw = {k: v for k, v in kw.items() if k not in ("precision", "mixed_fp64_band", "mixed_realaxis_fp32")}
    if "noneq_percent_intercuts" not in okw:
        okw["noneq_percent_intercuts"] = None
    o = oracle.OracleTube(**okw)
    assert g.num_field_sites == o.N
    if U is None:
        U = _potential(g.num_field_sites, g.site_positions(), seed)
    if Uc is None:
        Uc = (U[0], U[-1])
    g.set_potential(U, Uc)
    o.set_potential(U, Uc)
    return g, o


CASES = {
    # equilibrium with Matsubara poles (config-1 shape, shorter tube)
    "equilibrium_poles": dict(type_id=(17, 0), num_unitcells=10, num_modes=2, contact_mu=(-1.0, -1.0),
                              contact_T=(300.0, 300.0), eq_integration_pts=(32, 32, 32), E_pole_max=3.0),
    # bias: three Gauss-Legendre non-equilibrium paths with intercuts
    "bias_gl_paths": dict(type_id=(17, 0), num_unitcells=25, num_modes=3, contact_mu=(0.0, -0.4),
                          contact_T=(300.0, 300.0), eq_integration_pts=(24, 24, 40), noneq_integration_pts=(30, 60, 30),
                          noneq_percent_intercuts=(25.0, 75.0)),
    # explicit uniform real-axis window (config-2 shape, shorter)
    "window_regular": dict(type_id=(17, 0), num_unitcells=50, num_modes=8, contact_mu=(0.0, -0.5),
                           contact_T=(300.0, 300.0), eq_integration_pts=(64, 64, 128), E_zPlus_imag=1e-4,
                           realaxis_window=(-1.5, 1.5, 768, 0)),
    # tiny tube: one partial checkpoint segment
    "tiny_N4": dict(type_id=(17, 0), num_unitcells=1, num_modes=2, contact_mu=(0.1, -0.2), contact_T=(300.0, 300.0),
                    eq_integration_pts=(8, 8, 8), noneq_integration_pts=(40,)),
    # N not a multiple of the 16-site segment, chiral tube (2 rings per unit cell)
    "chiral_N34": dict(type_id=(13, 2), num_unitcells=17, num_modes=3, contact_mu=(0.05, -0.15),
                       contact_T=(300.0, 300.0), eq_integration_pts=(16, 16, 16), noneq_integration_pts=(64,)),
    # different contact temperatures -> non-equilibrium without bias
    "temperatures": dict(type_id=(19, 0), num_unitcells=12, num_modes=4, contact_mu=(-0.2, -0.2),
                         contact_T=(300.0, 450.0), eq_integration_pts=(20, 20, 20), noneq_integration_pts=(80,)),
    # lead surface GF by decimation (use_decimation=1)
    "decimation": dict(type_id=(17, 0), num_unitcells=8, num_modes=2, contact_mu=(0.0, -0.3), contact_T=(300.0, 300.0),
                       eq_integration_pts=(16, 16, 16), noneq_integration_pts=(48,), use_decimation=1),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_charge_fp64_matches_oracle(oracle, name):
    g, o = _pair(oracle, seed=hash(name) % 1000, **CASES[name])
    Qg = g.Solve_NEGF()
    Qo = o.charge(nthreads=8)
    assert np.all(np.isfinite(Qg))
    assert _rel(Qg, Qo) <= FP64_TOL, _rel(Qg, Qo)


def test_faithful_reference_walk_small(oracle):
    """Against the oracle's faithful O(N^2) contact walk (the reference kernel's form)."""
    g, o = _pair(oracle, seed=5, **CASES["bias_gl_paths"])
    Qg = g.Solve_NEGF()
    Qf = o.charge(faithful=True, nthreads=8)
    assert _rel(Qg, Qf) <= FP64_TOL


def test_mixed_precision_error_bound(oracle):
    kw = dict(CASES["window_regular"], precision="mixed")
    g, o = _pair(oracle, seed=11, **kw)
    Qg = g.Solve_NEGF()
    from electrostatic_b200.negf import last_stats
    st = last_stats()
    assert st["updates_fp32"] > 0
    Qo = o.charge(nthreads=8)
    assert _rel(Qg, Qo) <= MIXED_TOL, _rel(Qg, Qo)


@pytest.mark.parametrize("cells", [25, 400])
def test_mixed_precision_broadened_real_axis(oracle, cells):
    """Broadened real axis (eta = 2 meV): the contour points run in FP32, the
    real-axis chains (running products over the whole tube) stay FP64."""
    kw = dict(type_id=(17, 0), num_unitcells=cells, num_modes=3, contact_mu=(0.0, -0.4), contact_T=(300.0, 300.0),
              eq_integration_pts=(24, 24, 40), noneq_integration_pts=(40, 60, 40),
              noneq_percent_intercuts=(30.0, 70.0), E_zPlus_imag=2e-3, precision="mixed")
    g, o = _pair(oracle, seed=13, **kw)
    Qg = g.Solve_NEGF()
    from electrostatic_b200.negf import last_stats
    st = last_stats()
    assert st["updates_fp32"] == st["contour_updates"] > 0
    Qo = o.charge(nthreads=8)
    assert np.all(np.isfinite(Qg))
    assert _rel(Qg, Qo) <= MIXED_TOL, _rel(Qg, Qo)


@pytest.mark.parametrize("cells", [25, 400])
def test_mixed_precision_fp32_real_axis(oracle, cells):
    """mixed_realaxis_fp32: the real-axis chains at eta = 2 meV (above the
    1 meV band) run in FP32 too, within the mixed tolerance."""
    kw = dict(type_id=(17, 0), num_unitcells=cells, num_modes=3, contact_mu=(0.0, -0.4), contact_T=(300.0, 300.0),
              eq_integration_pts=(24, 24, 40), noneq_integration_pts=(40, 60, 40),
              noneq_percent_intercuts=(30.0, 70.0), E_zPlus_imag=2e-3, precision="mixed", mixed_realaxis_fp32=True)
    g, o = _pair(oracle, seed=13, **kw)
    Qg = g.Solve_NEGF()
    from electrostatic_b200.negf import last_stats
    st = last_stats()
    assert st["updates_fp32"] > st["contour_updates"] > 0
    Qo = o.charge(nthreads=8)
    assert np.all(np.isfinite(Qg))
    assert _rel(Qg, Qo) <= MIXED_TOL, _rel(Qg, Qo)


def test_mixed_precision_band_edge_chains_stay_fp64(oracle):
    """A real-axis grid point on a lead band edge of mode 0: that chain stays
    FP64 in mixed mode (its other modes, and every chain further than the
    1 meV band from every edge, run in FP32), and the charge stays within the
    mixed tolerance of the FP64 oracle."""
    from electrostatic_b200.negf import CNT, last_stats
    base = dict(type_id=(17, 0), num_unitcells=60, num_modes=3, contact_mu=(0.05, -0.05), contact_T=(300.0, 300.0),
                eq_integration_pts=(16, 16, 24), E_zPlus_imag=2e-3)
    probe = CNT(**base)
    _, _, beta = probe.modes()
    gamma = 2.5
    edge = abs(abs(beta[0]) - gamma)  # inner band edge of mode 0 (contact potential 0)
    pts, half = 101, 0.075  # spacing 1.5 meV: only the centre point lies within 1 meV of the edge
    kw = dict(base, realaxis_window=(edge - half, edge + half, pts, 0), precision="mixed", mixed_realaxis_fp32=True)
    y = probe.site_positions()
    U = 0.15 * np.exp(-((y - y.mean()) ** 2) / 20.0)
    U[0] = U[-1] = 0.0
    g, o = _pair(oracle, U=U, Uc=(0.0, 0.0), **kw)
    Qg = g.Solve_NEGF()
    st = last_stats()
    E = np.linspace(edge - half, edge + half, pts)
    edges = [e for b in beta for e in (abs(abs(b) - gamma), abs(b) + gamma, -abs(abs(b) - gamma), -(abs(b) + gamma))]
    near = sum(1 for x in E for m, b in enumerate(beta)
               if any(abs(x - e) < 1e-3 for e in (abs(abs(b) - gamma), abs(b) + gamma, -abs(abs(b) - gamma),
                                                   -(abs(b) + gamma))))
    assert near >= 1 and any(abs(E[pts // 2] - e) < 1e-12 for e in edges)
    n_real32 = (pts * len(beta) - near) * g.num_field_sites
    assert st["updates_fp32"] == st["contour_updates"] + n_real32, (st, near)
    Qo = o.charge(nthreads=8)
    assert _rel(Qg, Qo) <= MIXED_TOL, _rel(Qg, Qo)


def test_batch_of_uneven_tubes(oracle):
    from electrostatic_b200.negf import compute_charge
    specs = [
        dict(type_id=(13, 0), num_unitcells=9, num_modes=2, contact_mu=(0.0, -0.3), contact_T=(300.0, 300.0),
             eq_integration_pts=(12, 12, 16), noneq_integration_pts=(40,)),
        dict(type_id=(17, 0), num_unitcells=30, num_modes=5, contact_mu=(0.0, -0.3), contact_T=(300.0, 300.0),
             eq_integration_pts=(16, 16, 24), noneq_integration_pts=(70,)),
        dict(type_id=(19, 0), num_unitcells=4, num_modes=3, contact_mu=(-0.5, -0.5), contact_T=(300.0, 300.0),
             eq_integration_pts=(20, 20, 20), E_pole_max=2.0),
    ]
    pairs = [_pair(oracle, seed=20 + i, **s) for i, s in enumerate(specs)]
    Q = compute_charge([p[0] for p in pairs])
    off = 0
    for g, o in pairs:
        Qo = o.charge(nthreads=8)
        assert _rel(Q[off:off + g.num_field_sites], Qo) <= FP64_TOL
        off += g.num_field_sites


def test_energy_shards_sum_to_full(oracle):
    g, _ = _pair(oracle, seed=3, **CASES["bias_gl_paths"])
    full = g.Solve_NEGF()
    parts = []
    for r in range(3):
        g.set_energy_shard(r, 3)
        parts.append(g.Compute_InducedCharge())
    g.set_energy_shard(0, 1)
    assert _rel(sum(parts), full) <= 1e-12
    # more shards than points: shard 1 of 2P+1 holds no point and (rank != 0) no Rho0
    pts = g.get_Total_Integration_Pts() + len(g.energy_points(1)[0])
    g.set_energy_shard(1, 2 * pts + 1)
    assert np.all(g.Compute_InducedCharge() == 0.0)
    g.set_energy_shard(0, 1)


def test_deterministic_bitwise():
    from electrostatic_b200.negf import CNT
    g = CNT(**CASES["window_regular"])
    U = _potential(g.num_field_sites, g.site_positions(), 9)
    g.set_potential(U)
    a = g.Solve_NEGF()
    b = g.Solve_NEGF()
    assert np.array_equal(a, b)


def test_flat_band_charge_vanishes():
    from electrostatic_b200.negf import CNT
    g = CNT(type_id=(17, 0), num_unitcells=6, num_modes=2, eq_integration_pts=(60, 60, 60))
    g.set_potential(np.zeros(g.num_field_sites), (0.0, 0.0))
    Q = g.Solve_NEGF()
    assert np.max(np.abs(Q)) < 1e-3


def test_contact_mu_update_rebuilds_paths(oracle):
    g, o = _pair(oracle, seed=4, **CASES["tiny_N4"])
    g.Solve_NEGF()
    g.set_Contact_Electrochemical_Potential((0.2, -0.1))
    o2 = oracle.OracleTube(**{**CASES["tiny_N4"], "contact_mu": (0.2, -0.1)})
    U = _potential(g.num_field_sites, g.site_positions(), 4)
    g.set_potential(U, (U[0], U[-1]))
    o2.set_potential(U, (U[0], U[-1]))
    assert _rel(g.Solve_NEGF(), o2.charge()) <= FP64_TOL


def test_device_output_and_write_files(tmp_path, oracle):
    import torch
    g, o = _pair(oracle, seed=8, **CASES["tiny_N4"])
    out = torch.zeros(g.num_field_sites, dtype=torch.float64, device="cuda")
    g.Solve_NEGF(out=out)
    torch.cuda.synchronize()
    Q = out.cpu().numpy()
    assert _rel(Q, o.charge()) <= FP64_TOL
    prefix = str(tmp_path / "step0001")
    g.Write_Data(prefix, Q, np.abs(Q))
    lines = open(prefix + "_Qout.dat").read().splitlines()
    assert lines[0].startswith("'axial location / (nm)'")
    vals = np.array([[float(x) for x in ln.split()] for ln in lines[1:]])
    np.testing.assert_allclose(vals[:, 1], Q, rtol=1e-14)
    np.testing.assert_allclose(vals[:, 0], g.site_positions(), rtol=1e-14)
    assert len(open(prefix + "_U.dat").read().splitlines()) == g.num_field_sites


def test_nonfinite_potential_rejected():
    from electrostatic_b200.negf import CNT
    from electrostatic_b200._lib import NEGFError
    g = CNT(num_unitcells=2)
    U = np.zeros(g.num_field_sites)
    U[3] = np.nan
    with pytest.raises(NEGFError, match="non-finite"):
        g.set_potential(U, (0.0, 0.0))


def test_broyden_matches_oracle(oracle):
    import torch
    from electrostatic_b200.negf import Broyden
    rng = np.random.default_rng(12)
    S = 300
    A = rng.normal(0, 0.4 / np.sqrt(S), (S, S))
    b = rng.normal(0, 1e-2, S)
    n0 = np.full(S, 1e-3)
    for norm_type in ("absolute", "relative"):
        ob = oracle.OracleBroyden(n0, max_step=60, fraction=0.1, norm_type=norm_type)
        gb = Broyden(torch.tensor(n0, device="cuda"), max_step=60, fraction=0.1, norm_type=norm_type)
        n_o = n0.copy()
        n_g = torch.tensor(n0, device="cuda")
        for it in range(25):
            out_o = A @ n_o + b
            mo, n_o, _ = ob.step(out_o)
            out_g = torch.tensor(A, device="cuda") @ n_g + torch.tensor(b, device="cuda")
            mg = gb.step(out_g, n_in_out=n_g)
            assert abs(mg - mo) <= 1e-9 * max(abs(mo), 1e-30)
            np.testing.assert_allclose(n_g.cpu().numpy(), n_o, rtol=1e-9, atol=1e-13)
        assert gb.step_number == ob.step_number == 26
        gb.reset(keep_charge=False, init_value=2e-3)
        assert gb.step_number == 1
        ptr_vals = torch.empty(S, dtype=torch.float64, device="cuda")
        ptr_vals.copy_(n_g)


def test_device_reciprocal_accuracy(negf_lib):
    """The kernels' reciprocal (hardware seed + series correction) against 1/x."""
    import ctypes as C
    rng = np.random.default_rng(0)
    x = np.exp(rng.uniform(np.log(1e-30), np.log(1e30), 200000))
    out = np.zeros_like(x)
    dp = C.POINTER(C.c_double)
    assert negf_lib.negf_device_selftest(0, len(x), x.ctypes.data_as(dp), out.ctypes.data_as(dp)) == 0
    rel = np.abs(out * x - 1.0)
    assert rel.max() <= 4 * np.finfo(np.float64).eps, rel.max()
    assert negf_lib.negf_device_selftest(1, len(x), x.ctypes.data_as(dp), out.ctypes.data_as(dp)) == 0
    xf = x.astype(np.float32).astype(np.float64)
    rel32 = np.abs(out * xf - 1.0)
    assert rel32.max() <= 4 * np.finfo(np.float32).eps, rel32.max()
