"""Batched self-consistency on the GPU: charge plans, device-resident Broyden
steps and CUDA-graph replay, against the host loop and the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch(oracle=None, modes=(2, 3, 2), cells=(10, 17, 6), chir=(17, 13, 19), mu=(0.0, -0.2), precision="fp64"):
    from electrostatic_b200.electrostatics import GateAllAround
    from electrostatic_b200.negf import CNT
    tubes, oracles, electros = [], [], []
    for m, uc, ch in zip(modes, cells, chir):
        kw = dict(type_id=(ch, 0), num_unitcells=uc, num_modes=m, contact_mu=mu, contact_T=(300.0, 300.0),
                  eq_integration_pts=(16, 16, 24), noneq_integration_pts=(24,), E_zPlus_imag=1e-5, E_pole_max=3.0)
        t = CNT(precision=precision, **kw)
        y = t.site_positions()
        e = GateAllAround(y, r_tube=0.0665e-9 * ch / 17 * 10, r_gate=1.5e-9 + 0.0665e-9 * ch / 17 * 10)
        tubes.append(t)
        electros.append(e)
        if oracle is not None:
            oracles.append(oracle.OracleTube(**kw))
    return tubes, electros, oracles


def test_plan_matches_compute_charge():
    import torch
    from electrostatic_b200.negf import ChargePlan, compute_charge
    tubes, _, _ = _batch()
    rng = np.random.default_rng(3)
    for t in tubes:
        U = 0.1 * rng.standard_normal(t.num_field_sites)
        t.set_potential(U, (U[0], U[-1]))
    S = sum(t.num_field_sites for t in tubes)
    ref = torch.zeros(S, dtype=torch.float64, device="cuda")
    compute_charge(tubes, out=ref)
    from electrostatic_b200.negf import last_stats
    ref_schedule = last_stats()["schedule"]  # 1 two-pass, 2 fused
    for autotune in (False, True):
        Q = torch.zeros(S, dtype=torch.float64, device="cuda")
        plan = ChargePlan(tubes, Q, autotune=autotune)
        plan.launch()
        torch.cuda.synchronize()
        info = plan.info()
        fused = info["pass2_warps_per_block"] == 0
        if fused == (ref_schedule == 2):
            assert torch.equal(Q, ref)  # same schedule: bitwise
        else:  # the autotuner chose the other schedule: equal to rounding
            assert float((Q - ref).abs().max() / ref.abs().max()) <= 1e-11
        assert info["pass2_warps_per_block"] in (0, 1, 2, 4) and info["segs_per_unit"] in (16, 32, 64)
        plan.close()


def test_plan_stale_after_contact_change():
    import torch
    from electrostatic_b200._lib import NEGFError
    from electrostatic_b200.negf import ChargePlan
    tubes, _, _ = _batch()
    Q = torch.zeros(sum(t.num_field_sites for t in tubes), dtype=torch.float64, device="cuda")
    plan = ChargePlan(tubes, Q)
    tubes[1].set_Contact_Electrochemical_Potential((0.0, -0.3))
    with pytest.raises(NEGFError, match="stale"):
        plan.launch()


def test_device_broyden_matches_host_steps():
    import torch
    from electrostatic_b200.negf import Broyden
    S = 300
    rng = np.random.default_rng(9)
    A = np.eye(S) * 0.5 + 0.01 * rng.standard_normal((S, S))
    b = rng.standard_normal(S)
    n0 = torch.zeros(S, dtype=torch.float64, device="cuda")
    h = Broyden(n0, max_step=50, fraction=0.2)
    d = Broyden(n0, max_step=50, fraction=0.2)
    flags = torch.zeros(4, dtype=torch.int32, device="cuda")
    for _ in range(12):
        xh = torch.from_numpy(A @ _read(h.input_device_ptr(), S) + b).cuda()
        h.step(xh)
        xd = torch.from_numpy(A @ _read(d.input_device_ptr(), S) + b).cuda()
        d.step_device(xd, 1e-30, flags)
    torch.cuda.synchronize()
    assert np.array_equal(_read(h.input_device_ptr(), S), _read(d.input_device_ptr(), S))
    assert flags.cpu().tolist()[:3] == [0, 12, 0] and d.step_number == 13


def test_broyden_initial_jacobian_exact_inverse():
    """Seeded with secant pairs whose residual differences are the unit
    vectors, G0 is the exact inverse Jacobian of a linear map, so the first
    step (host or device-resident) lands on the fixed point."""
    import torch
    from electrostatic_b200._lib import NEGFError
    from electrostatic_b200.negf import Broyden
    S = 16
    rng = np.random.default_rng(11)
    A = 0.3 * rng.standard_normal((S, S)) / np.sqrt(S)  # n_out = A n_in + b
    b = rng.standard_normal(S)
    J = np.eye(S) - A  # F = n_in - n_out = J n_in - b
    nstar = np.linalg.solve(J, b)
    dn = torch.from_numpy(np.linalg.inv(J).T.copy()).cuda()  # dn_j = J^-1 e_j, so dF_j = e_j
    dF = torch.eye(S, dtype=torch.float64, device="cuda")
    V, W = Broyden.secant_rows(dn, dF, fraction=0.2)
    for device in (False, True):
        br = Broyden(torch.zeros(S, dtype=torch.float64, device="cuda"), max_step=40, fraction=0.2)
        br.set_initial_jacobian(V, W)
        x = torch.from_numpy(A @ _read(br.input_device_ptr(), S) + b).cuda()
        if device:
            flags = torch.zeros(4, dtype=torch.int32, device="cuda")
            br.step_device(x, 1e-30, flags)
        else:
            br.step(x)
        n1 = _read(br.input_device_ptr(), S)
        assert np.max(np.abs(n1 - nstar)) <= 1e-10 * np.max(np.abs(nstar))
        with pytest.raises(NEGFError, match="before the first step"):
            br.set_initial_jacobian(V, W)
        br.reset()
        br.set_initial_jacobian(None, None)  # k = 0: the plain simple-mixing start
    small = Broyden(torch.zeros(S, dtype=torch.float64, device="cuda"), max_step=20, fraction=0.2)
    with pytest.raises(NEGFError, match="max_step / 2"):
        small.set_initial_jacobian(V, W)


def _np_broyden(n, F_of, steps, alpha, W=None, V=None, offsets=None):
    """Modified-second Broyden in numpy (Broyden_Second_Parallel.cpp:9-211)
    starting from secant rows W, V; returns the iterates and the rows.
    offsets: per-segment dot products (the segmented update)."""
    W, V = list(W or []), list(V or [])
    Fp = npv = None
    out = []
    off = [0, len(n)] if offsets is None else list(offsets)

    def dot(a, b):  # per-segment a.b broadcast over the segment's sites
        r = np.empty(len(a))
        for lo, hi in zip(off[:-1], off[1:]):
            r[lo:hi] = a[lo:hi] @ b[lo:hi]
        return r

    for _ in range(steps):
        F = F_of(n)
        if Fp is not None:
            dF = F - Fp
            s = sum(w * dot(v, dF) for w, v in zip(W, V)) if W else 0.0
            W.append(-alpha * dF + (n - npv) - s)
            V.append(dF / dot(dF, dF))
        step = alpha * F + (sum(w * dot(v, F) for w, v in zip(W, V)) if W else 0.0)
        Fp, npv = F, n.copy()
        n = n - step
        out.append(n.copy())
    return out, W, V


@pytest.mark.parametrize("keep", [100, 3, 0])
def test_broyden_restart_carries_rows(keep):
    """negf_broyden_restart: a second solve (another linear map, as at the next
    bias point) starts from the first solve's secant rows (all of them when
    they fit in `keep`, else none), matching the numpy twin step by step."""
    import torch
    from electrostatic_b200.negf import Broyden
    S = 24
    rng = np.random.default_rng(7)
    A1 = 0.5 * rng.standard_normal((S, S)) / np.sqrt(S)
    A2 = A1 + 0.05 * rng.standard_normal((S, S)) / np.sqrt(S)
    b1, b2 = rng.standard_normal(S), rng.standard_normal(S)
    alpha = 0.3
    n0 = np.zeros(S)
    it1, W, V = _np_broyden(n0, lambda n: n - (A1 @ n + b1), 6, alpha)
    W, V = (W, V) if len(W) <= keep else ([], [])
    it2, _, _ = _np_broyden(it1[-1], lambda n: n - (A2 @ n + b2), 5, alpha, W, V)
    br = Broyden(torch.zeros(S, dtype=torch.float64, device="cuda"), max_step=60, fraction=alpha)
    for A, b, ref in ((A1, b1, it1), (A2, b2, it2)):
        for k in range(len(ref)):
            x = torch.from_numpy(A @ _read(br.input_device_ptr(), S) + b).cuda()
            br.step(x)
            np.testing.assert_allclose(_read(br.input_device_ptr(), S), ref[k], rtol=1e-9, atol=1e-12)
        br.restart(keep_rows=keep)
        assert br.step_number == 1


@pytest.mark.parametrize("device_steps", [False, True])
def test_broyden_segments_match_numpy(device_steps):
    """negf_broyden_set_segments: per-segment secant updates on a block-diagonal
    linear map (three segments of uneven length) match the numpy twin step by
    step, through host steps and device-resident steps alike; one segment
    [0, S] is the whole-vector update bit for bit."""
    import torch
    from electrostatic_b200.negf import Broyden
    off = [0, 7, 20, 33]
    S = off[-1]
    rng = np.random.default_rng(11)
    A = np.zeros((S, S))
    for lo, hi in zip(off[:-1], off[1:]):
        A[lo:hi, lo:hi] = 0.6 * rng.standard_normal((hi - lo, hi - lo)) / np.sqrt(hi - lo)
    b = rng.standard_normal(S)
    alpha = 0.3
    ref, _, _ = _np_broyden(np.zeros(S), lambda n: n - (A @ n + b), 8, alpha, offsets=off)
    br = Broyden(torch.zeros(S, dtype=torch.float64, device="cuda"), max_step=40, fraction=alpha)
    br.set_segments(off)
    flags = torch.zeros(4, dtype=torch.int32, device="cuda")
    for k in range(len(ref)):
        x = torch.from_numpy(A @ _read(br.input_device_ptr(), S) + b).cuda()
        if device_steps:
            br.step_device(x, 0.0, flags)
        else:
            br.step(x)
        np.testing.assert_allclose(_read(br.input_device_ptr(), S), ref[k], rtol=1e-9, atol=1e-12)
    # one segment: bitwise the default update
    runs = []
    for segs in (None, [0, S]):
        br2 = Broyden(torch.zeros(S, dtype=torch.float64, device="cuda"), max_step=40, fraction=alpha)
        if segs is not None:
            br2.set_segments(segs)
        for k in range(6):
            br2.step(torch.from_numpy(A @ _read(br2.input_device_ptr(), S) + b).cuda())
        runs.append(_read(br2.input_device_ptr(), S))
        br2.close()
    assert np.array_equal(runs[0], runs[1])
    br.close()


def _read(ptr, n):
    from electrostatic_b200.scf import device_view
    return device_view(ptr, n).cpu().numpy()


def test_batch_scf_graph_equals_loop_and_oracle(oracle):
    from electrostatic_b200.scf import run_scf_batch
    from oracle.scf_oracle import run_scf_batch_oracle
    Vg = [0.0, 0.15]
    tubes, electros, oracles = _batch(oracle)
    r_graph = run_scf_batch(tubes, electros, Vg, use_graph=True, iters_per_graph=4, autotune=False)
    tubes2, electros2, _ = _batch()
    r_loop = run_scf_batch(tubes2, electros2, Vg, use_graph=False, autotune=False)
    for a, b in zip(r_graph.steps, r_loop.steps):
        assert a.iterations == b.iterations
        assert np.array_equal(a.Q, b.Q)
    r_o = run_scf_batch_oracle(oracles, [e.K for e in electros], Vg)
    for a, b in zip(r_graph.steps, r_o.steps):
        assert a.iterations == b.iterations
        assert np.max(np.abs(a.Q - b.Q)) <= 1e-8 * np.max(np.abs(b.Q))


def test_broyden_non_finite_residual_is_an_error():
    """A NaN in the NEGF output is never read as convergence."""
    import torch
    from electrostatic_b200._lib import NEGFError
    from electrostatic_b200.negf import Broyden
    S = 100
    x = torch.zeros(S, dtype=torch.float64, device="cuda")
    x[17] = float("nan")
    h = Broyden(torch.zeros(S, dtype=torch.float64, device="cuda"))
    with pytest.raises(NEGFError, match="non-finite"):
        h.step(x)
    d = Broyden(torch.zeros(S, dtype=torch.float64, device="cuda"))
    flags = torch.zeros(4, dtype=torch.int32, device="cuda")
    d.step_device(x, 1e-6, flags)
    assert flags.cpu().tolist() == [0, 1, 2, 1]


def test_batch_scf_precision_switch_matches_fp64(oracle):
    """Mixed-precision tubes with the FP64 finish: the converged charge is an
    FP64 fixed point (same tolerance as the plain FP64 loop)."""
    from electrostatic_b200.scf import run_scf_batch
    Vg = [0.1]
    tubes, electros, _ = _batch(precision="mixed")
    r_sw = run_scf_batch(tubes, electros, Vg, use_graph=True, iters_per_graph=4, switch_norm=1e-4)
    tubes2, electros2, _ = _batch()
    r_64 = run_scf_batch(tubes2, electros2, Vg, use_graph=True, iters_per_graph=4)
    a, b = r_sw.steps[0], r_64.steps[0]
    assert 0 < a.lowprec_iterations < a.iterations
    assert np.max(np.abs(a.Q - b.Q)) < 1e-5


def test_affine_potential_toeplitz_equals_dense():
    """negf_affine_potential_toeplitz (the kernel read from its lattice-distance
    table) equals the dense n x n operator of the same gate-all-around tube."""
    import torch
    from electrostatic_b200.negf import affine_potential_masked, affine_potential_toeplitz
    tubes, electros, _ = _batch(cells=(10, 300, 6))  # 1200 sites: two staged chunks
    for t, e in zip(tubes, electros):
        N = t.num_field_sites
        Kd, U0 = e.device_operator(0.2)
        tab, idx = e.device_toeplitz()
        q = torch.randn(N, dtype=torch.float64, device="cuda", generator=torch.Generator(device="cuda").manual_seed(N))
        Ua = torch.empty(N, dtype=torch.float64, device="cuda")
        Ub = torch.empty(N, dtype=torch.float64, device="cuda")
        affine_potential_masked(Kd, U0, q, Ua, N, None)
        affine_potential_toeplitz(tab, idx, U0, q, Ub, N, None)
        torch.cuda.synchronize()
        assert float((Ua - Ub).abs().max()) <= 1e-12 * float(Ua.abs().max())


def test_potential_batch_equals_dense():
    """negf_potential_batch (every tube's lattice-distance update in one launch)
    equals the dense operators tube by tube."""
    import torch
    from electrostatic_b200.negf import PotentialBatch, affine_potential_masked
    tubes, electros, _ = _batch(cells=(10, 300, 6))
    Ns = [t.num_field_sites for t in tubes]
    offs = np.concatenate([[0], np.cumsum(Ns)]).astype(int)
    q = torch.randn(int(offs[-1]), dtype=torch.float64, device="cuda", generator=torch.Generator(device="cuda").manual_seed(5))
    Ub = torch.zeros(int(offs[-1]), dtype=torch.float64, device="cuda")
    ops = [e.device_operator(0.1) for e in electros]
    toes = [e.device_toeplitz() for e in electros]
    pb = PotentialBatch([t[0] for t in toes], [t[1] for t in toes], [U0 for _, U0 in ops],
                        [q.data_ptr() + 8 * int(o) for o in offs[:-1]], [Ub.data_ptr() + 8 * int(o) for o in offs[:-1]],
                        Ns)
    pb.launch()
    for (Kd, U0), a, b in zip(ops, offs[:-1], offs[1:]):
        Ua = torch.empty(b - a, dtype=torch.float64, device="cuda")
        affine_potential_masked(Kd, U0, q[a:b], Ua, b - a, None)
        torch.cuda.synchronize()
        assert float((Ua - Ub[a:b]).abs().max()) <= 1e-12 * float(Ua.abs().max())
    pb.close()
