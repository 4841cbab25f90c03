"""Surrogate-model kernels: the BF16 tensor-core GEMM in its four layouts
against FP32 matmul of the same BF16 values, the hand-written backward pass
against autograd of the same operator, and a training smoke test."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", [1, 2, 3])  # tcgen05 (TMA where possible), mma.sync, tcgen05 register-staged
@pytest.mark.parametrize("at,bt", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("M,N,K,batch", [(130, 70, 45, 3), (1, 128, 300, 1), (256, 256, 4, 2), (64, 256, 257, 1),
                                         (200, 136, 160, 2), (128, 128, 2048, 1), (384, 256, 512, 2)])
def test_gemm_layouts(at, bt, M, N, K, batch, path):
    import torch
    from electrostatic_b200 import _lib
    from electrostatic_b200.negf import TUNE_NN_GEMM, set_tuning
    L = _lib.load()
    set_tuning(TUNE_NN_GEMM, path)
    g = torch.Generator().manual_seed(M * 7 + N + K)
    A = torch.randn(batch, *((K, M) if at else (M, K)), generator=g).to(torch.bfloat16)
    B = torch.randn(batch, *((N, K) if bt else (K, N)), generator=g).to(torch.bfloat16)
    C0 = torch.randn(batch, M, N, generator=g)
    Af, Bf = A.float(), B.float()
    ref = (Af.transpose(1, 2) if at else Af) @ (Bf.transpose(1, 2) if bt else Bf) + C0
    dA, dB, dC = A.cuda(), B.cuda(), C0.cuda().contiguous()
    dCb = torch.empty(batch, M, N, dtype=torch.bfloat16, device="cuda")
    lda, ldb = (M if at else K), (K if bt else N)
    vp = lambda t: __import__("ctypes").c_void_p(t.data_ptr())
    rc = L.negf_nn_gemm(at, bt, M, N, K, batch, vp(dA), lda, dA[0].numel(), vp(dB), ldb, dB[0].numel(), vp(dC), N,
                        M * N, vp(dCb), 1, None)
    assert rc == 0
    torch.cuda.synchronize()
    out = dC.cpu()
    set_tuning(TUNE_NN_GEMM, 0)
    assert torch.allclose(out, ref, rtol=1e-5, atol=1e-4 * (1 + ref.abs().max().item()))
    assert torch.allclose(dCb.float().cpu(), out.to(torch.bfloat16).float())


def _torch_reference(model, U, Vg, Vds, y):
    """The same operator in FP32 autograd (BF16-rounded weights and bases)."""
    import torch
    from electrostatic_b200.surrogate import LAYERS
    P = {k: v.detach().to(torch.bfloat16).float().clone().requires_grad_(True) for k, v in model.params.items()}
    F, G = model.F.float(), model.G.float()
    x = model.features(U, Vg, Vds).float()
    h = x @ P["W_lift"] + P["b_lift"]
    B, S = U.shape
    for l in range(LAYERS):
        s1 = h @ P[f"W{l}"]
        hb = h.reshape(B, S, -1)
        hat = torch.einsum("ks,bsc->bkc", F, hb)  # [B][64][W]
        hk = hat.reshape(B, 32, 2 * hb.shape[-1])
        z = torch.einsum("bki,kio->bko", hk, P[f"R{l}"]).reshape(B, 64, -1)
        s2 = torch.einsum("sk,bkc->bsc", G, z).reshape(B * S, -1)
        h = torch.nn.functional.gelu(s1 + s2 + P[f"b{l}"], approximate="tanh")
    q = h @ P["w_p"] + P["b_p"]
    loss = ((q - y) ** 2).mean()
    loss.backward()
    return {k: v.grad for k, v in P.items()}, loss.item()


def test_backward_matches_autograd():
    import torch
    from electrostatic_b200.surrogate import FourierOperator
    S, B = 256, 2
    m = FourierOperator(S, seed=3)
    g = torch.Generator().manual_seed(0)
    U = (0.3 * torch.randn(B, S, generator=g)).cuda()
    Vg, Vds = torch.tensor([0.2, 0.5]).cuda(), torch.tensor([0.1, 0.4]).cuda()
    y = (0.1 * torch.randn(B * S, generator=g)).cuda()
    ref, _ = _torch_reference(m, U, Vg, Vds, y)
    q = m.forward(m.features(U, Vg, Vds), B, keep=True)
    dq, _ = m.loss_grad(q, y)
    m.backward(dq, B)
    torch.cuda.synchronize()
    for k in ("W_lift", "b_lift", "W0", "R0", "b0", "W5", "R5", "w_p", "b_p"):
        a, r = m.grads[k].cpu().float(), ref[k].cpu().float()
        rel = (a - r).norm() / max(r.norm().item(), 1e-12)
        assert rel < 5e-2, (k, float(rel))


def test_training_reduces_loss():
    import torch
    from electrostatic_b200.surrogate import FourierOperator
    S, n = 256, 32
    g = torch.Generator().manual_seed(1)
    U = (0.3 * torch.randn(n, S, generator=g)).cuda()
    Vg, Vds = torch.rand(n, generator=g).cuda(), torch.rand(n, generator=g).cuda()
    Q = (torch.tanh(U) * 0.02 + 0.01 * Vg[:, None]).double()
    m = FourierOperator(S, seed=5)
    r = m.fit(U, Vg, Vds, Q, epochs=30, batch=8, lr=2e-3)
    assert r["loss"][-1] < 0.2 * r["loss"][0]
    pred = m.predict(U, Vg, Vds)
    assert pred.shape == Q.shape and torch.isfinite(pred).all()


def test_surrogate_started_sweep_is_judged_by_negf():
    """Pipeline on a small tube: pairs from self-consistent solves of the
    engine, a short training, and a surrogate-started gate sweep whose
    converged charges are NEGF fixed points (same tolerance as the plain
    sweep)."""
    import numpy as np
    from electrostatic_b200 import surrogate as S
    from electrostatic_b200.negf import CNT
    from electrostatic_b200.workloads import gate_with_contacts
    U, Vg, Vds, Q, _ = S.generate_scf_pairs(96, unitcells=32, modes=2, vds_bins=3)
    assert U.shape == (96, 128) and np.isfinite(Q.cpu().numpy()).all()
    m = S.FourierOperator(128, seed=0)
    m.fit(U, Vg, Vds, Q, epochs=4, batch=8)
    tube = CNT(**S.tube_kwargs(0.3, unitcells=32, modes=2))
    R = 1.42e-10 * np.sqrt(3.0) * 17 / (2 * np.pi)
    el = gate_with_contacts(tube.site_positions(), R, vds=0.3)
    plain = S.scf_sweep(tube, el, [0.1, 0.3], 0.3)
    sur = S.scf_sweep(tube, el, [0.1, 0.3], 0.3, model=m, keep_history=False)
    for a, b in zip(plain, sur):
        assert np.max(np.abs(a["Q"] - b["Q"])) < 1e-5


def test_fixed_point_surrogate_set_sweep():
    """Tube-set pipeline on three small tubes: fixed-point pairs from batched
    self-consistent solves (per-tube secant updates), a short training, and a
    surrogate-started mixed-precision sweep whose converged charges are NEGF
    fixed points of the FP64 plain sweep (same 1e-6 residual; the mixed
    precision's own error stays below 1e-5 of the charge)."""
    import numpy as np
    from electrostatic_b200.electrostatics import GateAllAround
    from electrostatic_b200.negf import CNT
    from electrostatic_b200.scf import run_scf_batch
    from electrostatic_b200.surrogate_set import (TubeSetOperator, fixed_point_sweep, generate_fixed_points,
                                                  tube_descriptor)
    specs = [((17, 0), 24, 2), ((13, 0), 40, 3), ((19, 0), 16, 2)]

    def make(lv, precision="fp64"):
        return [CNT(type_id=ch, num_unitcells=uc, num_modes=m, contact_mu=(0.0, -float(lv)), contact_T=(300.0, 300.0),
                    eq_integration_pts=(24, 24, 32), noneq_integration_pts=(64,), E_zPlus_imag=2e-3, E_pole_max=3.0,
                    precision=precision, mixed_realaxis_fp32=precision == "mixed") for ch, uc, m in specs]

    tubes = make(0.2)
    electros = [GateAllAround(t.site_positions(), 0.0665e-9 * ch[0] / 17 * 10,
                              1.5e-9 + 0.0665e-9 * ch[0] / 17 * 10, contact_length=1e-9, Vds=0.2)
                for t, (ch, _, _) in zip(tubes, specs)]
    U, Vg, Vds, tid, Q, secs, its = generate_fixed_points(make, electros, 96, vds_bins=2, vds_max=0.2, vg_max=0.3,
                                                          fraction=0.1, bump_amp=0.05, tol=1e-5)
    assert U.shape[0] == 96 and np.isfinite(Q.cpu().numpy()).all() and secs > 0
    assert len([i for i in its if i > 0]) == 32
    for e in electros:
        e.Vds = 0.2
    model = TubeSetOperator([tube_descriptor(t) for t in tubes], seed=0)
    model.fit_set(U, Vg, Vds, tid, Q, epochs=3, batch=16)
    mixed = make(0.2, "mixed")
    vg = [0.1, 0.2, 0.3]
    plain = run_scf_batch(tubes, electros, vg, use_graph=True, iters_per_graph=4)
    for start in ("extrapolated", "difference", "surrogate", "extrapolation", "continuation", "zero"):
        out, alpha, lam, _ = fixed_point_sweep(mixed, electros, vg, model, start=start,
                                               fraction=None if start == "surrogate" else 0.2)
        assert 0.05 <= alpha <= 0.2 and (lam is not None) == (start == "surrogate")
        for r, p in zip(out, plain.steps):
            assert r["negf_iterations"] > 0
            assert np.max(np.abs(r["Q"] - p.Q)) <= 1e-5 * np.max(np.abs(p.Q)) + 2e-6
    # segments with the plain solver's settings: the same fixed points
    seg = run_scf_batch(make(0.2), electros, vg, use_graph=True, iters_per_graph=4, segments=True)
    for a, b in zip(seg.steps, plain.steps):
        assert np.max(np.abs(a.Q - b.Q)) <= 2e-6
    for t in tubes + mixed:
        t.close()
