"""Surrogate charge model: a 1D Fourier neural operator for the Broyden start.

Maps the site potential U of a tube (plus the gate and drain biases) to the
induced charge Q that the NEGF engine would return.  It is trained on (U, Q)
pairs produced by the engine itself and serves as the initial guess of the
self-consistent loop; the NEGF engine judges every converged charge.  The
reference has no counterpart (its loop starts from a constant charge,
Broyden_Parallel_General.cpp:68-248).

Architecture (channel-last activations, rows = samples x sites):
  lift      h0 = x W_lift + b_lift,                                  24 -> 128
            x = (U at the 17 sites n-8 .. n+8 (0 beyond the ends), Vg, Vds,
                 n / S, ring parity +-1, exp(-n / 40), exp(-(S-1-n) / 40), 0)
  6 layers  h  = GELU(h W_l + G (R_l * (F h)) + b_l)                 128 -> 128
            F: real DFT basis of the first 32 frequencies (cos, sin: 64 rows),
            G: its synthesis basis, R_l: per-frequency 256 x 256 mixing of the
            (cos, sin) coefficient pair over all channels
  project   q  = h w_p + b_p                                          128 -> 1
Every product is a BF16 tensor-core GEMM with FP32 accumulation
(negf_nn_gemm); GELU, bias, loss, reductions and Adam are the library's own
kernels; PyTorch only allocates the device buffers.  Master weights and
optimiser state are FP32, their BF16 copies feed the GEMMs.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import _lib
from ._lib import check

WIDTH, MODES, LAYERS, FEAT = 128, 32, 6, 24
WIN = 8  # half-width of the potential window of each site


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class FourierOperator:
    """The operator for tubes of S sites.  All state lives on the device."""

    def __init__(self, S: int, seed: int = 0, device: str = "cuda", feat: int = FEAT):
        import torch
        self.torch = torch
        self.S, self.dev = int(S), device
        self.feat = int(feat)
        g = torch.Generator().manual_seed(seed)
        W, M = WIDTH, MODES
        f32 = dict(dtype=torch.float32)

        def init(shape, fan_in):
            return (torch.randn(*shape, generator=g, **f32) / math.sqrt(fan_in)).to(device)

        self.params = {
            "W_lift": init((self.feat, W), self.feat),
            "b_lift": torch.zeros(W, device=device, **f32),
            "w_p": init((W,), W),
            "b_p": torch.zeros(1, device=device, **f32),
        }
        for l in range(LAYERS):
            self.params[f"W{l}"] = init((W, W), W)
            self.params[f"R{l}"] = init((M, 2 * W, 2 * W), 2 * W) * 0.5
            self.params[f"b{l}"] = torch.zeros(W, device=device, **f32)
        self.bf = {k: v.to(torch.bfloat16) for k, v in self.params.items()}
        self.grads = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.m = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.step = 0
        # analysis / synthesis bases on the site grid: rows (cos k, sin k), k < 32
        s = np.arange(self.S)
        F = np.zeros((2 * M, self.S))
        for k in range(M):
            F[2 * k] = np.cos(2 * np.pi * k * s / self.S) * (1.0 if k == 0 else 2.0) / self.S
            F[2 * k + 1] = np.sin(2 * np.pi * k * s / self.S) * 2.0 / self.S
        G = np.zeros((self.S, 2 * M))
        for k in range(M):
            G[:, 2 * k] = np.cos(2 * np.pi * k * s / self.S)
            G[:, 2 * k + 1] = np.sin(2 * np.pi * k * s / self.S)
        self.F = torch.tensor(F, dtype=torch.bfloat16, device=device)
        self.G = torch.tensor(G, dtype=torch.bfloat16, device=device)
        # per-sample bases (Fb [B][2M][S], Gb [B][S][2M]) replace F and G when set
        self._basis = None
        self.x_scale = torch.ones(self.feat, device=device)
        self.q_scale = 1.0
        self._bufs = {}
        # window gather: site n reads U[n + d], d = -WIN..WIN, masked to 0 beyond the ends
        nw = 2 * WIN + 1
        j = np.arange(self.S)[:, None] + np.arange(-WIN, WIN + 1)[None, :]
        self._widx = torch.tensor(np.clip(j, 0, self.S - 1).reshape(-1), dtype=torch.long, device=device)
        self._wmask = torch.tensor(((j >= 0) & (j < self.S)).astype(np.float32), device=device)
        # fixed site features: n / S, parity, contact proximity
        n = np.arange(self.S)
        fixed = np.zeros((self.S, self.feat - nw - 2), dtype=np.float32)
        fixed[:, 0] = n / self.S
        fixed[:, 1] = np.where(n % 2 == 0, 1.0, -1.0)
        fixed[:, 2] = np.exp(-n / 40.0)
        fixed[:, 3] = np.exp(-(self.S - 1 - n) / 40.0)
        self._fixed = torch.tensor(fixed, device=device)

    # ------------------------------------------------------------------ helpers
    def _buf(self, name, shape, dtype=None):
        t = self.torch
        dtype = dtype or t.float32
        key = (name, tuple(shape), dtype)
        b = self._bufs.get(key)
        if b is None:
            b = t.empty(*shape, dtype=dtype, device=self.dev)
            self._bufs[key] = b
        return b

    def _s(self):
        """The current torch stream (every kernel of the model runs on it)."""
        return C.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    def _bases(self):
        """Analysis and synthesis bases with their batch strides (0: shared)."""
        if self._basis is None:
            return self.F, 0, self.G, 0
        n = 2 * MODES * self.S
        return self._basis[0], n, self._basis[1], n

    def _gemm(self, at, bt, M, N, K, batch, A, lda, sA, B, ldb, sB, Cf, ldc, sC, Cb=None, acc=0):
        check(_lib.load().negf_nn_gemm(at, bt, M, N, K, batch, _p(A), lda, sA, _p(B), ldb, sB, _p(Cf), ldc, sC, _p(Cb),
                                       acc, self._s()), "negf_nn_gemm")

    # ------------------------------------------------------------------ model
    def features(self, U, Vg, Vds):
        """x[b][s] (see the module docstring), potentials divided by the stored
        potential scale, as BF16 rows [B*S][self.feat]."""
        t = self.torch
        B = U.shape[0]
        nw = 2 * WIN + 1
        x = t.empty(B, self.S, self.feat, device=self.dev)
        x[:, :, :nw] = U.float()[:, self._widx].reshape(B, self.S, nw) * (self._wmask / self.x_scale[0])
        x[:, :, nw] = Vg[:, None]
        x[:, :, nw + 1] = Vds[:, None]
        x[:, :, nw + 2:] = self._fixed
        return x.to(t.bfloat16).reshape(B * self.S, self.feat)

    def forward(self, xb, B, keep=False):
        """xb: BF16 [B*S][4]; returns q [B*S] (FP32, in units of q_scale)."""
        t, L = self.torch, _lib.load()
        S, W, M = self.S, WIDTH, MODES
        R = B * S
        cache = {"xb": xb} if keep else None
        h = self._buf("h0", (R, W))
        hb = self._buf("h0b", (R, W), t.bfloat16)
        self._gemm(0, 0, R, W, self.feat, 1, xb, self.feat, 0, self.bf["W_lift"], W, 0, h, W, 0)
        check(L.negf_nn_gelu_fwd(R, W, _p(h), None, _p(self.params["b_lift"]), None, _p(h), _p(hb), 0, self._s()),
              "lift")
        for l in range(LAYERS):
            s1 = self._buf(f"s1_{l}", (R, W))
            hat = self._buf(f"hat{l}", (B, 2 * M, W))
            hatb = self._buf(f"hatb{l}", (B, 2 * M, W), t.bfloat16)
            z = self._buf(f"z{l}", (B, 2 * M, W))
            zb = self._buf(f"zb{l}", (B, 2 * M, W), t.bfloat16)
            s2 = self._buf(f"s2_{l}", (R, W))
            self._gemm(0, 0, R, W, W, 1, hb, W, 0, self.bf[f"W{l}"], W, 0, s1, W, 0)
            Fa, sF, Ga, sG = self._bases()
            self._gemm(0, 0, 2 * M, W, S, B, Fa, S, sF, hb, W, S * W, hat, W, 2 * M * W, hatb)
            # per frequency k: rows b of hat[b][2k:2k+2][:] (256 values) times R[k]
            self._gemm(0, 0, B, 2 * W, 2 * W, M, hatb, 2 * M * W, 2 * W, self.bf[f"R{l}"], 2 * W, 4 * W * W,
                       z, 2 * M * W, 2 * W, zb)
            self._gemm(0, 0, S, W, 2 * M, B, Ga, 2 * M, sG, zb, W, 2 * M * W, s2, W, S * W)
            pre = self._buf(f"pre{l}", (R, W)) if keep else None
            hn = self._buf(f"h{l + 1}", (R, W))
            hnb = self._buf(f"h{l + 1}b", (R, W), t.bfloat16)
            check(L.negf_nn_gelu_fwd(R, W, _p(s1), _p(s2), _p(self.params[f"b{l}"]), _p(pre), _p(hn), _p(hnb), 1,
                                     self._s()), "gelu")
            if keep:
                cache[l] = (hb, hatb, zb, pre)
            h, hb = hn, hnb
        q = self._buf("q", (R,))
        check(L.negf_nn_rowdot(R, W, _p(h), _p(self.params["w_p"]), _p(self.params["b_p"]), _p(q), self._s()), "proj")
        if keep:
            cache["h_last"], cache["h_lastb"] = h, hb
            self._cache = cache
        return q

    def backward(self, dq, B):
        """Gradients of the loss for dq = dL/dq [B*S] (after forward(keep=True))."""
        t, L = self.torch, _lib.load()
        S, W, M = self.S, WIDTH, MODES
        R = B * S
        c = self._cache
        gr = self.grads
        # projection
        dqb = self._buf("dqb", (R,), t.bfloat16)
        check(L.negf_nn_cast_bf16(R, _p(dq), _p(dqb), self._s()), "cast")
        self._gemm(0, 0, 1, W, R, 1, dqb, R, 0, c["h_lastb"], W, 0, gr["w_p"], W, 0)
        check(L.negf_nn_colsum(R, 1, _p(dq), _p(gr["b_p"]), 0, self._s()), "colsum")
        dh = self._buf("dh", (R, W))
        check(L.negf_nn_outer(R, W, _p(dq), _p(self.params["w_p"]), _p(dh), None, self._s()), "outer")
        for l in reversed(range(LAYERS)):
            hb, hatb, zb, pre = c[l]
            dpre = self._buf("dpre", (R, W))
            dpreb = self._buf("dpreb", (R, W), t.bfloat16)
            check(L.negf_nn_gelu_bwd(R * W, _p(dh), _p(pre), _p(dpre), _p(dpreb), self._s()), "gelu_bwd")
            check(L.negf_nn_colsum(R, W, _p(dpre), _p(gr[f"b{l}"]), 0, self._s()), "colsum")
            # pointwise path: dW = h^T dpre ; dh = dpre W^T
            self._gemm(1, 0, W, W, R, 1, hb, W, 0, dpreb, W, 0, gr[f"W{l}"], W, 0)
            dhn = self._buf("dhn", (R, W))
            self._gemm(0, 1, R, W, W, 1, dpreb, W, 0, self.bf[f"W{l}"], W, 0, dhn, W, 0)
            # spectral path: dz = G^T dpre ; dR_k = hat_k^T dz_k ; dhat_k = dz_k R_k^T ; dh += F^T dhat
            dz = self._buf("dz", (B, 2 * M, W))
            dzb = self._buf("dzb", (B, 2 * M, W), t.bfloat16)
            Fa, sF, Ga, sG = self._bases()
            self._gemm(1, 0, 2 * M, W, S, B, Ga, 2 * M, sG, dpreb, W, S * W, dz, W, 2 * M * W, dzb)
            self._gemm(1, 0, 2 * W, 2 * W, B, M, hatb, 2 * M * W, 2 * W, dzb, 2 * M * W, 2 * W, gr[f"R{l}"], 2 * W,
                       4 * W * W)
            dhat = self._buf("dhat", (B, 2 * M, W))
            dhatb = self._buf("dhatb", (B, 2 * M, W), t.bfloat16)
            self._gemm(0, 1, B, 2 * W, 2 * W, M, dzb, 2 * M * W, 2 * W, self.bf[f"R{l}"], 2 * W, 4 * W * W, dhat,
                       2 * M * W, 2 * W, dhatb)
            self._gemm(1, 0, S, W, 2 * M, B, Fa, S, sF, dhatb, W, 2 * M * W, dhn, W, S * W, None, 1)
            dh, dhn = dhn, dh
            self._bufs[("dh", (R, W), t.float32)], self._bufs[("dhn", (R, W), t.float32)] = dh, dhn
        # lift
        dhb = self._buf("dhb", (R, W), t.bfloat16)
        check(L.negf_nn_cast_bf16(R * W, _p(dh), _p(dhb), self._s()), "cast")
        self._gemm(1, 0, self.feat, W, R, 1, c["xb"], self.feat, 0, dhb, W, 0, gr["W_lift"], W, 0)
        check(L.negf_nn_colsum(R, W, _p(dh), _p(gr["b_lift"]), 0, self._s()), "colsum")

    def adam(self, lr=1e-3, wd=0.0):
        L = _lib.load()
        self.step += 1
        for k, w in self.params.items():
            check(L.negf_nn_adam(w.numel(), _p(w), _p(self.grads[k]), _p(self.m[k]), _p(self.v[k]), _p(self.bf[k]),
                                 lr, 0.9, 0.999, 1e-8, self.step, wd, self._s()), "adam")

    def loss_grad(self, q, y):
        """MSE in units of q_scale; returns (dq, partial sums)."""
        L = _lib.load()
        n = q.numel()
        dq = self._buf("dq", (n,))
        part = self._buf("part", ((n + 255) // 256,))
        check(L.negf_nn_mse(n, _p(q), _p(y), _p(dq), _p(part), self._s()), "mse")
        return dq, part

    # ------------------------------------------------------------------ API
    def fit(self, U, Vg, Vds, Q, epochs=20, batch=16, lr=2e-3, log=None):
        """Train on device tensors U [n][S], Vg [n], Vds [n], Q [n][S] (float32)."""
        t = self.torch
        n = U.shape[0]
        self.x_scale = t.ones(self.feat, device=self.dev)
        self.x_scale[0] = float(U.abs().max())
        self.q_scale = float(Q.abs().max())
        y_all = (Q / self.q_scale).float()
        g = t.Generator(device="cpu").manual_seed(1)
        hist = []
        t0 = time.perf_counter()
        steps = epochs * (n // batch)
        for ep in range(epochs):
            perm = t.randperm(n, generator=g)
            tot = 0.0
            for i in range(n // batch):
                idx = perm[i * batch:(i + 1) * batch].to(self.dev)
                xb = self.features(U[idx], Vg[idx], Vds[idx])
                q = self.forward(xb, batch, keep=True)
                y = y_all[idx].reshape(-1).contiguous()
                dq, part = self.loss_grad(q, y)
                self.backward(dq, batch)
                frac = (ep * (n // batch) + i) / max(1, steps)
                self.adam(lr=lr * 0.5 * (1 + math.cos(math.pi * frac)))
                tot += float(part.sum()) / (batch * self.S)
            hist.append(tot / (n // batch))
            if log:
                log(ep, hist[-1])
        t.cuda.synchronize()
        return {"epochs": epochs, "seconds": time.perf_counter() - t0, "loss": hist}

    def bind(self, U_view, Vg, Vds, Q_out):
        """Fixed buffers for repeated single-sample inference (capturable in a
        CUDA graph after one call of infer()): U_view (float64 device view of a
        potential buffer), scalar biases, Q_out (float64 device, S)."""
        t = self.torch
        nw = 2 * WIN + 1
        self._bind = dict(U=U_view, Q=Q_out, x=t.empty(self.S, self.feat, device=self.dev),
                          xb=t.empty(self.S, self.feat, dtype=t.bfloat16, device=self.dev),
                          win=t.empty(self.S * nw, dtype=t.float64, device=self.dev),
                          wscale=self._wmask / self.x_scale[0])
        x = self._bind["x"]
        x[:, nw + 2:] = self._fixed
        self.set_bias(Vg, Vds)

    def set_bias(self, Vg, Vds):
        nw = 2 * WIN + 1
        x = self._bind["x"]
        x[:, nw] = float(Vg) / float(self.x_scale[nw])
        x[:, nw + 1] = float(Vds) / float(self.x_scale[nw + 1])

    def infer(self):
        """Q_out = model(U_view) with the bound buffers (no allocation after the first call)."""
        t = self.torch
        b = self._bind
        nw = 2 * WIN + 1
        t.index_select(b["U"], 0, self._widx, out=b["win"])
        b["x"][:, :nw].copy_(b["win"].view(self.S, nw))
        b["x"][:, :nw].mul_(b["wscale"])
        b["xb"].copy_(b["x"])
        q = self.forward(b["xb"], 1)
        b["Q"].copy_(q)
        b["Q"].mul_(self.q_scale)

    def predict(self, U, Vg, Vds, batch=16):
        """Charge [n][S] (float64) for potentials U [n][S]."""
        t = self.torch
        n = U.shape[0]
        out = t.empty(n, self.S, dtype=t.float64, device=self.dev)
        for i in range(0, n, batch):
            b = min(batch, n - i)
            xb = self.features(U[i:i + b], Vg[i:i + b], Vds[i:i + b])
            q = self.forward(xb, b)
            out[i:i + b] = (q[: b * self.S].reshape(b, self.S) * self.q_scale).double()
        return out


# ---------------------------------------------------------------------- data
def tube_kwargs(vds, eta=2e-3, unitcells=1000, modes=8, precision="fp64"):
    """The (17,0) 4000-site, 8-mode tube with 1024 contour + 3072 real-axis
    energies on [-1.5, 1.5] eV, contact mu (0, -Vds)."""
    return dict(type_id=(17, 0), num_unitcells=unitcells, num_modes=modes, contact_mu=(0.0, -float(vds)),
                contact_T=(300.0, 300.0), eq_integration_pts=(256, 256, 512), E_zPlus_imag=eta,
                realaxis_window=(-1.5, 1.5, 3072, 0), precision=precision)


def generate_pairs(n, seed=20261203 + 5, vds_bins=13, batch_tubes=16, unitcells=1000, modes=8, log=None):
    """n (U, Vg, Vds, Q) samples of the engine on the tube of tube_kwargs:
    Vg ~ U(0, 0.8) V, Vds ~ U(0, 0.6) V (rounded to vds_bins levels so that
    tubes of one level share their energy paths), U = the gate/contact
    stand-in's external potential (gate Vg, source 0, drain Vds) + the
    config-2 recipe of 5 seeded Gaussian bumps (amplitudes up to a, a drawn
    from U(0, 0.4) V per sample; widths U(2, 10) nm).
    Returns device tensors (float32 U, Vg, Vds; float64 Q) and the seconds
    the engine spent."""
    import torch
    from .negf import CNT, compute_charge
    from .workloads import gate_with_contacts, site_potential
    rng = np.random.default_rng(seed)
    levels = np.linspace(0.0, 0.6, vds_bins)
    vds = levels[rng.integers(0, vds_bins, n)]
    vg = rng.uniform(0.0, 0.8, n)
    U_all = np.zeros((n, 4 * unitcells))
    Q_all = torch.zeros(n, 4 * unitcells, dtype=torch.float64, device="cuda")
    engine = 0.0
    for lv in levels:
        idx = np.nonzero(vds == lv)[0]
        if len(idx) == 0:
            continue
        tubes = [CNT(**tube_kwargs(lv, unitcells=unitcells, modes=modes)) for _ in range(min(batch_tubes, len(idx)))]
        y = tubes[0].site_positions()
        R = 1.42e-10 * np.sqrt(3.0) * 17 / (2 * np.pi)
        ga = gate_with_contacts(y, R, vds=lv)
        for c in range(0, len(idx), len(tubes)):
            part = idx[c:c + len(tubes)]
            for t, i in zip(tubes, part):
                amp = rng.uniform(0.0, 0.4)
                U = ga.external(vg[i]) + site_potential(y, seed + 1000 + int(i), amp=amp, ramp=0.0)
                U_all[i] = U
                t.set_potential(U, (U[0], U[-1]))
            out = torch.empty(sum(t.num_field_sites for t in tubes[:len(part)]), dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            compute_charge(tubes[:len(part)], out=out)
            torch.cuda.synchronize()
            engine += time.perf_counter() - t0
            Q_all[torch.as_tensor(part, device="cuda")] = out.reshape(len(part), -1)
        if log:
            log(lv, len(idx))
        del tubes
    dev = "cuda"
    return (torch.tensor(U_all, dtype=torch.float32, device=dev), torch.tensor(vg, dtype=torch.float32, device=dev),
            torch.tensor(vds, dtype=torch.float32, device=dev), Q_all, engine)


def generate_scf_pairs(n, seed=20261203 + 5, vds_bins=13, max_iter=60, unitcells=1000, modes=8, log=None):
    """n (U, Vg, Vds, Q) pairs recorded along plain self-consistent solves of
    the tube of tube_kwargs inside its gate/contact stand-in at random
    Vg ~ U(0, 0.8) V and Vds ~ U(0, 0.6) V (vds_bins levels): every NEGF
    iteration of every solve is one pair, so the pairs cover the potentials
    that a self-consistent loop visits.  Returns device tensors and the
    seconds the engine spent."""
    import torch
    from .negf import CNT, Broyden, compute_charge
    from .scf import device_view
    from .workloads import gate_with_contacts
    rng = np.random.default_rng(seed)
    levels = np.linspace(0.0, 0.6, vds_bins)
    S = 4 * unitcells
    U_all = torch.zeros(n, S, dtype=torch.float32, device="cuda")
    Q_all = torch.zeros(n, S, dtype=torch.float64, device="cuda")
    vg_all = np.zeros(n)
    vd_all = np.zeros(n)
    tubes, electros = {}, {}
    R = 1.42e-10 * np.sqrt(3.0) * 17 / (2 * np.pi)
    k = 0
    engine = 0.0
    Q = torch.zeros(S, dtype=torch.float64, device="cuda")
    while k < n:
        lv = float(levels[rng.integers(0, vds_bins)])
        vg = float(rng.uniform(0.0, 0.8))
        if lv not in tubes:
            tubes[lv] = CNT(**tube_kwargs(lv, unitcells=unitcells, modes=modes))
            electros[lv] = gate_with_contacts(tubes[lv].site_positions(), R, vds=lv)
        t, el = tubes[lv], electros[lv]
        Kd, U0 = el.device_operator(vg)
        Up = t.potential_device_ptr()
        Uv = device_view(Up, S)
        br = Broyden(torch.zeros(S, dtype=torch.float64, device="cuda"), max_step=max_iter + 2, fraction=0.1)
        nin = device_view(br.input_device_ptr(), S)
        for _ in range(max_iter):
            check(_lib.load().negf_affine_potential(C.c_void_p(Kd.data_ptr()), C.c_void_p(U0.data_ptr()),
                                                    C.c_void_p(nin.data_ptr()), C.c_void_p(Up), S, None),
                  "negf_affine_potential")
            ends = Uv[[0, S - 1]].cpu().numpy()
            t.set_potential_device(Up, (float(ends[0]), float(ends[1])))
            t0 = time.perf_counter()
            compute_charge([t], out=Q)
            torch.cuda.synchronize()
            engine += time.perf_counter() - t0
            if k < n:
                U_all[k] = Uv.float()
                Q_all[k] = Q
                vg_all[k], vd_all[k] = vg, lv
                k += 1
            if not (br.step(Q) > 1e-6) or k >= n:
                break
        br.close()
        if log:
            log(k)
    dev = "cuda"
    return (U_all, torch.tensor(vg_all, dtype=torch.float32, device=dev),
            torch.tensor(vd_all, dtype=torch.float32, device=dev), Q_all, engine)


# ---------------------------------------------------------------------- SCF
def surrogate_secant_rows(model, Kd, U0, n0, Vg, Vds, k, fraction, rel_step=0.02):
    """Initial inverse-Jacobian rows from the surrogate at the charge n0: k
    secant pairs of its residual map F_s(n) = n - Q_s(U0 + K n) along the
    first k cosine modes of the charge (each step sized so that the
    potential moves by rel_step of its range, above the BF16 input
    resolution), turned into rows of the modified-second method."""
    import torch
    from .negf import Broyden
    N = n0.numel()
    K = Kd.view(N, N)
    s = torch.arange(N, dtype=torch.float64, device=n0.device)
    D = torch.stack([torch.cos(math.pi * j * (s + 0.5) / N) for j in range(k)])  # [k][N]
    KD = D @ K.T  # potential change of each unit direction
    U_base = U0 + K @ n0
    scale = rel_step * float(U_base.abs().max().clamp_min(1e-12))
    dn = D * (scale / KD.abs().max(dim=1, keepdim=True).values.clamp_min(1e-300))
    n_all = torch.cat([n0[None], n0[None] + dn])  # [k+1][N]
    U_all = U0[None] + n_all @ K.T
    vg = torch.full((k + 1,), float(Vg), dtype=torch.float32, device=n0.device)
    vd = torch.full((k + 1,), float(Vds), dtype=torch.float32, device=n0.device)
    Q = model.predict(U_all.float(), vg, vd, batch=min(16, k + 1))
    F = n_all - Q
    return Broyden.secant_rows(dn, F[1:] - F[0][None], fraction=fraction)


def scf_sweep(tube, electro, Vg_list, Vds, model=None, fraction=0.1, max_norm=1e-6, max_step=200,
              use_graph=True, iters_per_graph=4, surrogate_norm=1e-3, surrogate_max_step=60, keep_history=True,
              seed_rows=0):
    """Gate sweep of one tube, plain or surrogate-started.

    Plain: Broyden from n = 0 with the NEGF charge (device-resident steps,
    CUDA-graph replay).  Surrogate-started: the same Broyden first converges
    the loop with the surrogate's charge (to surrogate_norm) and then
    continues, without a reset, with the NEGF charge; the Broyden history
    built on the surrogate is the initial inverse Jacobian of the NEGF phase
    (keep_history=False: only the charge is kept; seed_rows=k > 0: the NEGF
    phase starts from the surrogate's charge with k secant rows of the
    surrogate at that charge as its initial inverse Jacobian,
    negf_broyden_set_initial_jacobian) and only an NEGF charge can end the
    step.  A surrogate phase that does not converge within
    surrogate_max_step steps (or turns non-finite) is discarded and the step
    starts plain.  Returns per-step records (NEGF iterations, surrogate
    iterations, whether the surrogate start was used, seconds, charge)."""
    import torch
    from . import negf as ng
    N = tube.num_field_sites
    dev = "cuda"
    stream = torch.cuda.Stream()
    out = []
    with torch.cuda.stream(stream):
        Q = torch.zeros(N, dtype=torch.float64, device=dev)
        # history capacity for both phases; the NEGF phase alone stays within max_step
        br = ng.Broyden(torch.zeros(N, dtype=torch.float64, device=dev), max_step=max_step + surrogate_max_step,
                        fraction=fraction, stream=stream)
        nin = br.input_device_ptr()
        nin_t = __import__("electrostatic_b200.scf", fromlist=["device_view"]).device_view(nin, N)
        Kd, U0 = electro.device_operator(0.0)
        U0 = U0.clone()
        Up = tube.potential_device_ptr()
        Uview = __import__("electrostatic_b200.scf", fromlist=["device_view"]).device_view(Up, N)
        flags = torch.zeros(8, dtype=torch.int32, device=dev)
        skip = flags.data_ptr() + 12
        ng.affine_potential_masked(Kd, U0, nin, Up, N, None, stream=stream)
        plan = ng.ChargePlan([tube], Q)

        def body(s):
            ng.affine_potential_masked(Kd, U0, nin, Up, N, skip, stream=s)
            plan.launch(skip=skip, stream=s)
            br.step_device(Q, max_norm, flags, stream=s)

        graph = None
        if use_graph:
            flags[3] = 1
            body(stream)
            stream.synchronize()
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph, stream=stream):
                for _ in range(iters_per_graph):
                    body(torch.cuda.current_stream())
        sgraph = None
        if model is not None:
            # the surrogate phase: potential -> surrogate charge -> Broyden step, captured
            Qs = torch.zeros(N, dtype=torch.float64, device=dev)
            flags_s = torch.zeros(8, dtype=torch.int32, device=dev)
            model.bind(Uview, 0.0, Vds, Qs)

            def sbody(s):
                ng.affine_potential_masked(Kd, U0, nin, Up, N, flags_s.data_ptr() + 12, stream=s)
                model.infer()
                br.step_device(Qs, surrogate_norm, flags_s, stream=s)

            flags_s[3] = 1
            sbody(stream)  # allocates the model's buffers outside the capture
            stream.synchronize()
            sgraph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(sgraph, stream=stream):
                for _ in range(iters_per_graph):
                    sbody(torch.cuda.current_stream())
        for Vg in Vg_list:
            U0.copy_(electro.device_operator(Vg)[1])
            flags.zero_()
            stream.synchronize()
            t0 = time.perf_counter()
            sur_it = 0
            used = False
            if model is not None:
                model.set_bias(Vg, Vds)
                flags_s.zero_()
                while True:
                    sgraph.replay()
                    f = flags_s.cpu().numpy()
                    sur_it = int(f[1])
                    if f[3] or sur_it >= surrogate_max_step:
                        break
                used = bool(f[0]) and not f[2]
                if not used:  # discard the surrogate phase
                    br.reset(stream=stream)
                elif seed_rows > 0:
                    nkeep = nin_t.clone()
                    V, W = surrogate_secant_rows(model, Kd, U0, nkeep, Vg, Vds, seed_rows, fraction)
                    br.reset(stream=stream)
                    nin_t.copy_(nkeep)
                    br.set_initial_jacobian(V.contiguous(), W.contiguous(), stream=stream)
                elif not keep_history:
                    nkeep = nin_t.clone()
                    br.reset(stream=stream)
                    nin_t.copy_(nkeep)
                # the NEGF phase continues from here
            while True:
                if graph is not None:
                    graph.replay()
                else:
                    body(stream)
                f = flags.cpu().numpy()
                if f[3]:
                    break
            dt = time.perf_counter() - t0
            if f[2]:
                raise RuntimeError("NEGF self-consistency failed (flag %d)" % f[2])
            out.append(dict(Vg=float(Vg), negf_iterations=int(f[1]), surrogate_iterations=sur_it,
                            surrogate_used=used, seconds=dt, Q=Q.cpu().numpy().copy()))
            br.reset(stream=stream)
        stream.synchronize()
    del graph
    del sgraph
    plan.close()
    br.close()
    return out
