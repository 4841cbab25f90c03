"""Surrogate over a set of tubes: one Fourier neural operator for every tube of
an uneven batch, trained on the batch's self-consistent fixed points, and the
surrogate-started gate sweep.

The operator of surrogate.py maps a fixed-length potential to a charge.  Here
one operator serves the whole batch (tubes of 800-8000 sites, chiralities
(13,0), (17,0), (19,0), 2-10 modes): every tube sits on a canvas of S sites
(its own sites first, padding after), and per-site descriptors tell the
operator which tube it reads.  One inference is one batch of canvases, a
fixed set of launches whatever the tube count.

What it maps: the EXTERNAL site potential U_ext of a tube (the gate and
contact electrodes' potential with no charge on the tube) plus (Vg, Vds) to
the tube's self-consistent charge n* (the fixed point n* = Q(U_ext + K n*) of
the NEGF-Poisson loop).  One inference is then the Broyden start of a bias
point; no surrogate loop runs.

Features per site (FEAT_SET = 40):
  0..16  U_ext at sites n-8 .. n+8 of the tube (indices clamped to the tube:
         the leads continue at the end-site potential), divided by the
         potential scale
  17, 18 Vg, Vds
  19..39 n / N, ring parity +-1, exp(-n / 40), exp(-(N-1-n) / 40), inside
         mask, chirality one-hot (13, 17, 19), modes / 10, inner band edge of
         the lowest and of the highest kept mode / gamma, channels / 20, N / S,
         exp(-n / 3), exp(-(N-1-n) / 3), exp(-n / 12), exp(-(N-1-n) / 12),
         end-site indicators (n = 0, n = N-1), two zeros (the end sites carry
         the largest charges: the leads attach there)

Training pairs come from the engine itself (generate_fixed_points): batched
self-consistent solves of the whole set at random drain biases Vds ~ U(0,
0.6) V (vds_bins levels: the tubes of one level share their energy paths)
and per-tube gate voltages Vg ~ U(0, 0.8) V; in a bump_fraction of the solves
the external potential also carries 5 seeded Gaussian bumps (the config-2
recipe of random potentials), so the operator sees more than the
two-parameter family of a gate sweep.  The loss is the mean square error over
the tubes' own sites (padding masked out), per tube relative to its largest
charge.

Spectral path: instead of the shared canvas-length Fourier basis of
surrogate.py, every tube gets the first 64 cosine (DCT-II) modes of its own
length (pairs of modes share one mixing matrix, as the (cos, sin) pairs do
there), so short and long tubes are resolved alike.

The sweep (fixed_point_sweep): per gate point, one inference gives the
start -- by default the linear extrapolation of the two previous gate
points' converged charges plus the operator's second difference over the
three gate points (the operator's change alone at the second point, its
charge at the first), which cancels the part of the operator's error that
varies slowly with the bias -- and a BatchSCF solve converges it:
mixed-precision plan until the residual falls below switch_norm, the FP64
plan after, one secant update per tube (segments); only an FP64 NEGF charge
ends a solve (the engine judges every converged charge).  The initial
inverse Jacobian is fraction * I, 0.2 by default.  With fraction=None it
comes from the surrogate's Jacobian: the fixed-point map's derivative
J = dn*/dU_ext = (I - chi K)^-1 chi gives J K = (I - chi K)^-1 chi K, whose
eigenvalues are -lambda / (1 + lambda) for the eigenvalues 1 + lambda of
the loop's Jacobian I - chi K; the largest |mu| by power iteration gives
lambda_max = |mu| / (1 - |mu|) and fraction = 2 / (2 + lambda_max), the
Richardson step for a spectrum in [1, 1 + lambda_max] (measured on the
16-tube set it saturates, |mu| >= 0.95, and the fixed 0.2 converges faster).
"""
from __future__ import annotations

import math
import time

import numpy as np

from .surrogate import MODES, WIN, FourierOperator

FEAT_SET = 40


def tube_descriptor(tube):
    """Per-tube constants of the features (from the engine's mode table)."""
    J, deg, beta = tube.modes()
    gamma = float(tube.desc.gamma)
    edges = np.abs(np.abs(beta) - gamma) / gamma
    return dict(N=tube.num_field_sites, m=int(tube.desc.type_id[0]), M=len(beta), edge_lo=float(edges.min()),
                edge_hi=float(edges.max()), channels=int(np.sum(deg)))


class TubeSetOperator(FourierOperator):
    """The Fourier operator on a canvas of S sites for a fixed set of tubes."""

    def __init__(self, descriptors, S=None, seed=0, device="cuda"):
        import torch
        nmax = max(d["N"] for d in descriptors)
        S = int(S or ((nmax + 255) // 256) * 256)
        super().__init__(S, seed=seed, device=device, feat=FEAT_SET)
        self.desc = list(descriptors)
        T = len(self.desc)
        nw = 2 * WIN + 1
        fixed = np.zeros((T, S, FEAT_SET - nw - 2), dtype=np.float32)
        widx = np.zeros((T, S, nw), dtype=np.int64)
        mask = np.zeros((T, S), dtype=np.float32)
        n = np.arange(S)
        for t, d in enumerate(self.desc):
            N = d["N"]
            inside = n < N
            fixed[t, :, 0] = np.where(inside, n / N, 0.0)
            fixed[t, :, 1] = np.where(n % 2 == 0, 1.0, -1.0)
            fixed[t, :, 2] = np.exp(-n / 40.0)
            fixed[t, :, 3] = np.where(inside, np.exp(-np.clip(N - 1 - n, 0, None) / 40.0), 0.0)
            fixed[t, :, 4] = inside
            fixed[t, :, 5 + {13: 0, 17: 1, 19: 2}.get(d["m"], 1)] = 1.0
            fixed[t, :, 8] = d["M"] / 10.0
            fixed[t, :, 9] = d["edge_lo"]
            fixed[t, :, 10] = d["edge_hi"]
            fixed[t, :, 11] = d["channels"] / 20.0
            fixed[t, :, 12] = N / S
            tail = np.clip(N - 1 - n, 0, None)
            fixed[t, :, 13] = np.exp(-n / 3.0)
            fixed[t, :, 14] = np.where(inside, np.exp(-tail / 3.0), 0.0)
            fixed[t, :, 15] = np.exp(-n / 12.0)
            fixed[t, :, 16] = np.where(inside, np.exp(-tail / 12.0), 0.0)
            fixed[t, 0, 17] = 1.0
            fixed[t, N - 1, 18] = 1.0
            widx[t] = np.clip(n[:, None] + np.arange(-WIN, WIN + 1)[None, :], 0, N - 1)
            mask[t] = inside
        # per-tube spectral bases: the first 2 * MODES cosine (DCT-II) modes of the
        # tube's own length, so that every tube, short or long, gets the same
        # resolution (a shared canvas-length basis would give an 800-site tube
        # only a few modes); pairs of modes (2j, 2j + 1) share one mixing matrix
        Fa = np.zeros((T, 2 * MODES, S), dtype=np.float32)
        Ga = np.zeros((T, S, 2 * MODES), dtype=np.float32)
        for t, d in enumerate(self.desc):
            N = d["N"]
            k = np.arange(2 * MODES)[:, None]
            c = np.cos(np.pi * k * (np.arange(N)[None, :] + 0.5) / N)
            Fa[t, :, :N] = c * np.where(k == 0, 1.0, 2.0) / N
            Ga[t, :N, :] = c.T
        self.F_all = torch.tensor(Fa, dtype=torch.bfloat16, device=device)
        self.G_all = torch.tensor(Ga, dtype=torch.bfloat16, device=device)
        self._fixed_set = torch.tensor(fixed, device=device)
        self._widx_set = torch.tensor(widx.reshape(T, S * nw), device=device)
        self._mask_set = torch.tensor(mask, device=device)
        self.Ns = [d["N"] for d in self.desc]
        self.offs = np.concatenate([[0], np.cumsum(self.Ns)]).astype(np.int64)

    # ------------------------------------------------------------------ features
    def features_set(self, U, Vg, Vds, tid):
        """U: canvas potentials [B][S] (float32; a tube's sites first), Vg,
        Vds [B], tid [B] tube indices -> BF16 rows [B*S][FEAT_SET]."""
        t = self.torch
        B = U.shape[0]
        nw = 2 * WIN + 1
        x = t.empty(B, self.S, FEAT_SET, device=self.dev)
        win = t.gather(U.float(), 1, self._widx_set[tid]).view(B, self.S, nw)
        x[:, :, :nw] = win / self.x_scale[0]
        x[:, :, nw] = (Vg.float() / self.x_scale[nw])[:, None]
        x[:, :, nw + 1] = (Vds.float() / self.x_scale[nw + 1])[:, None]
        x[:, :, nw + 2:] = self._fixed_set[tid]
        return x.to(t.bfloat16).reshape(B * self.S, FEAT_SET)

    # ------------------------------------------------------------------ training
    def fit_set(self, U, Vg, Vds, tid, Q, epochs=20, batch=64, lr=2e-3, log=None):
        """Train on canvas tensors U, Q [n][S] (float32), Vg, Vds [n], tid [n];
        the loss covers every tube's own sites only."""
        t = self.torch
        n = U.shape[0]
        nw = 2 * WIN + 1
        self.x_scale = t.ones(FEAT_SET, device=self.dev)
        self.x_scale[0] = float(U.abs().max())
        self.x_scale[nw] = max(float(Vg.abs().max()), 1e-3)
        self.x_scale[nw + 1] = max(float(Vds.abs().max()), 1e-3)
        # per-tube output scales: the tubes' charges differ by their channel counts
        qs = t.zeros(len(self.desc), device=self.dev)
        qs.scatter_reduce_(0, tid, Q.abs().amax(dim=1).float(), reduce="amax")
        self.qs_t = qs.clamp_min(1e-12)
        self.q_scale = float(self.qs_t.max())
        g = t.Generator(device="cpu").manual_seed(1)
        hist = []
        t0 = time.perf_counter()
        steps = epochs * (n // batch)
        for ep in range(epochs):
            perm = t.randperm(n, generator=g)
            tot = t.zeros((), dtype=t.float64, device=self.dev)
            cnt = t.zeros((), dtype=t.float64, device=self.dev)
            for i in range(n // batch):
                idx = perm[i * batch:(i + 1) * batch].to(self.dev)
                ti = tid[idx]
                xb = self.features_set(U[idx], Vg[idx], Vds[idx], ti)
                self._basis = (self.F_all[ti], self.G_all[ti])
                q = self.forward(xb, batch, keep=True)
                m = self._mask_set[ti].reshape(-1)
                q.mul_(m)
                y = (Q[idx] / self.qs_t[ti][:, None]).reshape(-1).float().mul_(m)
                dq, part = self.loss_grad(q, y)
                dq.mul_(m)
                self.backward(dq, batch)
                frac = (ep * (n // batch) + i) / max(1, steps)
                self.adam(lr=lr * 0.5 * (1 + math.cos(math.pi * frac)))
                tot += part.sum()
                cnt += m.sum()
            hist.append(float(tot) / max(float(cnt), 1.0))
            if log:
                log(ep, hist[-1])
        t.cuda.synchronize()
        self._basis = None
        return {"epochs": epochs, "seconds": time.perf_counter() - t0, "loss": hist}

    def predict_set(self, U, Vg, Vds, tid, batch=16):
        """Charge canvases [n][S] (float64) for canvas potentials U [n][S]."""
        t = self.torch
        n = U.shape[0]
        out = t.empty(n, self.S, dtype=t.float64, device=self.dev)
        for i in range(0, n, batch):
            b = min(batch, n - i)
            xb = self.features_set(U[i:i + b], Vg[i:i + b], Vds[i:i + b], tid[i:i + b])
            self._basis = (self.F_all[tid[i:i + b]], self.G_all[tid[i:i + b]])
            q = self.forward(xb, b)
            self._basis = None
            out[i:i + b] = (q[: b * self.S].reshape(b, self.S) * self.qs_t[tid[i:i + b]][:, None]).double()
        return out * self._mask_set[tid].double()

    # ------------------------------------------------------------------ bound inference over the set
    def bind_set(self, Ucat, Qcat, Vg, Vds):
        """Fixed buffers for repeated inference over the whole set (capturable
        after one call of infer_set): Ucat, Qcat float64 device vectors of the
        concatenated tubes' sites (tube order as the descriptors)."""
        t = self.torch
        T, S, nw = len(self.desc), self.S, 2 * WIN + 1
        # window index of every canvas site into Ucat, output index of every tube site into the canvas
        wi = self._widx_set.view(T, S, nw) + t.tensor(self.offs[:-1], device=self.dev).view(T, 1, 1)
        qi = np.concatenate([t_ * S + np.arange(N) for t_, N in enumerate(self.Ns)])
        self._bs = dict(U=Ucat, Q=Qcat, widx=wi.reshape(-1).contiguous(), qidx=t.tensor(qi, device=self.dev),
                        win=t.empty(T * S * nw, dtype=t.float64, device=self.dev),
                        x=t.empty(T, S, FEAT_SET, device=self.dev),
                        xb=t.empty(T * S, FEAT_SET, dtype=t.bfloat16, device=self.dev),
                        qd=t.empty(T * S, dtype=t.float64, device=self.dev),
                        qscale=self.qs_t.double().repeat_interleave(S).contiguous())
        x = self._bs["x"]
        x[:, :, nw + 2:] = self._fixed_set
        self.set_bias_set(Vg, Vds)

    def set_bias_set(self, Vg, Vds):
        nw = 2 * WIN + 1
        x = self._bs["x"]
        x[:, :, nw] = float(Vg) / float(self.x_scale[nw])
        x[:, :, nw + 1] = float(Vds) / float(self.x_scale[nw + 1])

    def infer_set(self):
        """Qcat = model(Ucat) over all tubes (no allocation after the first call)."""
        t = self.torch
        b = self._bs
        T, S, nw = len(self.desc), self.S, 2 * WIN + 1
        t.index_select(b["U"], 0, b["widx"], out=b["win"])
        b["x"][:, :, :nw].copy_(b["win"].view(T, S, nw))
        b["x"][:, :, :nw].div_(self.x_scale[0])
        b["xb"].copy_(b["x"].view(T * S, FEAT_SET))
        self._basis = (self.F_all, self.G_all)
        q = self.forward(b["xb"], T)
        self._basis = None
        b["qd"].copy_(q)
        b["qd"].mul_(b["qscale"])
        t.index_select(b["qd"], 0, b["qidx"], out=b["Q"])


# ---------------------------------------------------------------------- data
def generate_fixed_points(make_tubes, electros, n_pairs, seed=20261203 + 5, vds_bins=13, vds_max=0.6,
                          vg_max=0.8, bump_fraction=0.5, bump_amp=0.2, tol=3e-6, fraction=0.15, max_step=300, S=None,
                          log=None):
    """n_pairs (canvas U_ext, Vg, Vds, tube id, canvas n*) from batched
    self-consistent solves of the tube set (module docstring): per solve every
    tube gets its own gate voltage in [0, vg_max] V, the drain bias is one of
    vds_bins levels in [0, vds_max] V; solves to a max-norm residual of tol
    with per-tube secant updates at the given fraction (a solve that passes
    max_step is dropped and drawn again).  make_tubes(vds) returns the set's
    tubes at that drain bias.  Returns device tensors, the seconds of the
    solves and their iteration counts (dropped solves as -1)."""
    import torch
    from .scf import BatchSCF
    from .workloads import site_potential
    rng = np.random.default_rng(seed)
    levels = np.linspace(0.0, vds_max, vds_bins)
    T = len(electros)
    dev = "cuda"
    Ns = [e.N for e in electros]
    S = int(S or ((max(Ns) + 255) // 256) * 256)
    n_solves = -(-n_pairs // T)
    per_level = [n_solves // vds_bins + (1 if i < n_solves % vds_bins else 0) for i in range(vds_bins)]
    U_all = torch.zeros(n_solves * T, S, dtype=torch.float32, device=dev)
    Q_all = torch.zeros(n_solves * T, S, dtype=torch.float32, device=dev)
    vg_all = np.zeros(n_solves * T)
    vd_all = np.zeros(n_solves * T)
    tid_all = np.tile(np.arange(T), n_solves)
    k = 0
    seconds, iters = 0.0, []
    for lv, count in zip(levels, per_level):
        if count == 0:
            continue
        lv = float(lv)
        for e in electros:
            e.Vds = lv
        tubes = make_tubes(lv)
        scf = BatchSCF(tubes, electros, fraction=fraction, max_norm=tol, max_step=max_step, iters_per_graph=4,
                       segments=True)
        done = 0
        while done < count:
            U0 = []
            for t_, e in enumerate(electros):
                vg = float(rng.uniform(0.0, vg_max))
                u = e.external(vg)
                if rng.uniform() < bump_fraction:
                    u = u + site_potential(e.y_nm, int(rng.integers(1 << 30)), amp=float(rng.uniform(0.0, bump_amp)),
                                           ramp=0.0)
                U0.append(u)
                U_all[k + t_, :Ns[t_]] = torch.as_tensor(u, dtype=torch.float32, device=dev)
                vg_all[k + t_], vd_all[k + t_] = vg, lv
            scf.set_external(U0=U0)
            scf.reset(keep_charge=False)
            scf.stream.synchronize()
            t0 = time.perf_counter()
            try:
                it, _ = scf.solve()
            except RuntimeError:
                it = -1
            scf.stream.synchronize()
            seconds += time.perf_counter() - t0
            iters.append(it)
            if it < 0:
                if iters.count(-1) > max(4, n_solves // 10):
                    raise RuntimeError("too many training solves failed to converge")
                continue
            done += 1
            for t_ in range(T):
                Q_all[k + t_, :Ns[t_]] = scf.n_in[scf.offs[t_]:scf.offs[t_ + 1]].float()
            k += T
            if log:
                log(lv, k, it)
        scf.close()
        for tube in tubes:
            tube.close()
    order = torch.tensor(rng.permutation(k)[:n_pairs], device=dev)
    return (U_all[order], torch.tensor(vg_all, dtype=torch.float32, device=dev)[order],
            torch.tensor(vd_all, dtype=torch.float32, device=dev)[order], torch.tensor(tid_all, device=dev)[order],
            Q_all[order], seconds, iters)


# ---------------------------------------------------------------------- SCF
START_MODES = ("extrapolated", "difference", "surrogate", "extrapolation", "continuation", "zero")


def fixed_point_sweep(tubes, electros, Vg_list, model, fraction=0.2, max_fraction=0.2, max_norm=1e-6,
                      max_step=200, switch_norm=3e-6, segments=True, carry_rows=False, iters_per_graph=4,
                      power_iters=6, autotune=True, start="extrapolated"):
    """Surrogate-started gate sweep of a tube set (module docstring).  Tubes
    in mixed precision run on their own plan until the residual falls below
    switch_norm, then on an FP64 plan.  fraction: the scalar initial inverse
    Jacobian (None: 2 / (2 + lambda_max) from the surrogate's Jacobian, at
    most max_fraction).  start, with n_k the converged charge and S_k the
    operator's charge at gate point k:
      "extrapolated"  2 n_{k-1} - n_{k-2} + (S_k - 2 S_{k-1} + S_{k-2}): the
                      linear extrapolation of the converged charges plus the
                      operator's curvature ("difference" at k = 1, S_0 at 0);
      "difference"    n_{k-1} + S_k - S_{k-1} (S_0 at k = 0);
      "surrogate"     S_k;
      "extrapolation" 2 n_{k-1} - n_{k-2} without the operator (n_0 at k = 1,
                      zero at k = 0);
      "continuation"  n_{k-1} (zero at k = 0);
      "zero".
    carry_rows: start each gate point from the previous points' secant rows
    (negf_broyden_restart; all of them while they fit in max_step / 2, else
    none).  Returns per-step records, the fraction, lambda_max (None unless
    fraction is None) and the one-off set-up seconds (plans, graphs; outside
    the per-step times)."""
    if start not in START_MODES:
        raise ValueError(f"start must be one of {START_MODES}")
    import torch
    from . import negf as ng
    from .scf import BatchSCF
    dev = "cuda"
    Ns = [t.num_field_sites for t in tubes]
    offs = np.concatenate([[0], np.cumsum(Ns)]).astype(np.int64)
    S = int(offs[-1])
    stream = torch.cuda.Stream()
    vds = float(electros[0].Vds)
    t_setup = time.perf_counter()
    with torch.cuda.stream(stream):
        Ucat = torch.zeros(S, dtype=torch.float64, device=dev)
        Qs = torch.zeros(S, dtype=torch.float64, device=dev)
        zero = torch.zeros(max(Ns), dtype=torch.float64, device=dev)
        Kds = [e.device_operator(Vg_list[0])[0] for e in electros]
        model.bind_set(Ucat, Qs, Vg_list[0], vds)
        # the external potential is affine in Vg: U_ext(Vg) = A + Vg B, formed on the device
        A = torch.tensor(np.concatenate([e.external(0.0) for e in electros]), dtype=torch.float64, device=dev)
        B = torch.tensor(np.concatenate([e.external(1.0) - e.external(0.0) for e in electros]),
                         dtype=torch.float64, device=dev)
        views = [Ucat[int(o):int(o) + N] for o, N in zip(offs, Ns)]

        def external(Vg):
            torch.add(A, B, alpha=float(Vg), out=Ucat)

        external(Vg_list[0])
        model.infer_set()  # allocates the model's inference buffers
        stream.synchronize()
    t_setup = time.perf_counter() - t_setup
    # ---- timed: the scalar initial inverse Jacobian from the surrogate's Jacobian (power iteration on J K)
    t0 = time.perf_counter()
    alpha, lam = fraction, None
    with torch.cuda.stream(stream):
        if alpha is None:
            g = torch.Generator(device="cpu").manual_seed(0)
            v = torch.randn(S, generator=g, dtype=torch.float64).to(dev)
            v /= v.norm()
            U0 = Ucat.clone()
            model.infer_set()
            q0 = Qs.clone()
            Kv = torch.empty(S, dtype=torch.float64, device=dev)
            mu = 0.0
            for _ in range(power_iters):
                for Kd, o, N in zip(Kds, offs, Ns):
                    ng.affine_potential_masked(Kd, zero, v.data_ptr() + 8 * int(o), Kv.data_ptr() + 8 * int(o), N,
                                               None, stream=stream)
                # the operator reads BF16 potentials: move them by about 0.02 V
                eps = 0.02 / float(Kv.abs().max())
                torch.add(U0, Kv, alpha=eps, out=Ucat)
                model.infer_set()
                w = (Qs - q0) / eps
                mu = float(w.norm())
                v = w / mu
            Ucat.copy_(U0)
            mu = min(mu, 0.95)
            lam = mu / (1.0 - mu)
            alpha = float(min(max_fraction, max(0.05, 2.0 / (2.0 + lam))))
        stream.synchronize()
    t_alpha = time.perf_counter() - t0
    t1 = time.perf_counter()
    switch = switch_norm if any(t.desc.precision == 1 for t in tubes) else None
    scf = BatchSCF(tubes, electros, fraction=alpha, max_norm=max_norm, max_step=max_step,
                   iters_per_graph=iters_per_graph, autotune=autotune, switch_norm=switch, segments=segments)
    t_setup += time.perf_counter() - t1
    out = []
    uses_model = start in ("extrapolated", "difference", "surrogate")
    with torch.cuda.stream(scf.stream):
        s1 = torch.zeros(S, dtype=torch.float64, device=dev)  # S_{k-1}
        s2 = torch.zeros(S, dtype=torch.float64, device=dev)  # S_{k-2}
        m1 = torch.zeros(S, dtype=torch.float64, device=dev)  # n_{k-1}
        m2 = torch.zeros(S, dtype=torch.float64, device=dev)  # n_{k-2}
        n0 = torch.zeros(S, dtype=torch.float64, device=dev)
    for step, Vg in enumerate(Vg_list):
        # the bias point's external potential (the electrostatics' part, untimed as in run_scf_batch)
        with torch.cuda.stream(scf.stream):
            external(Vg)
        scf.set_external(U0=views)
        scf.stream.synchronize()
        t0 = time.perf_counter()
        with torch.cuda.stream(scf.stream):
            if uses_model:
                model.set_bias_set(Vg, vds)
                model.infer_set()
            k = step
            if start == "zero" or (k == 0 and not uses_model):
                n0.zero_()
            elif start == "surrogate" or k == 0:
                n0.copy_(Qs)
            elif start == "continuation" or (start == "extrapolation" and k == 1):
                n0.copy_(m1)
            elif start == "difference" or (start == "extrapolated" and k == 1):
                torch.add(m1, Qs, out=n0)
                n0.sub_(s1)
            elif start == "extrapolation":
                torch.mul(m1, 2.0, out=n0)
                n0.sub_(m2)
            else:  # extrapolated, k >= 2
                torch.mul(m1, 2.0, out=n0)
                n0.sub_(m2).add_(Qs).sub_(s1, alpha=2.0).add_(s2)
            if uses_model:
                s2.copy_(s1)
                s1.copy_(Qs)
            if carry_rows and k > 0:
                scf.br.restart(keep_rows=max_step // 2, stream=scf.stream)
            else:
                scf.reset(keep_charge=True)
            scf.n_in.copy_(n0)
        it, low = scf.solve()
        scf.stream.synchronize()
        dt = time.perf_counter() - t0 + (t_alpha if step == 0 else 0.0)
        with torch.cuda.stream(scf.stream):
            rec = dict(Vg=float(Vg), negf_iterations=it, lowprec_iterations=low, seconds=dt,
                       Q=scf.Q.cpu().numpy().copy(), n_in=scf.n_in.cpu().numpy().copy(), start=n0.cpu().numpy().copy())
            if uses_model:
                rec["surrogate"] = Qs.cpu().numpy().copy()
            out.append(rec)
            m2.copy_(m1)
            m1.copy_(scf.n_in)  # the converged charge
    scf.close()
    return out, alpha, lam, t_setup
