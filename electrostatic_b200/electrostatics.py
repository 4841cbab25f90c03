"""Electrostatics stand-in for the self-consistent loop: U = U_ext + K Q.

The reference solves Poisson with AMReX MLMG on a 3D mesh and gathers the
ring-averaged potential at the atoms (Source/Solver/Electrostatics/MLMG.cpp,
Source/Solver/Transport/Nanostructure.cpp:285-317, 397-518); AMReX is not
available here.  For the gate-all-around geometry of the benchmark decks (a
tube on the axis of a cylindrical metal gate filled with one dielectric) the
problem is linear and axisymmetric, so the site potential is an affine map of
the ring charges:

    U_m = -V_g - sum_n K_mn Q_n        (eV; Q in units of e; U = -phi, Nanostructure.cpp:494-499)

with the Green's function of a ring charge inside a grounded cylinder of
radius a (separation of variables, Dirichlet at rho = a):

    phi(rho, z) = q / (2 pi eps a) sum_k J0(x_k rho'/a) J0(x_k rho/a) exp(-x_k |z - z'| / a) / (x_k J1(x_k)^2)

where x_k are the zeros of J0.  The series at rho = rho' diverges
logarithmically for an infinitely thin ring; a Gaussian factor
exp(-(x_k s / a)^2 / 2) with s = the mesh spacing smooths it the way the
reference's trilinear gather/deposit on a mesh of that spacing does.
"""
from __future__ import annotations

import numpy as np

Q_E = 1.602176634e-19      # C (Utils/SelectWarpXUtils/WarpXConst.H)
EPS0 = 8.8541878128e-12    # F/m


def ring_coupling_matrix(y_nm, r_tube, r_gate, eps_r=3.9, smear=0.1e-9, n_terms=4000):
    """K[m, n] in V per elementary charge: ring-averaged potential at ring m
    (radius r_tube) from a unit charge spread on ring n, inside a grounded
    coaxial cylinder of radius r_gate filled with relative permittivity eps_r."""
    from scipy.special import j0, j1, jn_zeros

    x = jn_zeros(0, n_terms)
    a = float(r_gate)
    w = j0(x * r_tube / a) ** 2 / (x * j1(x) ** 2) * np.exp(-0.5 * (x * smear / a) ** 2)
    pref = Q_E / (2.0 * np.pi * eps_r * EPS0 * a)
    y = np.asarray(y_nm, dtype=np.float64) * 1e-9
    dz = np.abs(y[:, None] - y[None, :])
    # sum_k w_k exp(-x_k dz / a): exponentially convergent for dz > 0; the
    # ring spacings repeat, so evaluate each distinct distance once
    uniq, inv = np.unique(np.round(dz / 1e-13).astype(np.int64), return_inverse=True)
    vals = np.array([np.sum(w * np.exp(-x * (u * 1e-13) / a)) for u in uniq])
    K = pref * vals[inv].reshape(dz.shape)
    return K


def _bessel_series(r_tube, r_gate, eps_r, smear, n_terms):
    from scipy.special import j0, j1, jn_zeros

    x = jn_zeros(0, n_terms)
    a = float(r_gate)
    w = j0(x * r_tube / a) ** 2 / (x * j1(x) ** 2) * np.exp(-0.5 * (x * smear / a) ** 2)
    pref = Q_E / (2.0 * np.pi * eps_r * EPS0 * a)
    return x, w, a, pref


def _lattice(y_nm):
    """Integer lattice indices of the ring positions when they sit on a grid
    (zigzag tubes: multiples of a_cc / 2), else None."""
    y = np.asarray(y_nm, dtype=np.float64)
    if len(y) < 2:
        return None, None
    d = np.diff(np.sort(y))
    d = d[d > 1e-9]
    if len(d) == 0:
        return None, None
    h = d.min()
    q = (y - y[0]) / h
    idx = np.round(q).astype(np.int64)
    if np.max(np.abs(q - idx)) > 1e-6:
        return None, None
    return idx, h


def step_response(dz_m, r_tube, r_gate, n_k=40000):
    """Potential at radius r_tube inside a cylinder of radius r_gate whose
    wall potential steps from 0 to 1 at dz = 0 (Laplace, axisymmetric):
        s(dz) = 1/2 + (1/pi) int_0^inf sin(k dz)/k * I0(k r)/I0(k a) dk,
    by the midpoint rule on k <= 60 / (a - r); |dz| > 30 a is the bare step
    (the correction there is below e^-70)."""
    from scipy.special import i0e

    a, r = float(r_gate), float(r_tube)
    dz = np.asarray(dz_m, dtype=np.float64)
    kmax = 60.0 / (a - r)
    dk = kmax / n_k
    k = (np.arange(n_k) + 0.5) * dk
    g = i0e(k * r) / i0e(k * a) * np.exp(-k * (a - r))
    out = np.where(dz > 0, 1.0, np.where(dz < 0, 0.0, 0.5))
    near = np.abs(dz) <= 30 * a
    for c in np.array_split(np.nonzero(near)[0], max(1, int(near.sum()) // 256 + 1)):
        if len(c):
            out[c] = 0.5 + (np.sin(np.outer(dz[c], k)) / k) @ g * dk / np.pi
    return out


class GateAllAround:
    """Affine potential operator of a gate-all-around tube: U = U_ext - K Q.

    K: ring charge inside a grounded coaxial cylinder (module docstring).
    U_ext: -V_g everywhere, or, with contact_length, the wall potential is
    V_S = 0 over the first contact_length of the tube, V_g over the channel
    and V_D = Vds over the last contact_length (metal source/drain wrapping
    the tube ends, as in the all-around-contact decks), solved by Laplace
    inside the cylinder (step_response).
    Ring positions on a lattice (every zigzag tube) make K a function of the
    lattice distance only: the Bessel series is evaluated once per distance
    and K is assembled by indexing, on the device for device_operator."""

    def __init__(self, y_nm, r_tube, r_gate, eps_r=3.9, smear=0.1e-9, n_terms=4000, contact_length=None, Vds=0.0):
        self.y_nm = np.asarray(y_nm, dtype=np.float64)
        self.N = len(self.y_nm)
        self._args = (r_tube, r_gate, eps_r, smear, n_terms)
        self.Vds = float(Vds)
        self._steps = None
        if contact_length is not None:
            y = self.y_nm * 1e-9
            z1, z2 = y.min() + contact_length, y.max() - contact_length
            self._steps = (step_response(y - z1, r_tube, r_gate), step_response(y - z2, r_tube, r_gate))
        self._idx, h = _lattice(self.y_nm)
        self._K = None
        self._Kd = None
        if self._idx is not None:
            x, w, a, pref = _bessel_series(r_tube, r_gate, eps_r, smear, n_terms)
            J = int(self._idx.max() - self._idx.min()) + 1
            dz = np.arange(J) * h * 1e-9
            tab = np.empty(J)
            for c in range(0, J, 512):
                tab[c:c + 512] = np.exp(-np.outer(dz[c:c + 512], x) / a) @ w
            self._table = pref * tab

    @property
    def K(self):
        if self._K is None:
            if self._idx is not None:
                self._K = self._table[np.abs(self._idx[:, None] - self._idx[None, :])]
            else:
                self._K = ring_coupling_matrix(self.y_nm, *self._args)
        return self._K

    def external(self, Vg):
        """U_ext [eV] = -phi_ext at the rings."""
        if self._steps is None:
            return np.full(self.N, -float(Vg))
        s1, s2 = self._steps
        phi = 0.0 + (float(Vg) - 0.0) * s1 + (self.Vds - float(Vg)) * s2
        return -phi

    def potential(self, Q, Vg):
        return self.external(Vg) - self.K @ np.asarray(Q, dtype=np.float64)

    def device_toeplitz(self, device="cuda"):
        """(tab_dev, idx_dev) for negf_affine_potential_toeplitz when the rings
        sit on a lattice (zigzag tubes): Kd[i][j] = tab[|idx[i] - idx[j]|] with
        Kd = -K; None otherwise."""
        if self._idx is None:
            return None
        import torch
        if getattr(self, "_toe", None) is None or str(self._toe[0].device) != str(torch.device(device)):
            idx = torch.tensor(self._idx - self._idx.min(), dtype=torch.int32, device=device)
            tab = torch.tensor(-self._table, dtype=torch.float64, device=device)
            self._toe = (tab, idx)
        return self._toe

    def device_operator(self, Vg, device="cuda"):
        """(K_dev, U0_dev) for negf_affine_potential: U = U0 + Kd Q with Kd = -K
        (Kd is built once on the device and reused)."""
        import torch
        if self._Kd is None or str(self._Kd.device) != str(torch.device(device)):
            if self._idx is not None:
                idx = torch.tensor(self._idx, device=device)
                tab = torch.tensor(-self._table, dtype=torch.float64, device=device)
                self._Kd = tab[(idx[:, None] - idx[None, :]).abs()].contiguous()
                del idx
            else:
                self._Kd = torch.tensor(-self.K, dtype=torch.float64, device=device).contiguous()
        if self._steps is None:
            U0 = torch.full((self.N,), -float(Vg), dtype=torch.float64, device=device)
        else:
            U0 = torch.tensor(self.external(Vg), dtype=torch.float64, device=device)
        return self._Kd, U0


class FDPoissonGAA:
    """Gate-all-around electrostatics from a 7-point finite-difference Poisson
    solve with cloud-in-cell deposit and trilinear gather (the mesh coupling
    of Source/Solver/Transport/Nanostructure.cpp:285-395 with MLMG replaced
    by a conjugate-gradient solve): U = U_ext(Vg, Vds) - K Q.

    Geometry: nodes on a (nx, ny, nz) grid, transverse spacing h_xy around
    the tube axis (z), axial spacing covering the tube plus `margin` at each
    end (the rings need not fall on nodes).  Inside the gate radius the
    permittivity is eps_r * eps0; the cylinder rho >= r_gate and the two end
    planes are metal (Dirichlet): the gate wall at Vg, the wall over the first
    and last contact_length of the tube (when given) and the source / drain
    end planes at 0 and Vds.  Atoms (CNT.cpp:93-132): atom j of ring r at
    angle 2 pi j / m (+ (sqrt(3)/2) acc / R on rings 1, 2 of each unit cell),
    radius R; a ring charge Q_r (units of e) puts Q_r / m on each atom,
    deposited to its 8 neighbour nodes with trilinear weights over the cell
    volume (Deposit_ChargeDensityToMesh, :343-395); the potential is gathered
    at the atoms with the same weights and averaged per ring, U = -phi
    (Obtain_PotentialAtSites, :397-518).  K (V per e) takes one solve per
    ring (batched), U_ext one solve per electrode; every solve is a
    Jacobi-preconditioned conjugate gradient to a relative residual of tol.
    Same interface as GateAllAround (K, external, potential,
    device_operator)."""

    def __init__(self, y_nm, r_tube, r_gate, m, acc=1.42e-10, shape=(64, 64, 128), h_xy=0.1e-9, eps_r=3.9,
                 margin=None, contact_length=None, Vds=0.0, device=None, tol=1e-10, max_iter=20000):
        import torch
        self.y_nm = np.asarray(y_nm, dtype=np.float64)
        self.N = len(self.y_nm)
        self.Vds = float(Vds)
        self.dev = device or ("cuda" if torch.cuda.is_available() else "cpu")
        nx, ny, nz = shape
        self.shape = shape
        y = self.y_nm * 1e-9
        margin = 2.0 * r_gate if margin is None else margin
        z0, z1 = y.min() - margin, y.max() + margin
        self.h = (h_xy, h_xy, (z1 - z0) / (nz - 1))
        self.lo = (-(nx - 1) / 2 * h_xy, -(ny - 1) / 2 * h_xy, z0)
        if (nx - 1) / 2 * h_xy <= r_gate or (ny - 1) / 2 * h_xy <= r_gate:
            raise ValueError("the transverse grid must reach beyond the gate radius")
        self.eps = eps_r * EPS0
        self.tol, self.max_iter = tol, max_iter
        gx = self.lo[0] + h_xy * np.arange(nx)
        gy = self.lo[1] + h_xy * np.arange(ny)
        gz = z0 + self.h[2] * np.arange(nz)
        X, Y, Z = np.meshgrid(gx, gy, gz, indexing="ij")
        rho = np.hypot(X, Y)
        metal = (rho >= r_gate) | (Z <= z0 + 0.5 * self.h[2]) | (Z >= z1 - 0.5 * self.h[2])
        self._free = torch.tensor(~metal, device=self.dev)
        # electrode regions of the metal: wall over the contacts, end planes
        ends = (Z <= z0 + 0.5 * self.h[2]) | (Z >= z1 - 0.5 * self.h[2])
        if contact_length is not None:
            zs, zd = y.min() + contact_length, y.max() - contact_length
            src = metal & (((Z < zs) & ~ends) | (Z <= z0 + 0.5 * self.h[2]))
            drn = metal & (((Z > zd) & ~ends) | (Z >= z1 - 0.5 * self.h[2]))
        else:  # the gate wraps everything: end planes at the gate potential as well
            src = np.zeros_like(metal)
            drn = np.zeros_like(metal)
        gate = metal & ~src & ~drn
        self._elec = {"gate": torch.tensor(gate, device=self.dev), "source": torch.tensor(src, device=self.dev),
                      "drain": torch.tensor(drn, device=self.dev)}
        # atoms and their trilinear stencils
        R = float(r_tube)
        a = np.arange(m)
        pos = []
        for rr in range(self.N):
            th = a / m * 2 * np.pi + (0.0 if rr % 4 in (0, 3) else (np.sqrt(3.0) / 2.0) * (acc / R))
            pos.append(np.stack([R * np.sin(th), R * np.cos(th), np.full(m, y[rr])], 1))
        self._stencil(np.concatenate(pos), m)
        self._K = None
        self._Kd = None
        self._ext = None

    def _stencil(self, pos, m):
        """Node indices and trilinear weights of every atom (8 per atom)."""
        import torch
        nx, ny, nz = self.shape
        f = [(pos[:, d] - self.lo[d]) / self.h[d] for d in range(3)]
        i0 = [np.floor(v).astype(np.int64) for v in f]
        t = [v - i for v, i in zip(f, i0)]
        idx, w = [], []
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    ii, jj, kk = i0[0] + dx, i0[1] + dy, i0[2] + dz
                    idx.append((ii * ny + jj) * nz + kk)
                    w.append((t[0] if dx else 1 - t[0]) * (t[1] if dy else 1 - t[1]) * (t[2] if dz else 1 - t[2]))
        idx = np.stack(idx, 1)  # [atoms][8]
        w = np.stack(w, 1)
        if np.any(~self._free.cpu().numpy().reshape(-1)[idx]):
            raise ValueError("an atom's stencil touches the metal: refine the grid or enlarge the gate")
        self.m = m
        self._aidx = torch.tensor(idx, device=self.dev)
        self._aw = torch.tensor(w, device=self.dev)

    # ------------------------------------------------------------------ the operator
    def _apply(self, phi):
        """-div(eps grad phi) / eps on the free nodes (metal nodes: phi itself)."""
        import torch.nn.functional as Fn
        hx, hy, hz = self.h
        p = Fn.pad(phi, (1, 1, 1, 1, 1, 1))
        c = phi
        out = (2 * c - p[:, :-2, 1:-1, 1:-1] - p[:, 2:, 1:-1, 1:-1]) / hx ** 2 \
            + (2 * c - p[:, 1:-1, :-2, 1:-1] - p[:, 1:-1, 2:, 1:-1]) / hy ** 2 \
            + (2 * c - p[:, 1:-1, 1:-1, :-2] - p[:, 1:-1, 1:-1, 2:]) / hz ** 2
        return out * self._free

    def _cg(self, b):
        """Solve A x = b on the free nodes (x = 0 on the metal), batched."""
        import torch
        hx, hy, hz = self.h
        dinv = 1.0 / (2 / hx ** 2 + 2 / hy ** 2 + 2 / hz ** 2)
        x = torch.zeros_like(b)
        r = b.clone()
        z = r * dinv
        p = z.clone()
        rz = (r * z).sum(dim=(1, 2, 3))
        bn = b.flatten(1).norm(dim=1).clamp_min(1e-300)
        for it in range(self.max_iter):
            Ap = self._apply(p)
            alpha = rz / (p * Ap).sum(dim=(1, 2, 3))
            x += alpha.view(-1, 1, 1, 1) * p
            r -= alpha.view(-1, 1, 1, 1) * Ap
            if bool((r.flatten(1).norm(dim=1) / bn <= self.tol).all()):
                self.iterations = it + 1
                return x
            z = r * dinv
            rz_new = (r * z).sum(dim=(1, 2, 3))
            p = z + (rz_new / rz).view(-1, 1, 1, 1) * p
            rz = rz_new
        raise RuntimeError("FD Poisson: conjugate gradient did not converge")

    def _gather(self, phi):
        """Ring averages of phi at the atoms: [B][N]."""
        B = phi.shape[0]
        v = phi.reshape(B, -1)[:, self._aidx]  # [B][atoms][8]
        return (v * self._aw).sum(-1).view(B, self.N, self.m).mean(-1)

    def _deposit(self, Q):
        """Charge density / eps of ring charges Q [B][N] (units of e) on the nodes."""
        import torch
        B = Q.shape[0]
        nx, ny, nz = self.shape
        vol = self.h[0] * self.h[1] * self.h[2]
        qa = (Q * (Q_E / self.m / vol / self.eps)).repeat_interleave(self.m, dim=1)  # [B][atoms]
        rho = torch.zeros(B, nx * ny * nz, dtype=torch.float64, device=self.dev)
        rho.scatter_add_(1, self._aidx.view(1, -1).expand(B, -1), (qa[:, :, None] * self._aw[None]).reshape(B, -1))
        return rho.view(B, nx, ny, nz) * self._free

    def _build(self, batch=64):
        import torch
        nx, ny, nz = self.shape
        cols = []
        for s in range(0, self.N, batch):
            e = min(self.N, s + batch)
            Q = torch.zeros(e - s, self.N, dtype=torch.float64, device=self.dev)
            Q[torch.arange(e - s), torch.arange(s, e)] = 1.0
            cols.append(self._gather(self._cg(self._deposit(Q))))  # phi at rings from unit charges
        self._K = torch.cat(cols).T.contiguous().cpu().numpy()  # K[m][n]
        # electrode responses: phi with one electrode at 1 V, the others at 0, no charge
        ext = {}
        for name, msk in self._elec.items():
            if not bool(msk.any()):
                ext[name] = np.zeros(self.N)
                continue
            phi_d = msk.to(torch.float64)[None]  # the Dirichlet values
            b = -self._apply_full(phi_d)  # move the known values to the right-hand side
            ext[name] = (self._gather(self._cg(b) + phi_d)[0]).cpu().numpy()
        self._ext = ext

    def _apply_full(self, phi):
        """The stencil on the free nodes for a field with Dirichlet values set."""
        return self._apply(phi)

    @property
    def K(self):
        if self._K is None:
            self._build()
        return self._K

    def external(self, Vg):
        """U_ext [eV] = -phi at the rings from the electrodes (gate Vg, source 0, drain Vds)."""
        if self._ext is None:
            self._build()
        phi = float(Vg) * self._ext["gate"] + self.Vds * self._ext["drain"]
        return -phi

    def potential(self, Q, Vg):
        return self.external(Vg) - self.K @ np.asarray(Q, dtype=np.float64)

    def device_operator(self, Vg, device="cuda"):
        """(K_dev, U0_dev) for negf_affine_potential: U = U0 + Kd Q with Kd = -K."""
        import torch
        if self._Kd is None or str(self._Kd.device) != str(torch.device(device)):
            self._Kd = torch.tensor(-self.K, dtype=torch.float64, device=device).contiguous()
        return self._Kd, torch.tensor(self.external(Vg), dtype=torch.float64, device=device)
