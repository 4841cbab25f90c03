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
