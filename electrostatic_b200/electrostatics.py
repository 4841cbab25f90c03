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


class GateAllAround:
    """Affine potential operator of a gate-all-around tube: U = -V_g - K Q."""

    def __init__(self, y_nm, r_tube, r_gate, eps_r=3.9, smear=0.1e-9):
        self.K = ring_coupling_matrix(y_nm, r_tube, r_gate, eps_r, smear)
        self.N = len(y_nm)

    def potential(self, Q, Vg):
        return -float(Vg) - self.K @ np.asarray(Q, dtype=np.float64)

    def device_operator(self, Vg, device="cuda"):
        """(K_dev, U0_dev) for negf_affine_potential: U = U0 + Kd Q with Kd = -K
        (Kd is uploaded once and reused)."""
        import torch
        if getattr(self, "_Kd", None) is None or str(self._Kd.device) != str(torch.device(device)):
            self._Kd = torch.tensor(-self.K, dtype=torch.float64, device=device).contiguous()
        U0 = torch.full((self.N,), -float(Vg), dtype=torch.float64, device=device)
        return self._Kd, U0
