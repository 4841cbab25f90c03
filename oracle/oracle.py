"""ORACLE — test infrastructure only.

ctypes front end of ``liboracle.so``, the CPU FP64 restatement of the
ELEQTRONeX NEGF charge path (``negf_oracle.cpp`` cites the reference lines
each routine restates).  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this module; the product library never
does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (g++ only)."""
    src = os.path.join(_HERE, "negf_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-C", _HERE, "-s", "liboracle.so"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_gauss_legendre.argtypes = [C.c_int, _dp, _dp]
        L.orc_fixture_sigma_dos_T.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, _dp, C.c_double,
                                              C.c_int, _dp, _dp, _dp]
        L.orc_tube_new.restype = C.c_void_p
        L.orc_tube_new.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double]
        L.orc_tube_free.argtypes = [C.c_void_p]
        L.orc_tube_num_sites.argtypes = [C.c_void_p]
        L.orc_tube_num_modes.argtypes = [C.c_void_p]
        L.orc_tube_radius.argtypes = [C.c_void_p]
        L.orc_tube_radius.restype = C.c_double
        L.orc_tube_modes.argtypes = [C.c_void_p, _ip, _ip, _dp, _dp]
        L.orc_tube_set_contacts.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double]
        L.orc_tube_set_integration.argtypes = [C.c_void_p, _ip, C.c_int, _ip, C.c_void_p, C.c_double,
                                               C.c_double, C.c_double, C.c_double, C.c_double]
        L.orc_tube_set_realaxis_window.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_int]
        L.orc_tube_set_decimation.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int]
        L.orc_tube_set_sgf_mode.argtypes = [C.c_void_p, C.c_int]
        L.orc_tube_set_potential.argtypes = [C.c_void_p, _dp, C.c_double, C.c_double]
        L.orc_tube_sigma.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double, _dp]
        L.orc_tube_paths.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_tube_noneq.argtypes = [C.c_void_p]
        L.orc_tube_rho0.argtypes = [C.c_void_p, C.c_int]
        L.orc_tube_charge.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_tube_partial.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, _dp]
        L.orc_tube_sample.restype = C.c_longlong
        L.orc_tube_sample.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, _dp]
        L.orc_tube_dos.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p]
        L.orc_tube_set_flatband_dos_pts.argtypes = [C.c_void_p, C.c_int]
        L.orc_tube_current.argtypes = [C.c_void_p, C.c_int, _dp, C.c_void_p]
        L.orc_tube_noneq_integrand.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_tube_set_adaptive.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_void_p]
        L.orc_tube_correct_limits.argtypes = [C.c_void_p, C.c_int]
        L.orc_tube_noneq_layout.argtypes = [C.c_void_p, _ip, _dp, _dp]
        L.orc_tube_rs_charge.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, _dp]
        L.orc_broyden_new.restype = C.c_void_p
        L.orc_broyden_new.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int, _dp]
        L.orc_broyden_free.argtypes = [C.c_void_p]
        L.orc_broyden_step.restype = C.c_double
        L.orc_broyden_step.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.orc_broyden_stepno.argtypes = [C.c_void_p]
        L.orc_broyden_reset.argtypes = [C.c_void_p, C.c_int, C.c_double]
        _lib = L
    return _lib


def gauss_legendre(n: int):
    x = np.zeros(n)
    w = np.zeros(n)
    lib().orc_gauss_legendre(n, x, w)
    return x, w


def fixture_sigma_dos_T(N, beta, gamma, E, eta, root):
    """Sigma (nE,4), DOS (nE,2), T (nE,2) of the standalone RGF test programs."""
    E = np.ascontiguousarray(E, dtype=np.float64)
    nE = len(E)
    sig = np.zeros(4 * nE)
    dos = np.zeros(2 * nE)
    T = np.zeros(2 * nE)
    lib().orc_fixture_sigma_dos_T(N, beta, gamma, nE, E, eta, root, sig, dos, T)
    return sig.reshape(nE, 4), dos.reshape(nE, 2), T.reshape(nE, 2)


class OracleTube:
    """One nanotube of the oracle.  Parameter names follow the reference's
    input keys (``NS_default.*`` / ``CNT_default.*``)."""

    def __init__(self, type_id=(17, 0), num_unitcells=100, num_modes=1, acc=1.42e-10, gamma=2.5,
                 contact_T=(298.0, 298.0), contact_mu=(0.0, 0.0), eq_integration_pts=(30, 30, 30),
                 noneq_integration_pts=(100,), noneq_percent_intercuts=None, E_valence_min=-14.0,
                 E_pole_max=10.0, E_zPlus_imag=1e-8, Fermi_tail_factors=(14.0, 14.0),
                 realaxis_window=None, use_decimation=0, decimation_max_iter=30, decimation_layers=10,
                 decimation_rel_error=1e-5, decimation_tol_is_int=1, sgf_mode=0):
        L = lib()
        self._h = L.orc_tube_new(int(type_id[0]), int(type_id[1]), int(num_unitcells), int(num_modes),
                                 float(acc), float(gamma))
        self.N = L.orc_tube_num_sites(self._h)
        self.M = L.orc_tube_num_modes(self._h)
        L.orc_tube_set_contacts(self._h, contact_T[0], contact_T[1], contact_mu[0], contact_mu[1])
        eq = np.asarray(eq_integration_pts, dtype=np.int32)
        ne = np.asarray(noneq_integration_pts, dtype=np.int32)
        cuts = None
        if noneq_percent_intercuts is not None:
            self._cuts = np.ascontiguousarray(noneq_percent_intercuts, dtype=np.float64)
            cuts = self._cuts.ctypes.data_as(C.c_void_p)
        L.orc_tube_set_integration(self._h, eq, len(ne), ne, cuts, E_valence_min, E_pole_max, E_zPlus_imag,
                                   Fermi_tail_factors[0], Fermi_tail_factors[1])
        if realaxis_window is not None:
            lo, hi, pts, kind = realaxis_window
            L.orc_tube_set_realaxis_window(self._h, lo, hi, int(pts), int(kind))
        L.orc_tube_set_decimation(self._h, int(use_decimation), int(decimation_max_iter),
                                  int(decimation_layers), float(decimation_rel_error), int(decimation_tol_is_int))
        L.orc_tube_set_sgf_mode(self._h, int(sgf_mode))

    def __del__(self):
        try:
            if self._h:
                lib().orc_tube_free(self._h)
        except Exception:
            pass

    @property
    def radius(self):
        return lib().orc_tube_radius(self._h)

    def modes(self):
        J = np.zeros(self.M, np.int32)
        d = np.zeros(self.M, np.int32)
        b = np.zeros(self.M)
        g = np.zeros(self.M)
        lib().orc_tube_modes(self._h, J, d, b, g)
        return J, d, b, g

    def set_potential(self, U, U_contact):
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert len(U) == self.N
        lib().orc_tube_set_potential(self._h, U, float(U_contact[0]), float(U_contact[1]))

    def sigma(self, mode, E, Uc=0.0):
        out = np.zeros(2)
        lib().orc_tube_sigma(self._h, mode, E.real, E.imag, Uc, out)
        return complex(out[0], out[1])

    def paths(self, kind):
        """kind: 0 Rho0, 1 RhoEq contour, 2 poles, 3 NonEq.  Returns (E, w, J) complex arrays."""
        L = lib()
        n = L.orc_tube_paths(self._h, kind, None)
        buf = np.zeros(6 * max(n, 1))
        L.orc_tube_paths(self._h, kind, buf.ctypes.data_as(C.c_void_p))
        b = buf[: 6 * n].reshape(n, 6)
        return b[:, 0] + 1j * b[:, 1], b[:, 2] + 1j * b[:, 3], b[:, 4] + 1j * b[:, 5]

    def noneq(self):
        return bool(lib().orc_tube_noneq(self._h))

    def rho0(self, nthreads=1):
        lib().orc_tube_rho0(self._h, int(nthreads))

    def charge(self, faithful=False, nthreads=1, components=False):
        Q = np.zeros(self.N)
        if not components:
            lib().orc_tube_charge(self._h, int(faithful), int(nthreads), Q, None, None, None)
            return Q
        a, b, c = np.zeros(self.N), np.zeros(self.N), np.zeros(self.N)
        lib().orc_tube_charge(self._h, int(faithful), int(nthreads), Q, a.ctypes.data_as(C.c_void_p),
                              b.ctypes.data_as(C.c_void_p), c.ctypes.data_as(C.c_void_p))
        return Q, a, b, c

    def partial(self, kind, e_lo, e_hi, nthreads=1):
        out = np.zeros(self.N)
        lib().orc_tube_partial(self._h, int(kind), int(e_lo), int(e_hi), int(nthreads), out)
        return out


def _sample(self, stride, offset=0, faithful=True, nthreads=1):
    """Partial charge of the energy points with index = offset (mod stride);
    returns (per-site partial, number of updates)."""
    out = np.zeros(self.N)
    n = lib().orc_tube_sample(self._h, int(faithful), int(nthreads), int(stride), int(offset), out)
    return out, int(n)


OracleTube.sample = _sample


def _dos(self, faithful=True, nthreads=1, ldos=False, flatband_pts=None):
    """Compute_DensityOfStates over the tube's DOS path: dict with E (complex),
    dos, T, conductance, total_conductance and, if asked, ldos [E][N]."""
    L = lib()
    if flatband_pts is not None:
        L.orc_tube_set_flatband_dos_pts(self._h, int(flatband_pts))
    P = L.orc_tube_dos(self._h, int(faithful), int(nthreads), None, None, None, None, None, None)
    E = np.zeros(2 * P)
    dos, T, cond = np.zeros(P), np.zeros(P), np.zeros(P)
    tot = np.zeros(1)
    ld = np.zeros(P * self.N) if ldos else None
    vp = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
    L.orc_tube_dos(self._h, int(faithful), int(nthreads), vp(E), vp(dos), vp(T), vp(cond), vp(tot), vp(ld))
    out = dict(E=E[0::2] + 1j * E[1::2], dos=dos, T=T, conductance=cond, total_conductance=float(tot[0]))
    if ldos:
        out["ldos"] = ld.reshape(P, self.N)
    return out


def _current(self, nthreads=1, probes=False):
    """Compute_Current: (I[2], probes [3][P] or None) over the non-equilibrium paths."""
    L = lib()
    I = np.zeros(2)
    n = len(self.paths(3)[0])
    pr = np.zeros(3 * max(n, 1)) if probes else None
    L.orc_tube_current(self._h, int(nthreads), I, None if pr is None else pr.ctypes.data_as(C.c_void_p))
    return I, (pr[: 3 * n].reshape(3, n) if probes else None)


def _noneq_integrand(self, nthreads=1):
    """Compute_RhoNonEq integrand probes [3][P] (site N/2, N/4, 3N/4)."""
    L = lib()
    P = L.orc_tube_noneq_integrand(self._h, 1, None)
    out = np.zeros(3 * max(P, 1))
    L.orc_tube_noneq_integrand(self._h, int(nthreads), out.ctypes.data_as(C.c_void_p))
    return out[: 3 * P].reshape(3, P)


def _correct_limits(self, nthreads=1, kT_window=(1.0, 1.0), density=None):
    """One adaptive correction of the non-equilibrium intercuts and points
    (the window and the optional point densities are fixed on first use)."""
    L = lib()
    if not getattr(self, "_adaptive", False) or density is not None:
        self._dens = np.ascontiguousarray([] if density is None else density, dtype=np.float64)
        L.orc_tube_set_adaptive(self._h, kT_window[0], kT_window[1], len(self._dens),
                                self._dens.ctypes.data_as(C.c_void_p) if len(self._dens) else None)
        self._adaptive = True
    L.orc_tube_correct_limits(self._h, int(nthreads))


def _noneq_layout(self):
    pts = np.zeros(8, np.int32)
    cuts = np.zeros(8)
    Emax = np.zeros(1)
    n = lib().orc_tube_noneq_layout(self._h, pts, cuts, Emax)
    return pts[:n].copy(), cuts[: max(n - 1, 0)].copy(), float(Emax[0])


OracleTube.noneq_integrand = _noneq_integrand
OracleTube.correct_limits = _correct_limits
OracleTube.noneq_layout = _noneq_layout
def _rs_charge(self, Uatoms=None, iters=32, nthreads=1):
    """Real-space ring-block charge per ring (zigzag tubes): contour, poles and,
    when biased, the non-equilibrium real-axis term."""
    Q = np.zeros(self.N)
    ua = None
    if Uatoms is not None:
        self._ua = np.ascontiguousarray(Uatoms, dtype=np.float64)
        ua = self._ua.ctypes.data_as(C.c_void_p)
    rc = lib().orc_tube_rs_charge(self._h, ua, int(iters), int(nthreads), Q)
    if rc != 0:
        raise ValueError("real-space charge needs a zigzag tube")
    return Q


OracleTube.rs_charge = _rs_charge
OracleTube.dos = _dos
OracleTube.current = _current


class OracleBroyden:
    """Broyden modified-second mixing (CPU branch of the reference)."""

    def __init__(self, n_in, max_step=200, fraction=0.1, norm_type="absolute"):
        n_in = np.ascontiguousarray(n_in, dtype=np.float64)
        self.S = len(n_in)
        nt = 0 if norm_type.lower().startswith("abs") else 1
        self._h = lib().orc_broyden_new(self.S, int(max_step), float(fraction), nt, n_in)

    def __del__(self):
        try:
            if self._h:
                lib().orc_broyden_free(self._h)
        except Exception:
            pass

    def step(self, n_out):
        n_out = np.ascontiguousarray(n_out, dtype=np.float64)
        n_in = np.zeros(self.S)
        nrm = np.zeros(self.S)
        mx = lib().orc_broyden_step(self._h, n_out, n_in, nrm)
        return mx, n_in, nrm

    @property
    def step_number(self):
        return lib().orc_broyden_stepno(self._h)

    def reset(self, keep_charge=False, init_value=0.0):
        lib().orc_broyden_reset(self._h, int(bool(keep_charge)), float(init_value))
