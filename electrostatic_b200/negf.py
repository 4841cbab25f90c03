"""Host-side mirror of the reference's NEGF charge interface.

``CNT`` follows ``c_CNT`` / ``c_NEGF_Common<T>`` (Source/Solver/Transport/NEGF/
CNT.H:13-103, NEGF_Common.H:518-606): construction = Initialize_NEGF_Params +
Initialize_NEGF (Hamiltonian, contacts, energy limits, paths, Rho0);
``Solve_NEGF`` = set potential, update paths when the contact electrochemical
potentials changed, Compute_InducedCharge.  ``Broyden`` follows the
c_TransportSolver Broyden API (Transport.H:203-208).  Every compute call goes
through the C-ABI of libnegf_b200.so; there is no Python or CPU compute path.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import check

_dp = C.POINTER(C.c_double)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _ptr(x):
    """Device pointer of a torch tensor (or an int address)."""
    if x is None:
        return None
    if isinstance(x, int):
        return C.c_void_p(x)
    return C.c_void_p(x.data_ptr())


def _stream(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)


def tube_desc(type_id=(17, 0), num_unitcells=100, num_modes=1, acc=1.42e-10, gamma=2.5,
              contact_T=(298.0, 298.0), contact_mu=(0.0, 0.0), eq_integration_pts=(30, 30, 30),
              noneq_integration_pts=(100,), noneq_percent_intercuts=None, E_valence_min=-14.0,
              E_pole_max=10.0, E_zPlus_imag=1e-8, Fermi_tail_factors=(14.0, 14.0), use_decimation=0,
              decimation_max_iter=30, decimation_layers=10, realaxis_window=None, precision="fp64",
              mixed_fp64_band=1e-3, flatband_dos_integration_pts=100, flag_adaptive_integration_limits=0,
              integrand_correction_interval=500, kT_window_around_singularity=(1.0, 1.0),
              noneq_integration_pts_density=None, mixed_realaxis_fp32=False):
    """negf_tube_desc of the keyword arguments of CNT (host only; no device needed)."""
    L = _lib.load()
    d = _lib.TubeDesc()
    check(L.negf_tube_desc_init(C.byref(d)), "negf_tube_desc_init")
    d.type_id[0], d.type_id[1] = int(type_id[0]), int(type_id[1])
    d.num_unitcells = int(num_unitcells)
    d.num_modes = int(num_modes)
    d.acc = float(acc)
    d.gamma = float(gamma)
    d.contact_T[0], d.contact_T[1] = map(float, contact_T)
    d.contact_mu[0], d.contact_mu[1] = map(float, contact_mu)
    for i in range(3):
        d.eq_integration_pts[i] = int(eq_integration_pts[i])
    ne = list(noneq_integration_pts)
    d.num_noneq_paths = len(ne)
    for i, v in enumerate(ne):
        d.noneq_integration_pts[i] = int(v)
    if noneq_percent_intercuts is None:
        d.noneq_percent_intercuts[0] = -1.0
    else:
        for i, v in enumerate(noneq_percent_intercuts):
            d.noneq_percent_intercuts[i] = float(v)
    d.E_valence_min = float(E_valence_min)
    d.E_pole_max = float(E_pole_max)
    d.E_zPlus_imag = float(E_zPlus_imag)
    d.Fermi_tail_factors[0], d.Fermi_tail_factors[1] = map(float, Fermi_tail_factors)
    d.use_decimation = int(use_decimation)
    d.decimation_max_iter = int(decimation_max_iter)
    d.decimation_layers = int(decimation_layers)
    if realaxis_window is not None:
        lo, hi, pts, kind = realaxis_window
        d.realaxis_min, d.realaxis_max, d.realaxis_pts, d.realaxis_kind = float(lo), float(hi), int(pts), int(kind)
    d.precision = {"fp64": _lib.NEGF_PREC_FP64, "mixed": _lib.NEGF_PREC_MIXED}[precision]
    d.mixed_fp64_band = float(mixed_fp64_band)
    d.mixed_realaxis_fp32 = int(bool(mixed_realaxis_fp32))
    d.flatband_dos_integration_pts = int(flatband_dos_integration_pts)
    d.flag_adaptive_integration_limits = int(flag_adaptive_integration_limits)
    d.integrand_correction_interval = int(integrand_correction_interval)
    d.kT_window_around_singularity[0], d.kT_window_around_singularity[1] = map(float, kT_window_around_singularity)
    if noneq_integration_pts_density is not None:
        d.flag_noneq_integration_pts_density = 1
        for i, v in enumerate(noneq_integration_pts_density):
            d.noneq_integration_pts_density[i] = float(v)
    return d


def desc_energy_points(desc, kind: int):
    """Energy-point tables of a descriptor (host only): kind 0 Rho0, 1 RhoEq
    contour, 2 poles, 3 NonEq -> (E, w, J) complex arrays."""
    L = _lib.load()
    n = C.c_int()
    check(L.negf_desc_energy_points(C.byref(desc), int(kind), None, C.byref(n)), "negf_desc_energy_points")
    buf = np.zeros(6 * max(n.value, 1))
    check(L.negf_desc_energy_points(C.byref(desc), int(kind), _dptr(buf), C.byref(n)), "negf_desc_energy_points")
    b = buf[: 6 * n.value].reshape(-1, 6)
    return b[:, 0] + 1j * b[:, 1], b[:, 2] + 1j * b[:, 3], b[:, 4] + 1j * b[:, 5]


class CNT:
    """Mode-space zigzag carbon nanotube (c_CNT) on the GPU.

    Keyword names follow the reference input keys: type_id, num_unitcells,
    num_modes (BLOCK_SIZE), acc, gamma, contact_T, contact_mu,
    eq_integration_pts, num_noneq_paths, noneq_integration_pts,
    noneq_percent_intercuts, E_valence_min, E_pole_max, E_zPlus_imag,
    Fermi_tail_factors, use_decimation, decimation_max_iter,
    decimation_layers, flatband_dos_integration_pts,
    flag_adaptive_integration_limits, integrand_correction_interval,
    kT_window_around_singularity, noneq_integration_pts_density; plus
    realaxis_window=(min, max, pts, kind), precision ("fp64" | "mixed"),
    mixed_fp64_band and mixed_realaxis_fp32 (mixed mode: real-axis chains at
    least the band above the axis in FP32 too).
    """

    def __init__(self, type_id=(17, 0), num_unitcells=100, num_modes=1, acc=1.42e-10, gamma=2.5,
                 contact_T=(298.0, 298.0), contact_mu=(0.0, 0.0), eq_integration_pts=(30, 30, 30),
                 noneq_integration_pts=(100,), noneq_percent_intercuts=None, E_valence_min=-14.0,
                 E_pole_max=10.0, E_zPlus_imag=1e-8, Fermi_tail_factors=(14.0, 14.0), use_decimation=0,
                 decimation_max_iter=30, decimation_layers=10, realaxis_window=None, precision="fp64",
                 mixed_fp64_band=1e-3, flatband_dos_integration_pts=100, flag_adaptive_integration_limits=0,
                 integrand_correction_interval=500, kT_window_around_singularity=(1.0, 1.0),
                 noneq_integration_pts_density=None, mixed_realaxis_fp32=False):
        d = tube_desc(type_id=type_id, num_unitcells=num_unitcells, num_modes=num_modes, acc=acc, gamma=gamma,
                      contact_T=contact_T, contact_mu=contact_mu, eq_integration_pts=eq_integration_pts,
                      noneq_integration_pts=noneq_integration_pts, noneq_percent_intercuts=noneq_percent_intercuts,
                      E_valence_min=E_valence_min, E_pole_max=E_pole_max, E_zPlus_imag=E_zPlus_imag,
                      Fermi_tail_factors=Fermi_tail_factors, use_decimation=use_decimation,
                      decimation_max_iter=decimation_max_iter, decimation_layers=decimation_layers,
                      realaxis_window=realaxis_window, precision=precision, mixed_fp64_band=mixed_fp64_band,
                      flatband_dos_integration_pts=flatband_dos_integration_pts,
                      flag_adaptive_integration_limits=flag_adaptive_integration_limits,
                      integrand_correction_interval=integrand_correction_interval,
                      kT_window_around_singularity=kT_window_around_singularity,
                      noneq_integration_pts_density=noneq_integration_pts_density,
                      mixed_realaxis_fp32=mixed_realaxis_fp32)
        self.desc = d
        h = C.c_void_p()
        L = _lib.load()
        check(L.negf_tube_create(C.byref(d), C.byref(h)), "negf_tube_create")
        self._h = h
        n = C.c_int()
        check(L.negf_tube_num_sites(h, C.byref(n)), "negf_tube_num_sites")
        self.num_field_sites = n.value
        self.U_contact = (0.0, 0.0)

    @classmethod
    def from_deck(cls, deck, name: str, **overrides):
        """The nanostructure `name` of a ParmParse-format deck (inputs.Deck or
        a file path): NS_default / CNT_default layered under the name's keys."""
        from .inputs import Deck
        if isinstance(deck, str):
            deck = Deck.from_file(deck)
        kw = deck.tube_kwargs(name)
        kw.update(overrides)
        return cls(**kw)

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().negf_tube_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # --- geometry / modes
    def modes(self):
        L = _lib.load()
        M = int(self.desc.num_modes)
        J = (C.c_int * M)()
        dg = (C.c_int * M)()
        b = (C.c_double * M)()
        m = C.c_int()
        check(L.negf_tube_modes(self._h, C.byref(m), J, dg, b), "negf_tube_modes")
        return np.array(J[:]), np.array(dg[:]), np.array(b[:])

    def site_positions(self) -> np.ndarray:
        y = np.zeros(self.num_field_sites)
        check(_lib.load().negf_tube_site_positions(self._h, _dptr(y)), "negf_tube_site_positions")
        return y

    # --- potential and contacts
    def set_potential(self, U, U_contact=None):
        """h_U_loc_data and U_contact (default: the end-site potentials, Nanostructure.cpp:500-504)."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U_contact is None:
            U_contact = (U[0], U[-1])
        uc = (C.c_double * 2)(*map(float, U_contact))
        check(_lib.load().negf_tube_set_potential(self._h, _dptr(U), len(U), uc), "negf_tube_set_potential")
        self.U_contact = tuple(U_contact)

    def set_potential_device(self, U_dev, U_contact, stream=None):
        uc = (C.c_double * 2)(*map(float, U_contact))
        check(_lib.load().negf_tube_set_potential_device(self._h, _ptr(U_dev), self.num_field_sites, uc,
                                                         _stream(stream)), "negf_tube_set_potential_device")
        self.U_contact = tuple(U_contact)

    def potential_device_ptr(self) -> int:
        p = C.c_void_p()
        check(_lib.load().negf_tube_potential_device_ptr(self._h, C.byref(p)), "negf_tube_potential_device_ptr")
        return p.value

    def set_Contact_Electrochemical_Potential(self, mu):
        arr = (C.c_double * 2)(*map(float, mu))
        check(_lib.load().negf_tube_set_contact_mu(self._h, arr), "negf_tube_set_contact_mu")

    set_contact_mu = set_Contact_Electrochemical_Potential

    def set_energy_shard(self, rank: int, world: int):
        check(_lib.load().negf_tube_set_energy_shard(self._h, int(rank), int(world)), "negf_tube_set_energy_shard")

    # --- paths
    def energy_points(self, kind: int):
        """kind 0 Rho0, 1 RhoEq contour, 2 poles, 3 NonEq -> (E, w, J) complex arrays."""
        L = _lib.load()
        n = C.c_int()
        check(L.negf_tube_energy_points(self._h, int(kind), None, C.byref(n)), "negf_tube_energy_points")
        buf = np.zeros(6 * max(n.value, 1))
        check(L.negf_tube_energy_points(self._h, int(kind), _dptr(buf), C.byref(n)), "negf_tube_energy_points")
        b = buf[: 6 * n.value].reshape(-1, 6)
        return b[:, 0] + 1j * b[:, 1], b[:, 2] + 1j * b[:, 3], b[:, 4] + 1j * b[:, 5]

    def noneq(self) -> bool:
        v = C.c_int()
        check(_lib.load().negf_tube_noneq(self._h, C.byref(v)), "negf_tube_noneq")
        return bool(v.value)

    def get_Total_Integration_Pts(self) -> int:
        v = C.c_int()
        check(_lib.load().negf_tube_total_integration_pts(self._h, C.byref(v)), "negf_tube_total_integration_pts")
        return v.value

    # --- charge
    def Solve_NEGF(self, U=None, U_contact=None, out=None, stream=None, iter=None):
        """Solve_NEGF (NEGF_Common.cpp:1309-1340).  Returns the induced charge
        per site (numpy) or writes it into the device tensor `out`.  With
        flag_adaptive_integration_limits, iteration numbers that are multiples
        of integrand_correction_interval first correct the non-equilibrium
        intercuts (:1316-1336)."""
        if U is not None:
            self.set_potential(U, U_contact)
        d = self.desc
        if iter is not None and d.flag_adaptive_integration_limits and iter % d.integrand_correction_interval == 0:
            self.correct_integration_limits(stream=stream)
        return compute_charge([self], out=out, stream=stream)

    def correct_integration_limits(self, stream=None):
        check(_lib.load().negf_tube_correct_integration_limits(self._h, _stream(stream)),
              "negf_tube_correct_integration_limits")

    def noneq_integrand(self, stream=None):
        """Compute_RhoNonEq integrand probes [3][P] (sites N/2, N/4, 3N/4)."""
        P = len(self.energy_points(3)[0]) if self.noneq() else 0
        out = np.zeros(3 * max(P, 1))
        check(_lib.load().negf_tube_noneq_integrand(self._h, _dptr(out), _stream(stream)), "negf_tube_noneq_integrand")
        return out[: 3 * P].reshape(3, P)

    def noneq_layout(self):
        """(points per path, intercuts in percent, E* of the last correction)."""
        n = C.c_int()
        pts = (C.c_int * _lib.NEGF_MAX_NONEQ_PATHS)()
        cuts = np.zeros(_lib.NEGF_MAX_NONEQ_PATHS)
        Es = np.zeros(1)
        check(_lib.load().negf_tube_noneq_layout(self._h, C.byref(n), pts, _dptr(cuts), _dptr(Es)),
              "negf_tube_noneq_layout")
        return np.array(pts[: n.value]), cuts[: max(n.value - 1, 0)].copy(), float(Es[0])

    def Compute_InducedCharge(self, out=None, stream=None):
        return compute_charge([self], out=out, stream=stream)

    def realspace_charge(self, out=None, U_atoms=None, stream=None):
        """Induced charge per ring from the real-space ring-block RGF (zigzag
        tubes): contour and poles, plus the non-equilibrium real-axis term
        when the tube is biased.  U_atoms: optional device tensor [N][m] of
        per-atom potentials.  Mixed-precision tubes run the contour chains far
        from the real axis in FP32 on the tensor cores.  Returns numpy unless
        `out` (device float64) is given."""
        import torch
        Q = out if out is not None else torch.zeros(self.num_field_sites, dtype=torch.float64, device="cuda")
        check(_lib.load().negf_rs_compute_charge(self._h, _ptr(U_atoms), _ptr(Q), _stream(stream)),
              "negf_rs_compute_charge")
        return Q if out is not None else Q.cpu().numpy()

    # --- transport characteristics (PostProcess, Nanostructure.H:134-138)
    def Compute_DensityOfStates(self, ldos=False, stream=None) -> dict:
        """Compute_DensityOfStates (NEGF_Common.cpp:2390-2847) on the GPU: dict
        with E (complex), dos, T, conductance, total_conductance and, with
        ldos=True, ldos [E][N]."""
        L = _lib.load()
        n = C.c_int()
        check(L.negf_tube_dos_points(self._h, C.byref(n)), "negf_tube_dos_points")
        P = n.value
        E = np.zeros(2 * P)
        dos, T, cond = np.zeros(P), np.zeros(P), np.zeros(P)
        tot = np.zeros(1)
        ld = np.zeros(P * self.num_field_sites) if ldos else None
        check(L.negf_compute_dos(self._h, _dptr(E), _dptr(dos), _dptr(T), _dptr(cond), _dptr(tot),
                                 None if ld is None else ld.ctypes.data_as(C.c_void_p), _stream(stream)),
              "negf_compute_dos")
        out = dict(E=E[0::2] + 1j * E[1::2], dos=dos, T=T, conductance=cond, total_conductance=float(tot[0]))
        if ldos:
            out["ldos"] = ld.reshape(P, self.num_field_sites)
        return out

    def Compute_Current(self, integrand=False, stream=None):
        """Compute_Current (NEGF_Common.cpp:4321-4816) on the GPU: terminal
        currents [A] of contacts 0 and 1 and, with integrand=True, the
        (channel, source, drain) integrand probes [3][P] with their energies."""
        L = _lib.load()
        n = C.c_int()
        check(L.negf_tube_current_points(self._h, C.byref(n)), "negf_tube_current_points")
        I = np.zeros(2)
        pr = np.zeros(3 * max(n.value, 1)) if integrand else None
        check(L.negf_compute_current(self._h, _dptr(I), None if pr is None else pr.ctypes.data_as(C.c_void_p),
                                     _stream(stream)), "negf_compute_current")
        if not integrand:
            return I
        E = self.energy_points(3)[0] if n.value else np.zeros(0, complex)
        return I, pr[: 3 * n.value].reshape(3, n.value), E

    def Write_Eql_Characteristics(self, path: str, res: dict):
        E = np.ascontiguousarray(np.stack([res["E"].real, res["E"].imag], 1).ravel())
        check(_lib.load().negf_write_transport_char(self._h, path.encode(), len(res["dos"]), _dptr(E),
                                                    _dptr(res["dos"]), _dptr(res["T"]), _dptr(res["conductance"])),
              "negf_write_transport_char")

    def Write_Integrand(self, path: str, E, integrand):
        Eb = np.ascontiguousarray(np.stack([np.real(E), np.imag(E)], 1).ravel())
        pr = np.ascontiguousarray(integrand, dtype=np.float64)
        check(_lib.load().negf_write_integrand(self._h, path.encode(), len(E), _dptr(Eb), _dptr(pr)),
              "negf_write_integrand")

    def Write_Data(self, prefix: str, Q, norm=None):
        Q = np.ascontiguousarray(Q, dtype=np.float64)
        nrm = None if norm is None else _dptr(np.ascontiguousarray(norm, dtype=np.float64))
        check(_lib.load().negf_write_step(self._h, prefix.encode(), _dptr(Q), nrm), "negf_write_step")


def compute_charge(tubes: Sequence[CNT], out=None, stream=None):
    """Induced charge of a batch of tubes in one launch (Q of tube t at offset
    sum of the previous tubes' sites).  `out`: device tensor (float64) or None
    for a host numpy result."""
    L = _lib.load()
    arr = (C.c_void_p * len(tubes))(*[t.handle for t in tubes])
    total = sum(t.num_field_sites for t in tubes)
    if out is None:
        Q = np.zeros(total)
        check(L.negf_compute_charge(arr, len(tubes), Q.ctypes.data_as(C.c_void_p), 0, _stream(stream)),
              "negf_compute_charge")
        return Q
    check(L.negf_compute_charge(arr, len(tubes), _ptr(out), 1, _stream(stream)), "negf_compute_charge")
    return out


def release_scratch(stream=None):
    """negf_release_scratch: hand back the device scratch that the charge
    calls keep for the current device and `stream` (reallocated by the next
    call on that stream)."""
    check(_lib.load().negf_release_scratch(_stream(stream)), "negf_release_scratch")


def last_stats() -> dict:
    s = _lib.Stats()
    check(_lib.load().negf_last_stats(C.byref(s)), "negf_last_stats")
    return {k: getattr(s, k) for k, _ in _lib.Stats._fields_}


def set_timing(enable: bool):
    check(_lib.load().negf_set_timing(int(bool(enable))), "negf_set_timing")


TUNE_PASS2_WARPS_PER_BLOCK = 2
TUNE_PASS1_PIECES = 4
TUNE_SCHEDULE = 6
TUNE_NN_GEMM = 7
SCHEDULE_AUTO, SCHEDULE_TWO_PASS, SCHEDULE_FUSED = 0, 1, 2
NN_GEMM_DEFAULT, NN_GEMM_TCGEN05, NN_GEMM_MMA_SYNC, NN_GEMM_TCGEN05_STAGED = 0, 1, 2, 3


def set_tuning(key: int, value: int):
    """negf_set_tuning: launch-shape knobs of the charge calls (TUNE_* keys)."""
    check(_lib.load().negf_set_tuning(int(key), int(value)), "negf_set_tuning")


def shard_range(num_points: int, rank: int, world: int):
    lo, hi = C.c_int(), C.c_int()
    check(_lib.load().negf_shard_range(int(num_points), int(rank), int(world), C.byref(lo), C.byref(hi)),
          "negf_shard_range")
    return lo.value, hi.value


class Broyden:
    """Broyden modified-second mixing on the device (Set_Broyden_Parallel /
    Execute_Broyden_Modified_Second_Algorithm_Parallel / Reset_Broyden_Parallel)."""

    def __init__(self, n_in, max_step=200, fraction=0.1, norm_type="absolute", stream=None):
        L = _lib.load()
        self.S = int(n_in.shape[0])
        nt = _lib.NEGF_NORM_ABSOLUTE if norm_type.lower().startswith("abs") else _lib.NEGF_NORM_RELATIVE
        h = C.c_void_p()
        check(L.negf_broyden_create(self.S, int(max_step), float(fraction), nt, C.byref(h)), "negf_broyden_create")
        self._h = h
        if isinstance(n_in, np.ndarray):
            a = np.ascontiguousarray(n_in, dtype=np.float64)
            check(L.negf_broyden_set_input(h, a.ctypes.data_as(C.c_void_p), 0, _stream(stream)), "set_input")
        else:
            check(L.negf_broyden_set_input(h, _ptr(n_in), 1, _stream(stream)), "set_input")

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().negf_broyden_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n_out_dev, n_in_out=None, norm_out=None, stream=None) -> float:
        """One mixing step; returns Broyden_Norm (max residual of this input)."""
        mx = C.c_double()
        st = C.c_int()
        check(_lib.load().negf_broyden_step(self._h, _ptr(n_out_dev), _ptr(n_in_out), _ptr(norm_out),
                                            C.byref(mx), C.byref(st), _stream(stream)), "negf_broyden_step")
        return mx.value

    Execute_Broyden_Modified_Second_Algorithm_Parallel = step

    def step_device_switch(self, n_out_dev, max_norm, switch_norm, flags_dev, stream=None):
        """Device-resident step with precision switching (flags_dev int32[8])."""
        check(_lib.load().negf_broyden_step_device_switch(self._h, _ptr(n_out_dev), float(max_norm), float(switch_norm),
                                                          _ptr(flags_dev), _stream(stream)),
              "negf_broyden_step_device_switch")

    def step_device(self, n_out_dev, max_norm, flags_dev, stream=None):
        """Device-resident step (capturable): flags_dev int32[4] on the device
        = converged, steps taken, error, skip."""
        check(_lib.load().negf_broyden_step_device(self._h, _ptr(n_out_dev), float(max_norm), _ptr(flags_dev),
                                                   _stream(stream)), "negf_broyden_step_device")

    def reset(self, keep_charge=False, init_value=0.0, stream=None):
        check(_lib.load().negf_broyden_reset(self._h, int(bool(keep_charge)), float(init_value), _stream(stream)),
              "negf_broyden_reset")

    Reset_Broyden_Parallel = reset

    def history(self, stream=None):
        """(V, W, rows): zero-copy device views [rows][S] of the secant rows held now."""
        from .scf import device_view
        v, w, r = C.c_void_p(), C.c_void_p(), C.c_int()
        check(_lib.load().negf_broyden_history(self._h, C.byref(v), C.byref(w), C.byref(r), _stream(stream)),
              "negf_broyden_history")
        S = self.S
        return device_view(v.value, r.value * S).view(r.value, S), device_view(w.value, r.value * S).view(r.value, S), \
            r.value

    def restart(self, keep_rows=100, stream=None):
        """Next solve with the secant rows so far (at most keep_rows, the most
        recent) as its initial inverse Jacobian; n_in stays."""
        check(_lib.load().negf_broyden_restart(self._h, int(keep_rows), _stream(stream)), "negf_broyden_restart")

    def set_segments(self, offsets, stream=None):
        """Per-segment secant updates (one Broyden per segment, e.g. per tube)
        for offsets [0, ..., num_sites]; [0, num_sites] is the whole-vector
        update.  Call after create or reset, before seeding and stepping."""
        off = np.ascontiguousarray(offsets, dtype=np.int32)
        check(_lib.load().negf_broyden_set_segments(self._h, len(off) - 1,
                                                    off.ctypes.data_as(C.POINTER(C.c_int)), _stream(stream)),
              "negf_broyden_set_segments")

    def set_initial_jacobian(self, V, W, stream=None):
        """Initial inverse Jacobian G0 = fraction I + sum_j W[j] V[j]^T for the
        next solve (V, W: device float64 [k][S]); call after create or reset."""
        k = 0 if V is None else int(V.shape[0])
        check(_lib.load().negf_broyden_set_initial_jacobian(self._h, _ptr(V), _ptr(W), k, _stream(stream)),
              "negf_broyden_set_initial_jacobian")

    @staticmethod
    def secant_rows(dn, dF, fraction=0.1):
        """Rows (V, W) of the modified-second method for secant pairs
        dn[j], dF[j] (device float64 [k][S]): V[j] = dF[j] / |dF[j]|^2,
        W[j] = -fraction dF[j] + dn[j] - sum_{i<j} W[i] (V[i] . dF[j])
        (Broyden_Second_Parallel.cpp:381-403)."""
        V = dF / (dF * dF).sum(dim=1, keepdim=True)
        W = -fraction * dF + dn
        for j in range(1, dF.shape[0]):
            c = V[:j] @ dF[j]
            W[j] -= c @ W[:j]
        return V, W

    @property
    def step_number(self) -> int:
        v = C.c_int()
        check(_lib.load().negf_broyden_step_number(self._h, C.byref(v)), "negf_broyden_step_number")
        return v.value

    def input_device_ptr(self) -> int:
        p = C.c_void_p()
        check(_lib.load().negf_broyden_input_device_ptr(self._h, C.byref(p)), "negf_broyden_input_device_ptr")
        return p.value


def affine_potential(K_dev, U0_dev, Q_dev, U_dev, stream=None):
    n = int(U0_dev.shape[0])
    check(_lib.load().negf_affine_potential(_ptr(K_dev), _ptr(U0_dev), _ptr(Q_dev), _ptr(U_dev), n, _stream(stream)),
          "negf_affine_potential")


def write_current_header(path: str):
    """Define_FileHeaderForCurrent (NEGF_Common.cpp:69-84): append the I.dat header."""
    check(_lib.load().negf_write_current_header(path.encode()), "negf_write_current_header")


def write_current(path: str, step: int, Vds: float, Vgs: float, current, avg_intg_pts: float,
                  total_iterations: int, total_conductance: float):
    """Write_Current (NEGF_Common.cpp:4818-4840): append one I.dat line."""
    I = np.ascontiguousarray(current, dtype=np.float64)
    check(_lib.load().negf_write_current(path.encode(), int(step), float(Vds), float(Vgs), _dptr(I),
                                         float(avg_intg_pts), int(total_iterations), float(total_conductance)),
          "negf_write_current")


# --- file naming and restart (NEGF_Common.cpp:87-140, 178-285, 565-621)
NAME_DIGITS = 4  # negf_plt_name_digits, NEGF_Common.H:65


def concatenate(root: str, num: int, digits: int = NAME_DIGITS) -> str:
    """amrex::Concatenate: root followed by num zero-padded to `digits` digits."""
    return f"{root}{num:0{digits}d}"


def step_filename(folder: str, name: str, step: int) -> str:
    """Set_StepFilenameString: <folder>/<name>/stepNNNN."""
    return concatenate(f"{folder}/{name}/step", step)


def iter_filename(step_prefix: str, it: int) -> str:
    """Set_IterationFilenameString: <stepNNNN>_iter/iterMMMM."""
    return concatenate(f"{step_prefix}_iter/iter", it)


def restart_charge_filename(folder: str, name: str, restart_step: int) -> str:
    """Read_AtomLocationAndChargeDistributionFilename with restart: the
    _Qout.dat of step restart_step - 1."""
    return step_filename(folder, name, restart_step - 1) + "_Qout.dat"


def read_table1d(filename: str, n: int) -> np.ndarray:
    """Read_Table1D: the value column of a header + n-line table."""
    out = np.zeros(n)
    check(_lib.load().negf_read_table1d(filename.encode(), int(n), _dptr(out)), "negf_read_table1d")
    return out


class ChargePlan:
    """A batch of tubes with its launch tables on the device: launch() is
    kernel launches only (capturable in a CUDA graph); the contact potentials
    follow the end sites of each tube's potential buffer."""

    def __init__(self, tubes: Sequence[CNT], out, autotune=False, fp64=False):
        L = _lib.load()
        self.tubes = list(tubes)
        self.out = out
        arr = (C.c_void_p * len(tubes))(*[t.handle for t in tubes])
        h = C.c_void_p()
        flags = (_lib.NEGF_PLAN_AUTOTUNE if autotune else 0) | (_lib.NEGF_PLAN_FP64 if fp64 else 0)
        check(L.negf_charge_plan_create(arr, len(tubes), _ptr(out), flags, C.byref(h)), "negf_charge_plan_create")
        self._h = h

    def launch(self, skip=None, stream=None):
        check(_lib.load().negf_charge_plan_launch(self._h, _ptr(skip), _stream(stream)), "negf_charge_plan_launch")

    def info(self) -> dict:
        w, s, ms, up = C.c_int(), C.c_int(), C.c_double(), C.c_longlong()
        check(_lib.load().negf_charge_plan_info(self._h, C.byref(w), C.byref(s), C.byref(ms), C.byref(up)),
              "negf_charge_plan_info")
        pc = C.c_int()
        check(_lib.load().negf_charge_plan_pieces(self._h, C.byref(pc)), "negf_charge_plan_pieces")
        return dict(pass2_warps_per_block=w.value, segs_per_unit=s.value, tuned_ms=ms.value, updates=up.value,
                    pieces=pc.value)

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().negf_charge_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def affine_potential_toeplitz(tab_dev, idx_dev, U0_dev, Q_dev, U_dev, n, skip, stream=None):
    """U = U0 + K Q with K[i][j] = tab[|idx[i] - idx[j]|] (negf_affine_potential_toeplitz)."""
    check(_lib.load().negf_affine_potential_toeplitz(_ptr(tab_dev), int(tab_dev.numel()), _ptr(idx_dev), _ptr(U0_dev),
                                                     _ptr(Q_dev), _ptr(U_dev), int(n), _ptr(skip), _stream(stream)),
          "negf_affine_potential_toeplitz")


class PotentialBatch:
    """negf_potential_batch: the lattice-distance potential update of a batch of
    tubes in one launch (tables, lattice indices and U0 as device tensors; Q and
    U as device tensors or addresses, fixed at creation)."""

    def __init__(self, tabs, idxs, U0s, Qs, Us, ns):
        T = len(ns)

        def arr(vals):
            return (C.c_void_p * T)(*[_ptr(v) for v in vals])

        ntab = (C.c_int * T)(*[int(t.numel()) for t in tabs])
        nn = (C.c_int * T)(*[int(n) for n in ns])
        h = C.c_void_p()
        check(_lib.load().negf_potential_batch_create(T, arr(tabs), ntab, arr(idxs), arr(U0s), arr(Qs), arr(Us), nn,
                                                      C.byref(h)), "negf_potential_batch_create")
        self._h = h
        self._keep = (list(tabs), list(idxs), list(U0s), list(Qs), list(Us))

    def launch(self, skip=None, stream=None):
        check(_lib.load().negf_potential_batch_launch(self._h, _ptr(skip), _stream(stream)),
              "negf_potential_batch_launch")

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().negf_potential_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def affine_potential_masked(K_dev, U0_dev, Q_dev, U_dev, n, skip, stream=None):
    check(_lib.load().negf_affine_potential_masked(_ptr(K_dev), _ptr(U0_dev), _ptr(Q_dev), _ptr(U_dev), int(n),
                                                   _ptr(skip), _stream(stream)), "negf_affine_potential_masked")
