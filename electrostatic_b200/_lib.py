"""ctypes binding of libnegf_b200.so (declarations of include/negf_b200.h).

Loading fails loudly when the library has not been built: the package has no
CPU fallback for any compute call.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libnegf_b200.so")

NEGF_OK = 0
NEGF_PREC_FP64 = 0
NEGF_PREC_MIXED = 1
NEGF_NORM_ABSOLUTE = 0
NEGF_NORM_RELATIVE = 1
NEGF_MAX_NONEQ_PATHS = 8
NEGF_PLAN_AUTOTUNE = 1
NEGF_PLAN_FP64 = 2

# Every symbol include/negf_b200.h declares (checked by the CPU test suite).
EXPORTED = [
    "negf_tube_desc_init", "negf_tube_create", "negf_tube_destroy", "negf_tube_num_sites", "negf_tube_modes",
    "negf_tube_site_positions", "negf_tube_set_potential", "negf_tube_set_potential_device",
    "negf_tube_potential_device_ptr", "negf_tube_set_contact_mu", "negf_tube_energy_points",
    "negf_desc_energy_points", "negf_tube_noneq",
    "negf_tube_total_integration_pts", "negf_tube_set_energy_shard", "negf_shard_range", "negf_compute_charge",
    "negf_last_stats", "negf_set_timing", "negf_set_tuning", "negf_broyden_create", "negf_broyden_destroy", "negf_broyden_set_input",
    "negf_broyden_step", "negf_broyden_reset", "negf_broyden_step_number", "negf_broyden_input_device_ptr",
    "negf_broyden_set_initial_jacobian", "negf_broyden_restart", "negf_broyden_history", "negf_broyden_set_segments",
    "negf_affine_potential", "negf_write_step", "negf_last_error", "negf_device_selftest",
    "negf_compute_charge_noalloc", "negf_tube_dos_points", "negf_tube_current_points", "negf_compute_dos",
    "negf_compute_current", "negf_write_transport_char", "negf_write_current_header", "negf_write_current",
    "negf_write_integrand", "negf_tube_correct_integration_limits", "negf_tube_noneq_integrand",
    "negf_tube_noneq_layout", "negf_read_table1d", "negf_broyden_step_device", "negf_affine_potential_masked",
    "negf_charge_plan_create", "negf_charge_plan_launch", "negf_charge_plan_info", "negf_charge_plan_destroy",
    "negf_broyden_step_device_switch", "negf_rs_compute_charge", "negf_nn_gemm", "negf_nn_gelu_fwd",
    "negf_nn_gelu_bwd", "negf_nn_colsum", "negf_nn_cast_bf16", "negf_nn_adam", "negf_nn_rowdot", "negf_nn_outer",
    "negf_nn_mse", "negf_affine_potential_toeplitz", "negf_potential_batch_create", "negf_potential_batch_launch",
    "negf_potential_batch_destroy", "negf_charge_plan_pieces", "negf_release_scratch",
]


class TubeDesc(C.Structure):
    _fields_ = [
        ("type_id", C.c_int * 2),
        ("num_unitcells", C.c_int),
        ("num_modes", C.c_int),
        ("acc", C.c_double),
        ("gamma", C.c_double),
        ("contact_T", C.c_double * 2),
        ("contact_mu", C.c_double * 2),
        ("eq_integration_pts", C.c_int * 3),
        ("num_noneq_paths", C.c_int),
        ("noneq_integration_pts", C.c_int * NEGF_MAX_NONEQ_PATHS),
        ("noneq_percent_intercuts", C.c_double * NEGF_MAX_NONEQ_PATHS),
        ("E_valence_min", C.c_double),
        ("E_pole_max", C.c_double),
        ("E_zPlus_imag", C.c_double),
        ("Fermi_tail_factors", C.c_double * 2),
        ("use_decimation", C.c_int),
        ("decimation_max_iter", C.c_int),
        ("decimation_layers", C.c_int),
        ("realaxis_min", C.c_double),
        ("realaxis_max", C.c_double),
        ("realaxis_pts", C.c_int),
        ("realaxis_kind", C.c_int),
        ("precision", C.c_int),
        ("mixed_fp64_band", C.c_double),
        ("flatband_dos_integration_pts", C.c_int),
        ("flag_adaptive_integration_limits", C.c_int),
        ("integrand_correction_interval", C.c_int),
        ("kT_window_around_singularity", C.c_double * 2),
        ("flag_noneq_integration_pts_density", C.c_int),
        ("noneq_integration_pts_density", C.c_double * NEGF_MAX_NONEQ_PATHS),
        ("mixed_realaxis_fp32", C.c_int),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("rgf_kernel_ms", C.c_double),
        ("pass1_kernel_ms", C.c_double),
        ("pass2_kernel_ms", C.c_double),
        ("reduce_kernel_ms", C.c_double),
        ("updates", C.c_longlong),
        ("updates_fp32", C.c_longlong),
        ("contour_updates", C.c_longlong),
        ("realaxis_updates", C.c_longlong),
        ("chains", C.c_int),
        ("warps", C.c_int),
        ("units", C.c_int),
        ("kernel_launches", C.c_int),
        ("pieces", C.c_int),
        ("checkpoint_bytes", C.c_longlong),
        ("schedule", C.c_int),
    ]


class NEGFError(RuntimeError):
    pass


_lib = None


def load():
    """Load libnegf_b200.so (build it first with electrostatic_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise NEGFError(f"{LIB_PATH} is missing: build it with `python -m electrostatic_b200.build` "
                        "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
    sig = {
        "negf_tube_desc_init": [C.POINTER(TubeDesc)],
        "negf_tube_create": [C.POINTER(TubeDesc), C.POINTER(vp)],
        "negf_tube_destroy": [vp],
        "negf_tube_num_sites": [vp, ip],
        "negf_tube_modes": [vp, ip, ip, ip, dp],
        "negf_tube_site_positions": [vp, dp],
        "negf_tube_set_potential": [vp, dp, C.c_int, dp],
        "negf_tube_set_potential_device": [vp, vp, C.c_int, dp, vp],
        "negf_tube_potential_device_ptr": [vp, C.POINTER(vp)],
        "negf_tube_set_contact_mu": [vp, dp],
        "negf_tube_energy_points": [vp, C.c_int, dp, ip],
        "negf_desc_energy_points": [C.POINTER(TubeDesc), C.c_int, dp, ip],
        "negf_tube_noneq": [vp, ip],
        "negf_tube_total_integration_pts": [vp, ip],
        "negf_tube_set_energy_shard": [vp, C.c_int, C.c_int],
        "negf_shard_range": [C.c_int, C.c_int, C.c_int, ip, ip],
        "negf_compute_charge": [C.POINTER(vp), C.c_int, vp, C.c_int, vp],
        "negf_compute_charge_noalloc": [C.POINTER(vp), C.c_int, vp, vp],
        "negf_last_stats": [C.POINTER(Stats)],
        "negf_release_scratch": [vp],
        "negf_set_timing": [C.c_int],
        "negf_set_tuning": [C.c_int, C.c_int],
        "negf_broyden_create": [C.c_int, C.c_int, C.c_double, C.c_int, C.POINTER(vp)],
        "negf_broyden_destroy": [vp],
        "negf_broyden_set_input": [vp, vp, C.c_int, vp],
        "negf_broyden_step": [vp, vp, vp, vp, dp, ip, vp],
        "negf_broyden_reset": [vp, C.c_int, C.c_double, vp],
        "negf_broyden_set_initial_jacobian": [vp, vp, vp, C.c_int, vp],
        "negf_broyden_restart": [vp, C.c_int, vp],
        "negf_broyden_set_segments": [vp, C.c_int, ip, vp],
        "negf_broyden_history": [vp, C.POINTER(vp), C.POINTER(vp), ip, vp],
        "negf_broyden_step_number": [vp, ip],
        "negf_broyden_input_device_ptr": [vp, C.POINTER(vp)],
        "negf_affine_potential": [vp, vp, vp, vp, C.c_int, vp],
        "negf_write_step": [vp, C.c_char_p, dp, dp],
        "negf_last_error": [],
        "negf_device_selftest": [C.c_int, C.c_int, dp, dp],
        "negf_tube_dos_points": [vp, ip],
        "negf_tube_current_points": [vp, ip],
        "negf_compute_dos": [vp, dp, dp, dp, dp, dp, vp, vp],
        "negf_compute_current": [vp, dp, vp, vp],
        "negf_write_transport_char": [vp, C.c_char_p, C.c_int, dp, dp, dp, dp],
        "negf_write_current_header": [C.c_char_p],
        "negf_write_current": [C.c_char_p, C.c_int, C.c_double, C.c_double, dp, C.c_double, C.c_int, C.c_double],
        "negf_write_integrand": [vp, C.c_char_p, C.c_int, dp, dp],
        "negf_tube_correct_integration_limits": [vp, vp],
        "negf_tube_noneq_integrand": [vp, dp, vp],
        "negf_tube_noneq_layout": [vp, ip, ip, dp, dp],
        "negf_read_table1d": [C.c_char_p, C.c_int, dp],
        "negf_broyden_step_device": [vp, vp, C.c_double, vp, vp],
        "negf_broyden_step_device_switch": [vp, vp, C.c_double, C.c_double, vp, vp],
        "negf_rs_compute_charge": [vp, vp, vp, vp],
        "negf_nn_gemm": [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, vp, C.c_int, C.c_longlong, vp, C.c_int,
                         C.c_longlong, vp, C.c_int, C.c_longlong, vp, C.c_int, vp],
        "negf_nn_gelu_fwd": [C.c_longlong, C.c_int, vp, vp, vp, vp, vp, vp, C.c_int, vp],
        "negf_nn_gelu_bwd": [C.c_longlong, vp, vp, vp, vp, vp],
        "negf_nn_colsum": [C.c_longlong, C.c_int, vp, vp, C.c_int, vp],
        "negf_nn_cast_bf16": [C.c_longlong, vp, vp, vp],
        "negf_nn_adam": [C.c_longlong, vp, vp, vp, vp, vp, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int,
                         C.c_float, vp],
        "negf_nn_rowdot": [C.c_longlong, C.c_int, vp, vp, vp, vp, vp],
        "negf_nn_outer": [C.c_longlong, C.c_int, vp, vp, vp, vp, vp],
        "negf_nn_mse": [C.c_longlong, vp, vp, vp, vp, vp],
        "negf_affine_potential_masked": [vp, vp, vp, vp, C.c_int, vp, vp],
        "negf_affine_potential_toeplitz": [vp, C.c_int, vp, vp, vp, vp, C.c_int, vp, vp],
        "negf_potential_batch_create": [C.c_int, C.POINTER(vp), ip, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp),
                                        C.POINTER(vp), ip, C.POINTER(vp)],
        "negf_potential_batch_launch": [vp, vp, vp],
        "negf_potential_batch_destroy": [vp],
        "negf_charge_plan_create": [C.POINTER(vp), C.c_int, vp, C.c_int, C.POINTER(vp)],
        "negf_charge_plan_launch": [vp, vp, vp],
        "negf_charge_plan_info": [vp, ip, ip, dp, C.POINTER(C.c_longlong)],
        "negf_charge_plan_destroy": [vp],
        "negf_charge_plan_pieces": [vp, ip],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int
    L.negf_last_error.restype = C.c_char_p
    _lib = L
    return L


def check(rc: int, what: str = "") -> None:
    if rc != NEGF_OK:
        msg = load().negf_last_error().decode(errors="replace")
        raise NEGFError(f"{what} failed ({rc}): {msg}")
