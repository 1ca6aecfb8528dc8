"""ctypes binding of the C ABI declared in include/kapsel_spm.h.

The library is the in-tree build kapsel3_b200/_lib/libkapsel_spm.so.  There is
no fallback: if the library is missing or fails to load, every entry point of
this package raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

from . import build as _build

SPM_OK = 0
SPM_ERR_ARG = 1
SPM_ERR_CUDA = 2
SPM_ERR_NOMEM = 3
SPM_ERR_DEVICE = 4
SPM_ERR_NO_DEVICE = 5
SPM_PARTICLE_WORDS = 44
SPM_RIGID_WORDS = 16
SPM_RIGID_STATE_WORDS = 63
SPM_EQ_NAVIER_STOKES = 0
SPM_EQ_LEES_EDWARDS = 1
SPM_EQ_ELECTROLYTE = 2
SPM_EQ_SHEAR_NAVIER_STOKES = 3
SPM_JANUS_OFF, SPM_JANUS_TUMBLER, SPM_JANUS_SQUIRMER, SPM_JANUS_OBSTACLE = 0, 1, 2, 3
SPM_AXIS_NONE, SPM_AXIS_X, SPM_AXIS_Y, SPM_AXIS_Z = 0, 1, 2, 3
SPM_MAX_SPECIES = 4
SPM_PREC_FP64 = 0
SPM_PREC_FP32_MIXED = 1

HEADER = os.path.join(_build.ROOT, "include", "kapsel_spm.h")


class SpmParams(C.Structure):
    _fields_ = [
        ("npx", C.c_int), ("npy", C.c_int), ("npz", C.c_int),
        ("dx", C.c_double), ("rho", C.c_double), ("eta", C.c_double), ("kbt", C.c_double),
        ("alpha_v", C.c_double), ("alpha_o", C.c_double),
        ("equation", C.c_int),
        ("shear_rate", C.c_double),
        ("n_particles", C.c_int),
        ("mass_ratio", C.c_double),
        ("a", C.c_double), ("a_xi", C.c_double),
        ("epsilon", C.c_double),
        ("lj_powers", C.c_int), ("lj_truncate", C.c_int),
        ("rotation", C.c_int),
        ("fix_cell", C.c_int * 3),
        ("dt", C.c_double),
        ("body_force", C.c_double * 3),
        ("precision", C.c_int),
        ("mt_seed", C.c_uint),
        ("dielectric", C.c_double), ("salt", C.c_int), ("init_pb", C.c_int),
        ("valency", C.c_double * 2), ("onsager", C.c_double * 2), ("debye_length", C.c_double),
        ("surface_charge", C.c_double), ("e_field", C.c_int), ("e_ext", C.c_double * 3),
        ("e_frequency", C.c_double),
        ("janus_axis", C.c_int),
        ("janus_propulsion", C.c_int),
        ("janus_force", C.c_double * 3),
        ("janus_torque", C.c_double * 3),
        ("slip_vel", C.c_double),
        ("slip_mode", C.c_double),
        ("rotlet_c1", C.c_double),
        ("rotlet_c2", C.c_double),
        ("slip_tol", C.c_double),
        ("slip_iter", C.c_int),
        ("n_species", C.c_int),
        ("species_count", C.c_int * 4),
        ("species_mass_ratio", C.c_double * 4),
        ("species_surface_charge", C.c_double * 4),
        ("shear_ac", C.c_int),
        ("shear_frequency", C.c_double),
        ("rigid", C.c_int),
        ("rigid_beads", C.c_int * 4),
        ("rigid_count", C.c_int * 4),
        ("rigid_free", (C.c_int * 6) * 4),
        ("rigid_velocity", (C.c_double * 3) * 4),
        ("rigid_omega", (C.c_double * 3) * 4),
        ("rigid_gravity", C.c_double * 3),
    ]


class SpmServerConfig(C.Structure):
    _fields_ = [
        ("budget_bytes", C.c_size_t),
        ("pool_initial_capacity", C.c_int),
        ("use_graph", C.c_int),
        ("steps_per_launch", C.c_int),
        ("poll_us", C.c_int),
        ("device", C.c_int),
        ("pool_idle_s", C.c_double),
    ]


class SpmServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_longlong), ("rejected", C.c_longlong), ("admitted", C.c_longlong),
        ("completed", C.c_longlong), ("failed", C.c_longlong), ("cancelled", C.c_longlong),
        ("queued", C.c_longlong),
        ("run_steps", C.c_longlong),
        ("graph_captures", C.c_longlong),
        ("max_active", C.c_int),
        ("used_bytes", C.c_size_t), ("peak_bytes", C.c_size_t),
        ("busy_s", C.c_double),
        ("step_latency_p50_ms", C.c_double), ("step_latency_p99_ms", C.c_double),
        ("step_latency_max_ms", C.c_double),
        ("pool_step_device_p50_ms", C.c_double), ("pool_step_device_p99_ms", C.c_double),
        ("pool_create_max_ms", C.c_double), ("admit_max_ms", C.c_double), ("pool_destroy_max_ms", C.c_double),
        ("launch_max_ms", C.c_double), ("finish_max_ms", C.c_double),
    ]


SPM_REQ_QUEUED, SPM_REQ_RUNNING, SPM_REQ_DONE, SPM_REQ_FAILED, SPM_REQ_CANCELLED = range(5)
SPM_REQ_KEEP_VELOCITY = 1


class SpmError(RuntimeError):
    pass


_lib = None

_P = C.c_void_p
_D = C.POINTER(C.c_double)
_SIGS = {
    "spm_last_error": (C.c_char_p, []),
    "spm_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "spm_params_size": (C.c_size_t, []),
    "spm_params_default": (C.c_int, [C.POINTER(SpmParams)]),
    "spm_params_from_udf_keys": (C.c_int, [C.c_char_p, C.POINTER(SpmParams), _D, C.c_int]),
    "spm_params_from_udf": (C.c_int, [C.c_char_p, C.POINTER(SpmParams), _D, C.c_int]),
    "spm_udf_read_keys": (C.c_int, [C.c_char_p, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "spm_create": (C.c_int, [C.POINTER(SpmParams), _P, C.POINTER(_P)]),
    "spm_destroy": (C.c_int, [_P]),
    "spm_device_bytes": (C.c_int, [C.POINTER(SpmParams), C.POINTER(C.c_size_t)]),
    "spm_initialize": (C.c_int, [_P, _D]),
    "spm_step": (C.c_int, [_P, C.c_int]),
    "spm_synchronize": (C.c_int, [_P]),
    "spm_get_particles": (C.c_int, [_P, _D]),
    "spm_set_particles": (C.c_int, [_P, _D]),
    "spm_get_zeta": (C.c_int, [_P, _D, _D, _D]),
    "spm_set_zeta": (C.c_int, [_P, _D, _D, _D]),
    "spm_get_velocity": (C.c_int, [_P, _D, _D, _D]),
    "spm_get_phi": (C.c_int, [_P, _D]),
    "spm_get_time": (C.c_int, [_P, C.POINTER(C.c_int), _D]),
    "spm_get_shear_state": (C.c_int, [_P, _D, _D]),
    "spm_get_concentration": (C.c_int, [_P, C.c_int, _D]),
    "spm_set_solute": (C.c_int, [_P, C.c_int, _D, C.c_double]),
    "spm_save_state": (C.c_int, [_P, C.c_char_p]),
    "spm_load_state": (C.c_int, [_P, C.c_char_p]),
    "spm_load_restart": (C.c_int, [_P, C.c_char_p]),
    "spm_set_time": (C.c_int, [_P, C.c_int, C.c_double, C.c_double]),
    "spm_udf_out_open": (C.c_int, [_P, C.c_char_p]),
    "spm_udf_out_record": (C.c_int, [_P]),
    "spm_udf_out_close": (C.c_int, [_P]),
    "spm_save_restart": (C.c_int, [_P, C.c_char_p, C.c_char_p]),
    "spm_avs_open": (C.c_int, [_P, C.c_char_p, C.c_char_p, C.c_int]),
    "spm_avs_frame": (C.c_int, [_P]),
    "spm_avs_flush": (C.c_int, [_P]),
    "spm_avs_close": (C.c_int, [_P]),
    "spm_ns_solver_slaved_euler_host": (C.c_int, [_P, _D, _D, _D]),
    "spm_solenoidal_uk_host": (C.c_int, [_P, _D, _D, _D]),
    "spm_zeta_k2u_k_host": (C.c_int, [_P, _D, _D, _D, _D, _D, _D]),
    "spm_u_k2zeta_k_host": (C.c_int, [_P, _D, _D, _D, _D, _D, _D]),
    "spm_a2a_k_host": (C.c_int, [_P, _D]),
    "spm_a_k2a_host": (C.c_int, [_P, _D]),
    "spm_make_phi_particle_sum_host": (C.c_int, [_P, _D, _D, _D]),
    "spm_make_u_particle_sum_host": (C.c_int, [_P, _D, _D, _D, _D, _D]),
    "spm_make_phi_u_particle_host": (C.c_int, [_P, _D, _D, _D, _D, _D]),
    "spm_make_f_particle_dt_sole_host": (C.c_int, [_P, _D, _D, _D, _D, _D, _D, _D, _D, _D, _D]),
    "spm_calc_f_hydro_correct_precision_host": (C.c_int, [_P, _D, _D, _D, _D, _D]),
    "spm_calc_f_lennard_jones_host": (C.c_int, [_P, _D]),
    "spm_fft_forward_dev": (C.c_int, [_P, _P, C.c_int, C.c_size_t]),
    "spm_fft_inverse_dev": (C.c_int, [_P, _P, C.c_int, C.c_size_t]),
    "spm_row_complex": (C.c_int, [_P, C.POINTER(C.c_int)]),
    "spm_time_steps": (C.c_int, [_P, C.c_int, C.POINTER(C.c_float)]),
    "spm_kernel_launches": (C.c_int, [_P, C.POINTER(C.c_longlong), C.c_int]),
    "spm_profile_pass": (C.c_int, [_P, C.c_int, _D, _D, C.POINTER(C.c_longlong)]),
    "spm_profile_kernels": (C.c_int, [_P, C.c_int, C.c_char_p, C.c_size_t]),
    "spm_rigid_count": (C.c_int, [_P, C.POINTER(C.c_int)]),
    "spm_get_rigid": (C.c_int, [_P, _D]),
    "spm_get_rigid_state": (C.c_int, [_P, _D, _D]),
    "spm_set_rigid_state": (C.c_int, [_P, _D, _D]),
    "spm_make_f_particle_dt_sole_noalloc": (C.c_int, [_P] * 10 + [C.c_int, C.c_int, C.c_int, _P]),
    "spm_pool_device_bytes": (C.c_int, [C.POINTER(SpmParams), C.c_int, C.POINTER(C.c_size_t),
                                        C.POINTER(C.c_size_t)]),
    "spm_pool_create": (C.c_int, [C.POINTER(SpmParams), C.c_int, _P, C.POINTER(_P)]),
    "spm_pool_destroy": (C.c_int, [_P]),
    "spm_pool_admit": (C.c_int, [_P, C.POINTER(SpmParams), _D, C.POINTER(_P)]),
    "spm_pool_release": (C.c_int, [_P, _P]),
    "spm_pool_size": (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "spm_pool_run": (C.c_int, [_P, C.c_int, C.POINTER(_P)]),
    "spm_pool_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "spm_pool_step": (C.c_int, [_P, C.c_int, C.c_int]),
    "spm_pool_query": (C.c_int, [_P, C.POINTER(C.c_int)]),
    "spm_pool_synchronize": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_uint)]),
    "spm_pool_stats": (C.c_int, [_P, C.POINTER(C.c_longlong), C.POINTER(C.c_int)]),
    "spm_debug_fail_allocations": (C.c_int, [C.c_int]),
    "spm_set_wait_limit": (C.c_int, [_P, C.c_double]),
    "spm_debug_skip_tma_loads": (C.c_int, [_P, C.c_int]),
    "spm_release_cached_memory": (C.c_int, [C.POINTER(C.c_size_t)]),
    "spm_server_config_default": (C.c_int, [C.POINTER(SpmServerConfig)]),
    "spm_server_create": (C.c_int, [C.POINTER(SpmServerConfig), C.POINTER(_P)]),
    "spm_server_destroy": (C.c_int, [_P]),
    "spm_server_submit": (C.c_int, [_P, C.POINTER(SpmParams), _D, C.c_int, C.c_int, C.POINTER(C.c_longlong)]),
    "spm_server_cancel": (C.c_int, [_P, C.c_longlong]),
    "spm_server_wait": (C.c_int, [_P, C.c_longlong, C.c_double, C.POINTER(C.c_int)]),
    "spm_server_status": (C.c_int, [_P, C.c_longlong, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                    C.POINTER(C.c_int), C.c_char_p, C.c_size_t]),
    "spm_server_result": (C.c_int, [_P, C.c_longlong, _D, _D, _D, _D, _D, _D]),
    "spm_server_forget": (C.c_int, [_P, C.c_longlong]),
    "spm_server_get_stats": (C.c_int, [_P, C.POINTER(SpmServerStats)]),
    "spm_server_latencies": (C.c_int, [_P, C.POINTER(C.c_float), C.c_size_t, C.POINTER(C.c_size_t)]),
}


def declared_symbols():
    """Every function the public header declares."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(spm_[a-z0-9_]+)\s*\(", text))
                  - {"spm_params", "spm_ctx", "spm_pool", "spm_server", "spm_server_config", "spm_server_stats"})


def lib(build_if_missing: bool = True):
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if not os.path.exists(path):
        if not build_if_missing:
            raise SpmError(f"native library missing: {path}")
        _build.build()
    L = C.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    if L.spm_params_size() != C.sizeof(SpmParams):
        raise SpmError(f"{path} was built from another kapsel_spm.h: spm_params is {L.spm_params_size()} bytes "
                       f"there, {C.sizeof(SpmParams)} in this binding")
    _lib = L
    return L


def check(rc: int, what: str = ""):
    if rc != SPM_OK:
        msg = lib().spm_last_error().decode(errors="replace")
        raise SpmError(f"{what} failed (status {rc}): {msg}")


def dptr(a):
    """double* of a C-contiguous float64 numpy array."""
    assert a.dtype.name == "float64" and a.flags["C_CONTIGUOUS"], "need a contiguous float64 array"
    return a.ctypes.data_as(_D)
