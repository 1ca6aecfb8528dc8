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
SPM_PARTICLE_WORDS = 44
SPM_EQ_NAVIER_STOKES = 0
SPM_EQ_LEES_EDWARDS = 1
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
    ]


class SpmError(RuntimeError):
    pass


_lib = None

_P = C.c_void_p
_D = C.POINTER(C.c_double)
_SIGS = {
    "spm_last_error": (C.c_char_p, []),
    "spm_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "spm_params_default": (C.c_int, [C.POINTER(SpmParams)]),
    "spm_params_from_udf_keys": (C.c_int, [C.c_char_p, C.POINTER(SpmParams), _D, C.c_int]),
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
    "spm_make_f_particle_dt_sole_noalloc": (C.c_int, [_P] * 10 + [C.c_int, C.c_int, C.c_int, _P]),
}


def declared_symbols():
    """Every function the public header declares."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(spm_[a-z0-9_]+)\s*\(", text)) - {"spm_params", "spm_ctx"})


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
