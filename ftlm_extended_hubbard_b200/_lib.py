"""ctypes binding of the C ABI declared in include/ftlm_gpu.h (libftlm_gpu.so, built in-tree).

Loading fails loudly when the library is missing: there is no CPU fallback for any of the
compute entry points.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libftlm_gpu.so")

FTLM_OK = 0
FTLM_ERR_INVALID = 1
FTLM_QUAD_REFERENCE = 0
FTLM_QUAD_CONVERGED = 1
FTLM_ERR_CUDA = 2
FTLM_ERR_NOMEM = 3
FTLM_ERR_TIMEOUT = 4
FTLM_ERR_UNSUPPORTED = 5
FTLM_ERR_NUMERIC = 6
FTLM_START_REFERENCE = 0
FTLM_START_PHILOX = 1


class FtlmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[ftlm status {code}] {msg}")
        self.code = code


class FtlmParams(C.Structure):
    _fields_ = [("Lx", C.c_int), ("Ly", C.c_int), ("t", C.c_double), ("tp", C.c_double), ("U", C.c_double),
                ("V", C.c_double), ("phi_x", C.c_double), ("phi_y", C.c_double)]


class FtlmHop(C.Structure):
    _fields_ = [("frm", C.c_int), ("to", C.c_int), ("spin", C.c_int), ("coeff_re", C.c_double),
                ("coeff_im", C.c_double)]


class FtlmPair(C.Structure):
    _fields_ = [("i", C.c_int), ("j", C.c_int)]


_vp = C.c_void_p
_i = C.c_int
_d = C.c_double
_ll = C.c_longlong
_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int)

# name -> argtypes (all return int status unless listed in _RESTYPES)
SIGNATURES = {
    "ftlm_gpu_last_error": [],
    "ftlm_gpu_version_string": [],
    "ftlm_gpu_device_count": [_pi],
    "ftlm_gpu_build_geometry": [C.POINTER(FtlmParams), C.POINTER(FtlmHop), _i, _pi, C.POINTER(FtlmPair), _i, _pi],
    "ftlm_gpu_sector_create": [C.POINTER(FtlmParams), _i, _i, C.POINTER(_vp)],
    "ftlm_gpu_sector_create_hops": [_i, _i, _i, _d, _d, C.POINTER(FtlmHop), _i, C.POINTER(FtlmPair), _i,
                                    C.POINTER(_vp)],
    "ftlm_gpu_sector_create_host": [_i, _i, _i, _d, _d, C.POINTER(FtlmHop), _i, C.POINTER(FtlmPair), _i,
                                    C.POINTER(_vp)],
    "ftlm_gpu_sector_destroy": [_vp],
    "ftlm_gpu_sector_dim": [_vp, C.POINTER(_ll)],
    "ftlm_gpu_sector_masks": [_vp, _vp, _vp],
    "ftlm_gpu_sector_index_of": [_vp, C.c_uint64, C.c_uint64, C.POINTER(_ll)],
    "ftlm_gpu_sector_state": [_vp, _ll, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)],
    "ftlm_gpu_lanczos_host_op": [_ll, _vp, _vp, _i, C.c_uint, _i, _vp, _vp, _pi, _pi],
    "ftlm_gpu_ftlm_combine": [_vp, _vp, _vp, _i, _i, _d, _vp, _vp],
    "ftlm_gpu_sector_stats": [_vp, _pd, _pd, C.POINTER(_ll), C.POINTER(_ll)],
    "ftlm_gpu_sector_diag": [_vp, _ll, _pd],
    "ftlm_gpu_sector_down_table": [_vp, C.POINTER(_ll), C.POINTER(_ll), _vp, _vp, _pi],
    "ftlm_gpu_sector_down_table_gauge": [_vp, _pi, C.POINTER(_ll), C.POINTER(_ll), _pi, _vp, _vp, _vp, _vp],
    "ftlm_gpu_sector_down_table_form": [_vp, _pi, _vp, _pi, _vp],
    "ftlm_gpu_sector_up_table_packed": [_vp, _pi, C.POINTER(_ll), _vp, _vp, _vp, _vp],
    "ftlm_gpu_apply": [_vp, _vp, _vp, _vp],
    "ftlm_gpu_apply_host": [_vp, _vp, _vp],
    "ftlm_gpu_apply_profiled": [_vp, _vp, _vp, _vp, C.POINTER(C.c_float), _pi],
    "ftlm_gpu_set_apply_path": [_vp, _i],
    "ftlm_gpu_lanczos": [_vp, _i, C.c_uint, _i, _vp, _vp, _pi, _pi],
    "ftlm_gpu_lanczos_extrema": [_vp, _i, C.c_uint, _i, _pd, _pd, _pi],
    "ftlm_gpu_lanczos_op": [_ll, _vp, _vp, _i, C.c_uint, _i, _vp, _vp, _pi, _pi],
    "ftlm_gpu_tridiag_eig": [_vp, _vp, _vp, _i, _i, _i, _d, _vp, _vp],
    "ftlm_gpu_tridiag_quadrature": [_vp, _vp, _vp, _i, _i, _vp, _i, _vp, _vp],
    "ftlm_gpu_ritz_values": [_vp, _vp, _i, _i, _vp],
    "ftlm_gpu_tridiag_quadrature_noalloc": [_vp, _vp, _vp, _i, _i, _vp, _i, _vp, _vp, _vp],
    "ftlm_gpu_ftlm_sector": [_vp, _vp, _i, _i, _i, C.c_uint, _i, _vp, _vp],
    "ftlm_gpu_gc_reduce": [_vp, _vp, _vp, _i, _vp, _i, _vp, _i, _i, _vp, _vp, _vp],
    "ftlm_gpu_batched_lanczos": [_vp, _i, _i, C.c_uint, _vp, _vp, _vp],
    "ftlm_gpu_batched_set_cols_variant": [_vp, _i],
    "ftlm_gpu_batched_autotune": [_vp, _i, _vp, _vp],
    "ftlm_gpu_batched_ftlm_sector": [_vp, _vp, _i, _i, _i, C.c_uint, _vp, _vp],
    "ftlm_gpu_batched_sweep": [C.POINTER(FtlmParams), _i, _i, C.c_uint, _vp, _i, _vp, _i, _vp, _vp, _vp, _vp, _vp],
    "ftlm_gpu_batched_release": [],
    "ftlm_gpu_batched_ftlm_sector_checked": [_vp, _vp, _i, _i, _i, C.c_uint, _i, _vp, _vp, _vp],
    "ftlm_gpu_batched_sweep_checked": [C.POINTER(FtlmParams), _i, _i, C.c_uint, _vp, _i, _vp, _i, _i, _vp, _vp, _vp,
                                       _vp, _vp, _vp, _vp, _vp],
    "ftlm_gpu_set_fused_max_dim": [_ll],
    "ftlm_gpu_set_quadrature": [_i],
    "ftlm_gpu_autotune_apply": [_vp, _i, _vp, _vp, _vp],
    "ftlm_gpu_set_cols_variant": [_vp, _i],
    "ftlm_gpu_lanczos_sectors": [_vp, _i, _i, _i, C.c_uint, _i, _vp, _vp, _vp],
    "ftlm_gpu_grad_sector": [_vp, _vp, _d, _i, _i, C.c_uint, _i, _i, _vp, _vp],
    "ftlm_gpu_gc_logz": [C.POINTER(FtlmParams), _d, _d, _i, _i, C.c_uint, _i, _i, _vp, _vp, _pd],
    "ftlm_gpu_gc_logz_grad": [C.POINTER(FtlmParams), _d, _d, _i, _i, C.c_uint, _i, _i, _vp, _vp, _vp],
    "ftlm_gpu_tridiag_eigvec": [_vp, _vp, _i, _vp, _vp],
    "ftlm_gpu_tridiag_quadrature_exact": [_vp, _vp, _vp, _i, _i, _vp, _i, _vp, _vp],
    "ftlm_gpu_duhamel_weights": [_vp, _vp, _i, _d, _vp, _vp, _vp],
    "ftlm_gpu_orbit_create": [_vp, _i, _i, C.POINTER(_vp)],
    "ftlm_gpu_orbit_create_ex": [_vp, _i, _i, _d, C.POINTER(_vp)],
    "ftlm_gpu_sector_set_lattice": [_vp, _i, _i],
    "ftlm_gpu_orbit_entries_ex": [_vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "ftlm_gpu_orbit_destroy": [_vp],
    "ftlm_gpu_orbit_set_apply_path": [_vp, _i],
    "ftlm_gpu_orbit_dim": [_vp, C.POINTER(_ll)],
    "ftlm_gpu_orbit_entries": [_vp, _vp, _vp],
    "ftlm_gpu_orbit_apply": [_vp, _vp, _vp, _vp],
    "ftlm_gpu_orbit_apply_host": [_vp, _vp, _vp],
    "ftlm_gpu_orbit_ftlm": [_vp, _vp, _i, _i, _i, C.c_uint, _i, _vp, _vp],
    "ftlm_gpu_orbit_sector_ftlm": [_vp, _vp, _i, _i, _i, C.c_uint, _i, _i, _i, _vp, _vp, _vp],
    "ftlm_gpu_orbit_batched_ftlm": [_vp, _vp, _i, _i, _i, C.c_uint, _vp, _vp],
    "ftlm_gpu_orbit_sector_batched_ftlm": [_vp, _vp, _i, _i, _i, C.c_uint, _i, _i, _vp, _vp, _vp],
    "ftlm_gpu_gc_sweep": [C.POINTER(FtlmParams), _i, _i, C.c_uint, _i, _vp, _i, _vp, _i, _vp, _vp, _vp, _vp, _vp],
}
_RESTYPES = {"ftlm_gpu_last_error": C.c_char_p, "ftlm_gpu_version_string": C.c_char_p}

APPLY_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.c_void_p)

_lib = None


def lib() -> C.CDLL:
    """The loaded native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FtlmError(FTLM_ERR_UNSUPPORTED,
                            f"native library missing: {LIB_PATH} (run python -m ftlm_extended_hubbard_b200.build)")
        L = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = _RESTYPES.get(name, C.c_int)
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != FTLM_OK:
        raise FtlmError(status, lib().ftlm_gpu_last_error().decode())


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))
