"""ctypes binding of libpbbfmm3d_b200.so (the C ABI in include/pbbfmm3d_b200.h).

The shared library is built in-tree by ``pbbfmm3d_b200/csrc/Makefile`` (see
``pbbfmm3d_b200.build``).  There is no CPU fallback: if the library is
missing or fails to load, every call raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpbbfmm3d_b200.so")

# status codes
OK, ERR_ARG, ERR_CUDA, ERR_ALLOC, ERR_STATE, ERR_IO, ERR_UNSUPPORTED, ERR_NUMERIC, ERR_TIMEOUT = range(9)
PREC_FP64, PREC_MIXED = 0, 1
TC_OFF, TC_F16, TC_TF32 = 0, 1, 2


class FMMError(RuntimeError):
    """Raised when a C-ABI call returns a non-zero status."""

    def __init__(self, code: int, msg: str):
        super().__init__("pbbfmm error %d: %s" % (code, msg))
        self.code = code


class TreeParams(ctypes.Structure):
    _fields_ = [
        ("L", ctypes.c_double),
        ("tree_level", ctypes.c_int),
        ("interpolation_order", ctypes.c_int),
        ("epsilon", ctypes.c_double),
        ("use_chebyshev", ctypes.c_int),
        ("kernel", ctypes.c_int),
        ("kernel_param", ctypes.c_double * 4),
    ]


_lib = None
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p
_i64 = ctypes.c_int64

EXPORTS = {
    "pbbfmm_tree_create": ([ctypes.POINTER(TreeParams), ctypes.c_int, ctypes.POINTER(_vp)], ctypes.c_int),
    "pbbfmm_tree_create_user": ([ctypes.POINTER(TreeParams), _vp, ctypes.c_int, ctypes.POINTER(_vp)],
                                ctypes.c_int),
    "pbbfmm_tree_build": ([_vp, ctypes.c_char_p], ctypes.c_int),
    "pbbfmm_tree_set_operators": ([_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp], ctypes.c_int),
    "pbbfmm_tree_get_operators": ([_vp, _ip, _ip, _ip, _dp, _dp, _dp], ctypes.c_int),
    "pbbfmm_tree_destroy": ([_vp], ctypes.c_int),
    "pbbfmm_compute": ([_vp, _dp, _i64, _dp, _i64, _dp, ctypes.c_int, _dp], ctypes.c_int),
    "pbbfmm_compute_device": ([_vp, _vp, _i64, _vp, _i64, _vp, ctypes.c_int, _vp, ctypes.c_int, _vp], ctypes.c_int),
    "pbbfmm_compute_adjoint_device": ([_vp, _vp, _i64, _vp, _i64, _vp, _vp, ctypes.c_int, _vp, _vp,
                                       _vp, ctypes.c_int, _vp], ctypes.c_int),
    "pbbfmm_set_precision": ([_vp, ctypes.c_int], ctypes.c_int),
    "pbbfmm_set_tensor_cores": ([_vp, ctypes.c_int], ctypes.c_int),
    "pbbfmm_tensor_core_m2l": ([_vp], ctypes.c_int),
    "pbbfmm_set_timing": ([_vp, ctypes.c_int], ctypes.c_int),
    "pbbfmm_get_phase_times": ([_vp, ctypes.POINTER(ctypes.c_float), ctypes.c_int, _ip,
                                ctypes.POINTER(ctypes.c_char_p)], ctypes.c_int),
    "pbbfmm_debug_copy": ([_vp, ctypes.c_int, ctypes.c_int, _dp, _i64, ctypes.POINTER(_i64)], ctypes.c_int),
    "pbbfmm_tree_get_weights": ([_vp, _dp, _dp, _dp, _ip], ctypes.c_int),
    "pbbfmm_last_error": ([], ctypes.c_char_p),
    "pbbfmm_version": ([], ctypes.c_char_p),
    "pbbfmm_launch_count": ([], ctypes.c_longlong),
    "pbbfmm_reset_kernel_times": ([_vp], ctypes.c_int),
    "pbbfmm_get_kernel_times": ([_vp, ctypes.POINTER(ctypes.c_float), _ip, ctypes.c_int, _ip,
                                 ctypes.POINTER(ctypes.c_char_p)], ctypes.c_int),
    "pbbfmm_bin_points_noalloc": ([_vp, _i64, ctypes.c_double, ctypes.c_int, _vp, _vp, _vp, _vp],
                                  ctypes.c_int),
    "pbbfmm_measure_fma_peak": ([ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
    "pbbfmm_debug_set_pipeline_wait_limit": ([ctypes.c_int, ctypes.c_longlong], ctypes.c_int),
}


def lib():
    """Load the library once; raise loudly if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                "libpbbfmm3d_b200.so not built (run `python -c 'import __graft_entry__ as g; g.build()'`"
                " or `make -C pbbfmm3d_b200/csrc`)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in EXPORTS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def check(code: int) -> None:
    if code != OK:
        raise FMMError(code, lib().pbbfmm_last_error().decode(errors="replace"))
