"""ctypes binding of librd_b200.so (the C ABI declared in include/rd_c_api.h).

The library is built in-tree by ``make -C ridgedetection_b200/csrc`` (or
``__graft_entry__.build()``).  There is no fallback: if the shared object is
missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librd_b200.so")

RD_OK = 0
RD_ERR_ARG = 1
RD_ERR_CUDA = 2
RD_ERR_CAPACITY = 3
RD_ERR_NOT_CONVERGED = 4
RD_ERR_ALLOC = 5
RD_ERR_UNSUPPORTED = 6

RD_ROW_MAJOR = 0
RD_COL_MAJOR = 1
RD_LOOP_GRAPH = 0
RD_LOOP_HOST = 1

_STATUS_NAMES = {0: "RD_OK", 1: "RD_ERR_ARG", 2: "RD_ERR_CUDA", 3: "RD_ERR_CAPACITY",
                 4: "RD_ERR_NOT_CONVERGED", 5: "RD_ERR_ALLOC", 6: "RD_ERR_UNSUPPORTED"}


class RDError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{_STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class RunStats(ctypes.Structure):
    _fields_ = [("loop_iters", ctypes.c_int64), ("evolve_passes", ctypes.c_int64),
                ("max_passes", ctypes.c_int64), ("pairs", ctypes.c_double),
                ("err_bits", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("assign_ms", ctypes.c_double), ("assign_launches", ctypes.c_int64),
                ("point_passes", ctypes.c_double), ("dec_passes", ctypes.c_int64),
                ("dec_rounds", ctypes.c_int64)]


class CloudDesc(ctypes.Structure):
    _fields_ = [("offset", ctypes.c_int64), ("n", ctypes.c_int64), ("dim", ctypes.c_int32),
                ("r1", ctypes.c_float), ("r2", ctypes.c_float), ("pad", ctypes.c_int32)]


_vp = ctypes.c_void_p
_i = ctypes.c_int
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_f = ctypes.c_float
_pi64 = ctypes.POINTER(ctypes.c_int64)
_pf = ctypes.POINTER(ctypes.c_float)

# name -> argtypes (restype is rd_status = int unless listed in _RESTYPE)
SIGNATURES = {
    "rd_last_error": [],
    "rd_abi_version": [],
    "rd_supported_dims": [],
    "rd_probe_fp32_peak": [ctypes.POINTER(ctypes.c_double), _vp],
    "rd_tune_set": [ctypes.c_int, ctypes.c_int64, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                    ctypes.c_int],
    "rd_tune_get": [ctypes.c_int, ctypes.c_int64, ctypes.c_float, ctypes.POINTER(ctypes.c_int),
                    ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)],
    "rd_tune_reset": [],
    "rd_set_assign_cull": [ctypes.c_int],
    "rd_get_assign_cull": [ctypes.POINTER(ctypes.c_int)],
    "rd_set_tile_clusters": [ctypes.c_int, ctypes.c_int64, ctypes.c_int64],
    "rd_get_tile_clusters": [ctypes.POINTER(ctypes.c_int), _pi64, _pi64],
    "rd_autotune": [ctypes.c_int, _vp, ctypes.c_int64, ctypes.c_int64, ctypes.c_float, ctypes.c_int,
                    ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                    ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), _vp],
    "rd_hausdorff": [_i, _vp, _i64, _vp, _i64, _pf, _vp],
    "rd_distance_stats": [_i, _vp, _i64, _vp, _i64, _pf, _pf, _pf, _pf, _vp],
    "rd_segment_hausdorff": [_i, _vp, _i64, _pf, _vp],
    "rd_order_chains": [_i, _vp, _i64, _f, _vp, _vp, _pi64, _vp],
    "rd_text_cloud_shape": [ctypes.c_char_p, _pi64, ctypes.POINTER(ctypes.c_int)],
    "rd_load_text_cloud": [ctypes.c_char_p, _vp, _i64, _i],
    "rd_load_binary_cloud": [ctypes.c_char_p, _i64, _i, _vp],
    "rd_save_binary_cloud": [ctypes.c_char_p, _vp, _i64, _i],
    "rd_autotune_solve": [ctypes.c_int, _vp, ctypes.c_int64, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                          _vp, _vp, _vp, _vp, _vp],
    "rd_ordered_sum": [ctypes.c_int, _vp, _vp, ctypes.c_int64, _vp, ctypes.c_int, _vp],
    "rd_bf_create": [ctypes.POINTER(_vp), _i, _i, _i, _i64, _f, _f],
    "rd_bf_set_points": [_vp, _vp, _i64, _i, _vp],
    "rd_bf_set_loop_mode": [_vp, _i],
    "rd_bf_run": [_vp, _vp],
    "rd_bf_get_count": [_vp, _pi64],
    "rd_bf_get_points": [_vp, _vp, _i64, _i, _vp],
    "rd_bf_get_stats": [_vp, ctypes.POINTER(RunStats)],
    "rd_bf_set_profiling": [_vp, _i],
    "rd_bf_destroy": [_vp],
    "rd_tiled_create": [ctypes.POINTER(_vp), _i, _i, _i, _i64],
    "rd_tiled_set_points": [_vp, _vp, _i64, _i, _vp],
    "rd_tiled_set_loop_mode": [_vp, _i],
    "rd_tiled_set_policy": [_vp, _i],
    "rd_tiled_run": [_vp, _f, _f, _i64, ctypes.POINTER(ctypes.c_int32), _i, _vp],
    "rd_tiled_get_count": [_vp, _pi64],
    "rd_tiled_get_points": [_vp, _vp, _i64, _i, _vp],
    "rd_tiled_get_timers": [_vp, _pf, _pf, _pf, _pf],
    "rd_tiled_get_stats": [_vp, ctypes.POINTER(RunStats)],
    "rd_tiled_set_profiling": [_vp, _i],
    "rd_tiled_get_leaf_count": [_vp, _pi64],
    "rd_tiled_destroy": [_vp],
    "rd_choose": [_i, _vp, _i64, _f, _vp, _pi64, _vp],
    "rd_evolve": [_i, _vp, _i64, _vp, _i64, _f, _pi64, _vp],
    "rd_decimate": [_i, _vp, _i64, _f, _pi64, _vp],
    "rd_evolve_pass": [_i, _vp, _i64, _vp, _i64, _f, ctypes.POINTER(ctypes.c_int32), _vp],
    "rd_choose_ws": [_i, _vp, _i64, _i, _i64, _f, _vp, _i, _i64, _pi64, _vp,
                     ctypes.POINTER(ctypes.c_size_t), _vp],
    "rd_evolve_ws": [_i, _vp, _i64, _i, _i64, _vp, _i64, _i, _i64, _vp, _i64, _i, _i64, _f, _i64,
                     _pi64, ctypes.POINTER(ctypes.c_int32), _vp, ctypes.POINTER(ctypes.c_size_t),
                     _vp],
    "rd_decimate_ws": [_i, _vp, _i64, _i, _i64, _f, _pi64, _vp, ctypes.POINTER(ctypes.c_size_t),
                       _vp],
    "rd_decimate_noalloc": [_i, _vp, _i64, _f, _vp, _vp],
    "rd_evolve_adjoint": [_i, _vp, _i64, _vp, _i64, _f, _i, _i, _vp, _vp, _vp, _vp, _i, _vp],
    "rd_batch_create": [ctypes.POINTER(_vp)],
    "rd_batch_set_loop_mode": [_vp, _i],
    "rd_batch_run": [_vp, ctypes.POINTER(CloudDesc), _i32, _vp, _i64, _i, _vp],
    "rd_batch_get_counts": [_vp, _pi64],
    "rd_batch_get_points": [_vp, _i32, _vp, _i, _vp],
    "rd_batch_get_stats": [_vp, ctypes.POINTER(RunStats)],
    "rd_batch_destroy": [_vp],
}
_RESTYPE = {"rd_last_error": ctypes.c_char_p}

_lib = None


def lib():
    """Load librd_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} not found: build it with `make -C ridgedetection_b200/csrc` "
                "(the CUDA path has no fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, argtypes in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = argtypes
            fn.restype = _RESTYPE.get(name, ctypes.c_int)
        _lib = L
    return _lib


def check(status: int):
    if status != RD_OK:
        raise RDError(status, lib().rd_last_error().decode(errors="replace"))
    return status
