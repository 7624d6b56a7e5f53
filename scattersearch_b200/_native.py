"""ctypes binding of libscattersearch_b200.so (the C ABI in include/scattersearch.h).

The binding fails loudly: importing a search entry point without the built
library raises, and there is no CPU fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libscattersearch_b200.so")

SS_OK = 0
STATUS_NAMES = {
    0: "SS_OK", 1: "SS_ERR_INVALID_ARGUMENT", 2: "SS_ERR_IO", 3: "SS_ERR_FORMAT",
    4: "SS_ERR_NO_GRAPH", 5: "SS_ERR_CUDA", 6: "SS_ERR_OUT_OF_MEMORY", 7: "SS_ERR_UNSUPPORTED",
    8: "SS_ERR_SEARCH_LIMIT", 9: "SS_ERR_BUSY", 10: "SS_ERR_TIMEOUT",
}
SS_MAX_L = 4096
SS_MAX_DEGREE = 128
SS_MAX_INTRA_WIDTH = 16
SS_SCATTER_MAX_WARPS = 16
SS_NOALLOC_MAX_QUERIES = 65536
SS_NOALLOC_SCRATCH_BYTES = 256 + 4 * SS_NOALLOC_MAX_QUERIES

# Every function the header declares, with its ctypes signature.
_vp = ctypes.c_void_p
_u32 = ctypes.c_uint32
_i32 = ctypes.c_int
_f32p = ctypes.POINTER(ctypes.c_float)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_hp = ctypes.POINTER(ctypes.c_void_p)

SIGNATURES = {
    "ss_create": (_i32, [_u32, _u32, _f32p, _i32, _i32, _hp]),
    "ss_create_from_device": (_i32, [_u32, _u32, _vp, _i32, _i32, _hp]),
    "ss_destroy": (None, [_vp]),
    "ss_load_graph": (_i32, [_vp, ctypes.c_char_p]),
    "ss_set_graph": (_i32, [_vp, _u32p, _u32, _u32, _u32]),
    "ss_graph_info": (_i32, [_vp, _u32p, _u32p, _u32p, _u32p]),
    "ss_get_graph": (_i32, [_vp, _u32p, _u32]),
    "ss_search": (_i32, [_vp, _f32p, _i32, _i32, _u32p, _f32p]),
    "ss_search_batch": (_i32, [_vp, _f32p, _u32, _i32, _i32, _u32p, _f32p]),
    "ss_search_batch_uneven": (_i32, [_vp, _f32p, _u32, _i32p, _i32p, _u32p, _f32p]),
    "ss_search_batch_device": (_i32, [_vp, _vp, _u32, _vp, _vp, _vp, _i32, _i32, _i32, _vp, _vp,
                                      _vp, _vp, _vp]),
    "ss_batch_status": (_i32, [_vp, _u32p]),
    "ss_plan_create": (_i32, [_vp, _vp, _u32, _i32, _i32, _vp, _vp, _hp]),
    "ss_plan_create_uneven": (_i32, [_vp, _vp, _u32, _vp, _vp, _vp, _i32, _i32, _i32, _vp, _vp,
                                     _hp]),
    "ss_plan_launch": (_i32, [_vp, _vp]),
    "ss_plan_status": (_i32, [_vp, _u32p]),
    "ss_plan_destroy": (None, [_vp]),
    "ss_search_batch_noalloc": (_i32, [_vp, _vp, _u32, _i32, _i32, _vp, _vp, _vp]),
    "ss_search_intra": (_i32, [_vp, _f32p, _i32, _i32, _i32, _u32p, _f32p]),
    "ss_search_intra_batch": (_i32, [_vp, _f32p, _u32, _i32, _i32, _i32, _u32p, _f32p]),
    "ss_search_intra_batch_device": (_i32, [_vp, _vp, _u32, _i32, _i32, _i32, _vp, _vp, _vp, _vp,
                                            _vp]),
    "ss_set_tuning": (_i32, [_vp, _i32, _i32, _i32]),
    "ss_set_stage_layout": (_i32, [_vp, _i32, _i32]),
    "ss_set_row_copy": (_i32, [_vp, _i32]),
    "ss_set_visited_marks": (_i32, [_vp, _i32]),
    "ss_search_scatter_batch": (_i32, [_vp, _f32p, _u32, _i32, _i32, _i32, _i32, ctypes.c_uint64,
                                       _u32p, _f32p]),
    "ss_search_scatter_batch_stats": (_i32, [_vp, _f32p, _u32, _i32, _i32, _i32, _i32,
                                             ctypes.c_uint64, _u32p, _f32p, _u32p, _u32p, _u32p,
                                             _u32p]),
    "ss_search_scatter_batch_device": (_i32, [_vp, _vp, _u32, _i32, _i32, _i32, _i32,
                                              ctypes.c_uint64, _vp, _vp, _vp, _vp, _vp]),
    "ss_bruteforce": (_i32, [_vp, _f32p, _u32, _i32, _u32p, _f32p]),
    "ss_bruteforce_device": (_i32, [_vp, _vp, _u32, _i32, _vp, _vp, _vp]),
    "ss_server_create": (_i32, [_vp, _vp, _hp]),
    "ss_server_submit": (_i32, [_vp, _f32p, _i32, _i32, ctypes.POINTER(ctypes.c_uint64)]),
    "ss_server_wait": (_i32, [_vp, ctypes.c_uint64, _i32, _u32p, _f32p,
                              ctypes.POINTER(ctypes.c_double)]),
    "ss_server_replay": (_i32, [_vp, _f32p, _u32, _i32p, _i32p, ctypes.POINTER(ctypes.c_double),
                                _u32p, _f32p, ctypes.POINTER(ctypes.c_double)]),
    "ss_server_get_stats": (_i32, [_vp, _vp, _i32]),
    "ss_server_destroy": (None, [_vp]),
    "ss_load_fbin": (_i32, [ctypes.c_char_p, ctypes.POINTER(_f32p), _u32p, _u32p]),
    "ss_load_groundtruth": (_i32, [ctypes.c_char_p, ctypes.POINTER(_u32p), _u32p, _u32p]),
    "ss_free": (None, [_vp]),
    "ss_last_error": (ctypes.c_char_p, [_vp]),
    "ss_version": (ctypes.c_char_p, []),
}



class ServerConfig(ctypes.Structure):
    """ss_server_config (include/scattersearch.h)."""
    _fields_ = [("max_batch", ctypes.c_uint32), ("max_inflight", ctypes.c_uint32),
                ("max_pending", ctypes.c_uint32), ("K_max", ctypes.c_int32),
                ("L_max", ctypes.c_int32), ("memory_fraction", ctypes.c_float)]


class ServerStats(ctypes.Structure):
    """ss_server_stats (include/scattersearch.h)."""
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64),
                ("failed", ctypes.c_uint64), ("batches", ctypes.c_uint64),
                ("mean_batch", ctypes.c_double), ("p50_us", ctypes.c_double),
                ("p99_us", ctypes.c_double), ("p999_us", ctypes.c_double),
                ("max_us", ctypes.c_double), ("slots", ctypes.c_uint32)]


_lib = None


class SearchError(RuntimeError):
    """A C ABI call returned a nonzero ss_status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m scattersearch_b200.build` "
                "(there is no CPU fallback)")
        l = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def check(rc: int, handle=None) -> None:
    if rc != SS_OK:
        msg = lib().ss_last_error(handle)
        raise SearchError(rc, msg.decode() if msg else "")
