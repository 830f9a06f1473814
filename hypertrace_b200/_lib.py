"""ctypes binding of libhtcuda.so (the C ABI declared in include/htcuda.h).

The library is built in-tree by ``__graft_entry__.build()`` (or ``python -m
hypertrace_b200.build``). There is no fallback: if the shared library is missing every
render entry point raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhtcuda.so")

HTC_OK = 0
HTC_ERR_INVALID = -1
HTC_ERR_CUDA = -2
HTC_ERR_SCENE = -3
HTC_ERR_UNSUPPORTED = -4

HTC_RECIPE_HY = 1
HTC_RECIPE_EU = 2
HTC_RECIPE_HY_TILED = 3
HTC_RECIPE_EU_GRADIENT = 4
HTC_RECIPE_CUSTOM = 100
HTC_ERR_BUDGET = -5
HTC_FLAG_JITTER_YX = 1
HTC_FLAG_NO_SORT = 2

STAT_SAMPLES, STAT_HOPS, STAT_OBJECT_TESTS, STAT_HITS = 0, 1, 2, 3

# Every symbol include/htcuda.h declares: (name, restype, argtypes).
_vp = ctypes.c_void_p
_u32 = ctypes.c_uint32
_sz = ctypes.c_size_t
_i = ctypes.c_int
_f = ctypes.c_float
SIGNATURES = [
    ("htc_last_error", ctypes.c_char_p, []),
    ("htc_version", _i, []),
    ("htc_device_count", _i, [ctypes.POINTER(_i)]),
    ("htc_set_device", _i, [_i]),
    ("htc_program_create", _i, [_i, _u32, _i, _i, _u32, ctypes.POINTER(_vp)]),
    ("htc_program_destroy", None, [_vp]),
    ("htc_program_build", _i, [ctypes.c_char_p, _u32, _i, _u32, ctypes.c_char_p, _sz, ctypes.POINTER(_vp)]),
    ("htc_program_static_size", _i, [_vp, ctypes.POINTER(ctypes.c_uint64)]),
    ("htc_program_check", _i, [_vp, _vp]),
    ("htc_malloc", _i, [ctypes.POINTER(_vp), _sz]),
    ("htc_free", _i, [_vp]),
    ("htc_memcpy_htod", _i, [_vp, _vp, _sz, _vp]),
    ("htc_memcpy_dtoh", _i, [_vp, _vp, _sz, _vp]),
    ("htc_memset", _i, [_vp, _i, _sz, _vp]),
    ("htc_stream_sync", _i, [_vp]),
    ("htc_render", _i, [_vp, _u32, _u32, _vp, _sz, _vp, _vp, _vp]),
    ("htc_render_ex", _i, [_vp, _u32, _u32, _vp, _sz, _vp, _vp, _vp, _vp]),
    ("htc_render_passes", _i, [_vp, _u32, _u32, _vp, _sz, _vp, _vp, _u32, _vp, _vp]),
    ("htc_render_wavefront", _i, [_vp, _u32, _u32, _vp, _sz, _vp, _vp, _u32, _vp, _vp]),
    ("htc_render_passes_noalloc", _i, [_i, _u32, _i, _u32, _u32, _u32, _vp, _sz, _vp, _vp, _u32, _vp, _vp, _vp]),
    ("htc_extract", _i, [_u32, _u32, _u32, _vp, _vp, _vp]),
    ("htc_gamma", _i, [_u32, _u32, _f, _vp, _vp, _vp]),
    ("htc_pack", _i, [_u32, _u32, _vp, _vp, _vp]),
    ("htc_extract_gamma_pack", _i, [_u32, _u32, _u32, _f, _vp, _vp, _vp]),
    ("htc_fill_seeds", _i, [_vp, _u32, _u32, _u32, _vp]),
    ("htc_fp32_probe", _i, [_vp, _u32, _i, ctypes.POINTER(ctypes.c_double), _vp]),
    ("htc_batch_create", _i, [_u32, ctypes.POINTER(_vp)]),
    ("htc_batch_destroy", None, [_vp]),
    ("htc_batch_set_views", _i, [_vp, _vp, _u32, _u32, _u32, _vp]),
    ("htc_batch_render", _i, [_vp, _vp, _vp]),
    ("htc_batch_graph_launch", _i, [_vp, _vp, _vp]),
    ("htc_batch_check", _i, [_vp, _vp]),
    ("htc_batch_reserve", _i, [_vp, ctypes.c_uint64, _u32, _vp]),
    ("htc_serve_plan", _i, [_vp, _u32, ctypes.c_uint64, _vp]),
    ("htc_server_create", _i, [ctypes.c_uint64, ctypes.c_uint64, _u32, ctypes.POINTER(_vp)]),
    ("htc_server_destroy", None, [_vp]),
    ("htc_server_configure", _i, [_vp, _u32, _u32, _u32, ctypes.c_uint64, _vp]),
    ("htc_server_submit", _i, [_vp, _vp, ctypes.POINTER(ctypes.c_uint64)]),
    ("htc_server_step", _i, [_vp, _vp, ctypes.POINTER(_u32)]),
    ("htc_server_poll", _i, [_vp, _vp, _u32, ctypes.POINTER(_u32), _i]),
    ("htc_server_stats", _i, [_vp, _vp]),
]


class HtcView(ctypes.Structure):
    """struct htc_view (include/htcuda.h)."""
    _fields_ = [("scene", ctypes.c_void_p), ("scene_size", ctypes.c_uint64), ("canvas", ctypes.c_void_p),
                ("seeds", ctypes.c_void_p), ("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
                ("recipe", ctypes.c_int32), ("light_hops", ctypes.c_uint32), ("flags", ctypes.c_uint32),
                ("address_width", ctypes.c_int32), ("passes", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class HtcRequest(ctypes.Structure):
    """struct htc_request (include/htcuda.h)."""
    _fields_ = [("scene", ctypes.c_void_p), ("scene_size", ctypes.c_uint64), ("width", ctypes.c_uint32),
                ("height", ctypes.c_uint32), ("recipe", ctypes.c_int32), ("light_hops", ctypes.c_uint32),
                ("flags", ctypes.c_uint32), ("address_width", ctypes.c_int32), ("passes", ctypes.c_uint32),
                ("global_seed", ctypes.c_uint32), ("priority", ctypes.c_uint32), ("quantum", ctypes.c_uint32),
                ("gamma", ctypes.c_float), ("reserved", ctypes.c_uint32), ("out_rgba8", ctypes.c_void_p),
                ("out_canvas", ctypes.c_void_p), ("out_seeds", ctypes.c_void_p)]


class HtcPlanItem(ctypes.Structure):
    """struct htc_plan_item (include/htcuda.h)."""
    _fields_ = [("pixels", ctypes.c_uint64), ("remaining", ctypes.c_uint32), ("quantum", ctypes.c_uint32),
                ("priority", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class HtcServerInfo(ctypes.Structure):
    """struct htc_server_info (include/htcuda.h)."""
    _fields_ = [("waiting", ctypes.c_uint32), ("active", ctypes.c_uint32), ("in_flight", ctypes.c_uint32),
                ("finished", ctypes.c_uint32), ("used_bytes", ctypes.c_uint64), ("budget_bytes", ctypes.c_uint64),
                ("steps", ctypes.c_uint64)]


HTC_PRIORITY_INTERACTIVE = 0
HTC_PRIORITY_BATCH = 1


class HtcError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"htcuda error {code}: {message}")
        self.code = code


_lib = None


def lib() -> ctypes.CDLL:
    """Load libhtcuda.so (once). Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: the CUDA path is not built "
                               "(run __graft_entry__.build()); there is no CPU fallback")
        l = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def check(rc: int) -> None:
    if rc != HTC_OK:
        msg = lib().htc_last_error()
        raise HtcError(rc, msg.decode() if msg else "")


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))
