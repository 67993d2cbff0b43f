"""ctypes binding of libsmx.so (include/smx.h).

The library is built in-tree by ``make -C subgraphmatching_b200`` (called by
__graft_entry__.build()).  There is no fallback: if the library is missing the
import raises ImportError naming the build step.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libsmx.so")

SMX_OK = 0
SMX_EMPTY_CANDIDATES = 1
SMX_INVALID_ORDER = 2
SMX_TOO_LARGE = 3
SMX_TIMEOUT = 4
SMX_CUDA_ERROR = 5
SMX_BAD_ARGUMENT = 6
SMX_BAD_FORMAT = 7
SMX_IO_ERROR = 8
SMX_STOPPED = 9
SMX_NO_DEVICE = 10


class SmxError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"smx error {status}: {message}")
        self.status = status


class EnumOpts(ctypes.Structure):
    _fields_ = [
        ("explore", ctypes.c_int32),
        ("warps_per_block", ctypes.c_int32),
        ("blocks_per_sm", ctypes.c_int32),
        ("task_grab", ctypes.c_int32),
        ("stage_chunk", ctypes.c_int32),
        ("gallop_ratio", ctypes.c_int32),
        ("bitmap_min", ctypes.c_int32),
        ("use_tma", ctypes.c_int32),
        ("failing_sets", ctypes.c_int32),
        ("lane_depth", ctypes.c_int32),
        ("time_budget_ms", ctypes.c_double),
        ("budget_per_query", ctypes.c_int32),
        ("reserved0", ctypes.c_int32),
    ]


class StatsC(ctypes.Structure):
    _fields_ = [
        ("count", ctypes.c_uint64),
        ("raw_count", ctypes.c_uint64),
        ("intersections", ctypes.c_uint64),
        ("nodes", ctypes.c_uint64),
        ("bytes", ctypes.c_uint64),
        ("pruned", ctypes.c_uint64),
        ("tasks", ctypes.c_uint64),
        ("kernel_ms", ctypes.c_double),
        ("limit_reached", ctypes.c_int32),
        ("status", ctypes.c_int32),
    ]


_vp = ctypes.c_void_p
_pvp = ctypes.POINTER(ctypes.c_void_p)
_u32 = ctypes.c_uint32
_u64 = ctypes.c_uint64
_i32 = ctypes.c_int
_dbl = ctypes.c_double
_pu32 = ctypes.POINTER(ctypes.c_uint32)
_pu64 = ctypes.POINTER(ctypes.c_uint64)
_str = ctypes.c_char_p
_pf = ctypes.POINTER(ctypes.c_float)

# (name, restype, argtypes) for every entry point of include/smx.h
SIGNATURES = [
    ("smx_status_str", ctypes.c_char_p, [_i32]),
    ("smx_last_error", ctypes.c_char_p, []),
    ("smx_device_count", _i32, []),
    ("smx_mark_begin", _i32, [_vp]),
    ("smx_mark_end", _i32, [_vp, ctypes.POINTER(ctypes.c_double)]),
    ("smx_launch_count", _u64, []),
    ("smx_graph_create", _i32, [_pu64, _pu32, _pu32, _u32, _u64, _i32, _pvp]),
    ("smx_graph_load_text", _i32, [_str, _i32, _pvp]),
    ("smx_graph_generate", _i32, [_u32, _u64, _dbl, _u32, _dbl, _u64, _i32, _pvp]),
    ("smx_graph_info", _i32, [_vp, _pu32, _pu64, _pu32, _pu32]),
    ("smx_graph_export", _i32, [_vp, _pu64, _pu32, _pu32]),
    ("smx_graph_save_text", _i32, [_vp, _str]),
    ("smx_graph_destroy", None, [_vp]),
    ("smx_query_create", _i32, [_pu32, _pu32, _pu32, _u32, _pvp]),
    ("smx_query_load_text", _i32, [_str, _pvp]),
    ("smx_query_generate", _i32, [_vp, _u32, _i32, _u64, _pvp]),
    ("smx_query_info", _i32, [_vp, _pu32, _pu32, _pu32]),
    ("smx_query_export", _i32, [_vp, _pu32, _pu32, _pu32]),
    ("smx_query_kcore", _i32, [_vp, _pu32]),
    ("smx_query_save_text", _i32, [_vp, _str]),
    ("smx_query_destroy", None, [_vp]),
    ("smx_order_ri", _i32, [_vp, _pu32]),
    ("smx_order_gql", _i32, [_vp, _vp, _pu32]),
    ("smx_order_valid", _i32, [_vp, _pu32]),
    ("smx_filter", _i32, [_vp, _vp, _i32, _i32, _pvp]),
    ("smx_cand_counts", _i32, [_vp, _pu32]),
    ("smx_cand_export", _i32, [_vp, _u32, _pu32]),
    ("smx_table_info", _i32, [_vp, _u32, _u32, _pu32, _pu32, _pu32]),
    ("smx_table_export", _i32, [_vp, _u32, _u32, _pu32, _pu32, _pu32]),
    ("smx_cand_timing", _i32, [_vp, ctypes.POINTER(ctypes.c_double)]),
    ("smx_cand_destroy", None, [_vp]),
    ("smx_enum_opts_default", None, [ctypes.POINTER(EnumOpts)]),
    ("smx_enumerate", _i32, [_vp, _vp, _vp, _pu32, ctypes.POINTER(EnumOpts), _u64, _pu32, ctypes.POINTER(StatsC)]),
    ("smx_enumerate_noalloc", _i32, [_vp, _vp, _vp, _pu32, ctypes.POINTER(EnumOpts), _u64, _pu32,
                                     ctypes.POINTER(StatsC)]),
    ("smx_mlp_param_count", ctypes.c_size_t, []),
    ("smx_mlp_create", _i32, [_i32, _u32, _u64, _pvp]),
    ("smx_mlp_set_params", _i32, [_vp, _pf, ctypes.c_size_t]),
    ("smx_mlp_get_params", _i32, [_vp, _pf, ctypes.c_size_t]),
    ("smx_mlp_forward", _i32, [_vp, _pf, _u32, _pf]),
    ("smx_mlp_gradients", _i32, [_vp, _pf, _pf, _u32, _pf, _pf]),
    ("smx_mlp_train_step", _i32, [_vp, _pf, _pf, _u32, ctypes.c_float, _pf]),
    ("smx_mlp_destroy", None, [_vp]),
    ("smx_order_features", _i32, [_vp, _vp, _pu32, _pf]),
    ("smx_order_beam", _i32, [_vp, _vp, _u32, _u64, _pu32, _pu32]),
    ("smx_order_learned", _i32, [_vp, _vp, _vp, _u32, _u64, _pu32, _pf]),
    ("smx_stop_flag_create", _i32, [_i32, ctypes.POINTER(_pu32)]),
    ("smx_stop_flag_destroy", None, [_pu32]),
    ("smx_enumerate_batch", _i32, [_vp, _pvp, _pvp, ctypes.POINTER(_pu32), _u32, ctypes.POINTER(EnumOpts), _u64,
                                   _pu64, ctypes.POINTER(StatsC), ctypes.POINTER(ctypes.c_int32)]),
]


def load(path: str) -> ctypes.CDLL:
    """Open a library exporting include/smx.h and declare every signature."""
    handle = ctypes.CDLL(path)
    for name, res, args in SIGNATURES:
        f = getattr(handle, name)
        f.restype = res
        f.argtypes = args
    return handle


if not os.path.exists(LIB_PATH):
    raise ImportError(f"libsmx.so not built ({LIB_PATH}); run __graft_entry__.build() or make -C subgraphmatching_b200")

lib = load(LIB_PATH)


def last_error() -> str:
    m = lib.smx_last_error()
    return m.decode() if m else ""


def check(status: int) -> None:
    if status != SMX_OK:
        raise SmxError(status, f"{lib.smx_status_str(status).decode()}: {last_error()}")
