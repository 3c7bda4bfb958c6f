"""ctypes binding of libxbfs.so (the C ABI declared in include/xbfs.h).

The library is built in-tree (``python -m xbfs_b200.build``) and loaded from
this package directory. There is no fallback: if the shared library is
missing, importing the package raises, and every call that needs a GPU
returns XBFS_ERR_NO_DEVICE (raised as XbfsError) on a machine without one.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libxbfs.so")

XBFS_OK = 0
XBFS_ERR_INVALID_ARG = 1
XBFS_ERR_IO = 2
XBFS_ERR_FORMAT = 3
XBFS_ERR_CUDA = 4
XBFS_ERR_OOM = 5
XBFS_ERR_DEVICE_TIMEOUT = 6
XBFS_ERR_UNSUPPORTED = 7
XBFS_ERR_INTERNAL = 8
XBFS_ERR_NO_DEVICE = 9
XBFS_ERR_BUSY = 10
XBFS_ERR_LEVEL_OVERFLOW = 11

TD_QUEUE, TD_SCAN, BU = 0, 1, 2
STRATEGY_NAMES = {TD_QUEUE: "td_queue", TD_SCAN: "td_scan", BU: "bu"}
POLICY_HEURISTIC, POLICY_MLP, POLICY_FORCED, POLICY_BEAMER = 0, 1, 2, 3


class XbfsError(RuntimeError):
    def __init__(self, status: int, detail: str):
        super().__init__(f"xbfs error {status}: {detail}")
        self.status = status
        self.detail = detail


class Opts(C.Structure):
    _fields_ = [
        ("struct_size", C.c_int32),
        ("policy", C.c_int32),
        ("alpha", C.c_float),
        ("block_dim", C.c_int32),
        ("grid_dim", C.c_int32),
        ("async_bu", C.c_int32),
        ("small_max", C.c_int32),
        ("medium_max", C.c_int32),
        ("forced", C.POINTER(C.c_int8)),
        ("n_forced", C.c_int32),
        ("trace", C.c_int32),
        ("stream", C.c_void_p),
        ("padding", C.c_int32),
        ("beamer_alpha", C.c_float),
        ("beamer_beta", C.c_float),
        ("bu_probe", C.c_int32),
        ("wait_timeout_us", C.c_int32),
        ("test_absent_block", C.c_int32),
        ("reserved", C.c_int32),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("struct_size", C.c_int32),
        ("depth", C.c_int32),
        ("reached", C.c_int64),
        ("edges_mc", C.c_int64),
        ("device_ms", C.c_double),
        ("total_ms", C.c_double),
        ("n_td_queue", C.c_int32),
        ("n_td_scan", C.c_int32),
        ("n_bu", C.c_int32),
        ("n_async", C.c_int32),
        ("kernel_ms", C.c_double),
    ]


class LevelTrace(C.Structure):
    _fields_ = [
        ("level", C.c_int32),
        ("strategy", C.c_int32),
        ("n_f", C.c_int64),
        ("m_f", C.c_int64),
        ("n_u", C.c_int64),
        ("m_u", C.c_int64),
        ("us", C.c_double),
    ]


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA library first "
            "(python xbfs_b200/build.py, or __graft_entry__.build())")
    return C.CDLL(LIB_PATH)


lib = _load()


class ServeResult(C.Structure):
    _fields_ = [("struct_size", C.c_int32), ("state", C.c_int32), ("submit_us", C.c_double),
                ("admit_us", C.c_double), ("finish_us", C.c_double), ("edges_mc", C.c_int64),
                ("levels_dev", C.c_void_p)]

_p = C.c_void_p
_i32, _i64, _u64, _f32, _f64 = C.c_int32, C.c_int64, C.c_uint64, C.c_float, C.c_double
_PI64 = C.POINTER(C.c_int64)
_PI32 = C.POINTER(C.c_int32)
_PPI64 = C.POINTER(_PI64)
_PPI32 = C.POINTER(_PI32)

# name -> (restype, argtypes); every name here is also declared in include/xbfs.h
SIGNATURES = {
    "xbfs_strerror": (C.c_char_p, [_i32]),
    "xbfs_last_error": (C.c_char_p, []),
    "xbfs_version": (_i32, []),
    "xbfs_device_count": (_i32, [_PI32]),
    "xbfs_opts_init": (None, [C.POINTER(Opts)]),
    "xbfs_graph_load": (_i32, [C.c_char_p, C.c_char_p, _i32, C.POINTER(_p)]),
    "xbfs_graph_upload": (_i32, [_p, _p, _i64, _i64, _i32, C.POINTER(_p)]),
    "xbfs_graph_info": (_i32, [_p, _PI64, _PI64, _PI64, _PI64]),
    "xbfs_graph_download": (_i32, [_p, _p, _p]),
    "xbfs_graph_save": (_i32, [_p, C.c_char_p, C.c_char_p]),
    "xbfs_graph_free": (None, [_p]),
    "xbfs_bfs": (_i32, [_p, _i32, _p, _p, C.POINTER(Opts), C.POINTER(Stats)]),
    "xbfs_bfs_noalloc": (_i32, [_p, _i32, _p, _p, C.POINTER(Opts), C.POINTER(Stats)]),
    "xbfs_bfs_many": (_i32, [_p, _p, _i32, _p, C.POINTER(Opts), C.POINTER(Stats)]),
    "xbfs_graph_sort_adjacency": (_i32, [_p, _i32]),
    "xbfs_last_trace": (_i32, [_p, C.POINTER(LevelTrace), _i32, _PI32]),
    "xbfs_gen_rmat": (_i32, [_i32, _i32, _u64, _f64, _f64, _f64, _i32, C.POINTER(_p)]),
    "xbfs_gen_grid": (_i32, [_i32, _i32, _i32, C.POINTER(_p)]),
    "xbfs_gen_er": (_i32, [_i64, _f64, _u64, _i32, C.POINTER(_p)]),
    "xbfs_gen_rmat_host": (_i32, [_i32, _i32, _u64, _f64, _f64, _f64, _PPI64, _PPI32, _PI64, _PI64]),
    "xbfs_gen_grid_host": (_i32, [_i32, _i32, _PPI64, _PPI32, _PI64, _PI64]),
    "xbfs_gen_er_host": (_i32, [_i64, _f64, _u64, _PPI64, _PPI32, _PI64, _PI64]),
    "xbfs_free_host": (None, [_p]),
    "xbfs_convert_edge_list": (_i32, [C.c_char_p, _i32, _i32, _i32, _i32, _i32, C.c_char_p, _PI64, _PI64]),
    "xbfs_pick_sources": (_i32, [_p, _i64, _i32, _u64, _p]),
    "xbfs_bfs_batch": (_i32, [_p, _p, _i32, _p, C.POINTER(Opts), C.POINTER(Stats)]),
    "xbfs_bfs_batch_w": (_i32, [_p, _p, _i32, _p, C.POINTER(Opts), C.POINTER(Stats), _i32]),
    "xbfs_multi_create": (_i32, [C.POINTER(_p), _i32, _i32, C.POINTER(_p)]),
    "xbfs_multi_info": (_i32, [_p, _PI64, _PI64, _p]),
    "xbfs_multi_bfs": (_i32, [_p, _p, _p, C.POINTER(Opts), C.POINTER(Stats)]),
    "xbfs_multi_tune": (_i32, [_p, _p, _i32, _PI32, _PI32, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "xbfs_multi_set_config": (_i32, [_p, _i32, _i32, _f32]),
    "xbfs_multi_free": (None, [_p]),
    "xbfs_level_costs": (_i32, [_p, _i32, _i32, _i32, _p, C.POINTER(LevelTrace), _PI32]),
    "xbfs_serve_create": (_i32, [C.POINTER(_p), _i32, _i32, _i64, C.POINTER(_p)]),
    "xbfs_serve_run": (_i32, [_p, _i32, _p, _p, _p, _i32, _p, _p, _p, _p, C.POINTER(C.c_double)]),
    "xbfs_serve_start": (_i32, [_p]),
    "xbfs_serve_submit": (_i32, [_p, _i32, _i32, _i32, _p, _PI64]),
    "xbfs_serve_poll": (_i32, [_p, _i64, _i64, C.POINTER(ServeResult)]),
    "xbfs_serve_stop": (_i32, [_p]),
    "xbfs_serve_release": (_i32, [_p, _p, _i64]),
    "xbfs_serve_fetch": (_i32, [_p, _p, _i64, _p]),
    "xbfs_serve_free": (None, [_p]),
    "xbfs_part_create": (_i32, [_p, _p, _i64, _i64, _i64, _i32, _i32, C.POINTER(_p)]),
    "xbfs_part_free": (None, [_p]),
    "xbfs_part_reset": (_i32, [_p, _i32]),
    "xbfs_part_stats": (_i32, [_p, _p]),
    "xbfs_part_td_expand": (_i32, [_p, _p]),
    "xbfs_part_claim": (_i32, [_p, _p, _i32]),
    "xbfs_part_frontier_bits": (_i32, [_p, _p, _i64]),
    "xbfs_part_bottom_up": (_i32, [_p, _p, _i32]),
    "xbfs_part_levels": (_i32, [_p, _p]),
    "xbfs_mlp_num_params": (_i32, []),
    "xbfs_mlp_set_weights": (_i32, [_i32, _p, _i32]),
    "xbfs_mlp_logits": (_i32, [_i32, _p, _p, _i32, _p]),
    "xbfs_mlp_grad": (_i32, [_i32, _p, _p, _p, _i32, _p, _p]),
    "xbfs_mlp_train": (_i32, [_i32, _p, _p, _p, _i32, _i32, _f32, _f32, _p]),
}

for _name, (_res, _args) in SIGNATURES.items():
    _fn = getattr(lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args


def check(status: int) -> None:
    if status != XBFS_OK:
        detail = lib.xbfs_last_error().decode(errors="replace")
        raise XbfsError(status, f"{lib.xbfs_strerror(status).decode()}: {detail}")


def device_count() -> int:
    n = C.c_int32(0)
    check(lib.xbfs_device_count(C.byref(n)))
    return n.value
