"""CPU oracle for the XBFS hot path — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
legs may import this package. The product (xbfs_b200, libxbfs.so) never
does: it has no CPU fallback.

What is here (oracle.c):
  bfs_sweep  the reference's serial CPU BFS restated (bfs_gpu_update.cu:105-127)
  bfs_queue  serial FIFO BFS (ground truth at every scale)
  bfs_do     OpenMP direction-optimising BFS (multi-core CPU baseline)
  check_tree parent-tree check (level[parent] = level - 1, edge exists)
  reference_schedule  the reference's per-level direction switch
             (bfs_adaptiveFQ_wb_async.cuh:946-1078, 1114) replayed from levels

Input preparation of the oracle side (gen.c): gen_rmat, gen_grid and
pick_sources build the same seeded graphs and sources as the library's
generators with code of their own, so bench.py's reference arm needs no
product library and the tests can compare the two builds.

Parity pins: tests/golden/ holds level arrays produced by the reference's own
GPU path (oracle/_ref/xbfs_ref_harness, built from the reference sources by
oracle/Makefile and run on a B200; script: tests/golden/make_golden.py).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
REF_DIR = os.path.join(_HERE, "_ref")
REF_HARNESS = os.path.join(REF_DIR, "xbfs_ref_harness")


def build() -> str:
    srcs = [os.path.join(_HERE, f) for f in ("oracle.c", "gen.c")]
    if not os.path.exists(_LIB) or any(os.path.getmtime(_LIB) < os.path.getmtime(f) for f in srcs):
        subprocess.run(["make", "-s", "-C", _HERE, "all"], check=True)
    return _LIB


def _load():
    build()
    lib = C.CDLL(_LIB)
    p = C.c_void_p
    lib.oracle_bfs_queue.restype = C.c_int32
    lib.oracle_bfs_queue.argtypes = [p, p, C.c_int64, C.c_int32, p]
    lib.oracle_bfs_sweep.restype = C.c_int32
    lib.oracle_bfs_sweep.argtypes = [p, p, C.c_int64, C.c_int32, p, C.c_int32]
    lib.oracle_bfs_do.restype = C.c_int32
    lib.oracle_bfs_do.argtypes = [p, p, C.c_int64, C.c_int32, p, C.c_int32, C.c_double, C.c_double]
    lib.oracle_check_tree.restype = C.c_int64
    lib.oracle_check_tree.argtypes = [p, p, C.c_int64, C.c_int32, p, p]
    lib.oracle_edges_mc.restype = C.c_int64
    lib.oracle_edges_mc.argtypes = [p, C.c_int64, p]
    pp = C.POINTER(C.c_void_p)
    lib.oracle_gen_rmat.restype = C.c_int32
    lib.oracle_gen_rmat.argtypes = [C.c_int32, C.c_int32, C.c_uint64, C.c_double, C.c_double, C.c_double,
                                    pp, pp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    lib.oracle_gen_grid.restype = C.c_int32
    lib.oracle_gen_grid.argtypes = [C.c_int32, C.c_int32, pp, pp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    lib.oracle_pick_sources.restype = C.c_int32
    lib.oracle_pick_sources.argtypes = [p, C.c_int64, C.c_int32, C.c_uint64, p]
    lib.oracle_sort_adjacency_degree.restype = C.c_int32
    lib.oracle_sort_adjacency_degree.argtypes = [p, p, C.c_int64]
    lib.oracle_free.restype = None
    lib.oracle_free.argtypes = [C.c_void_p]
    return lib


_lib = _load()


def _arrs(beg, csr):
    beg = np.ascontiguousarray(beg, dtype=np.int64)
    csr = np.ascontiguousarray(csr, dtype=np.int32)
    if csr.size == 0:
        csr = np.zeros(1, dtype=np.int32)
    return beg, csr


def bfs_queue(beg, csr, src: int) -> np.ndarray:
    beg, csr = _arrs(beg, csr)
    out = np.empty(len(beg) - 1, dtype=np.int32)
    _lib.oracle_bfs_queue(beg.ctypes.data, csr.ctypes.data, len(beg) - 1, int(src), out.ctypes.data)
    return out


def bfs_sweep(beg, csr, src: int, threads: int = 1) -> tuple[np.ndarray, int]:
    """Returns (status, k) exactly as the reference's loop leaves them."""
    beg, csr = _arrs(beg, csr)
    out = np.empty(len(beg) - 1, dtype=np.int32)
    k = _lib.oracle_bfs_sweep(beg.ctypes.data, csr.ctypes.data, len(beg) - 1, int(src), out.ctypes.data,
                              int(threads))
    return out, int(k)


def bfs_do(beg, csr, src: int, threads: int = 0, alpha: float = 14.0, beta: float = 24.0) -> np.ndarray:
    beg, csr = _arrs(beg, csr)
    out = np.empty(len(beg) - 1, dtype=np.int32)
    _lib.oracle_bfs_do(beg.ctypes.data, csr.ctypes.data, len(beg) - 1, int(src), out.ctypes.data,
                       int(threads), alpha, beta)
    return out


def check_tree(beg, csr, src: int, levels, parents) -> int:
    """0 if parents form a BFS tree consistent with levels, else 1 + first bad vertex."""
    beg, csr = _arrs(beg, csr)
    lv = np.ascontiguousarray(levels, dtype=np.int32)
    pa = np.ascontiguousarray(parents, dtype=np.int32)
    return int(_lib.oracle_check_tree(beg.ctypes.data, csr.ctypes.data, len(beg) - 1, int(src),
                                      lv.ctypes.data, pa.ctypes.data))


def edges_mc(beg, levels) -> int:
    beg = np.ascontiguousarray(beg, dtype=np.int64)
    lv = np.ascontiguousarray(levels, dtype=np.int32)
    return int(_lib.oracle_edges_mc(beg.ctypes.data, len(beg) - 1, lv.ctypes.data))


def reference_schedule(beg, levels, alpha: float = 0.1) -> list[int]:
    """The reference's per-level choice (0 = scan-free / last-phase top-down,
    1 = second-phase single-scan top-down, -1 = bottom-up) for a traversal
    whose final levels are known: count[L] is the degree sum of level-L
    vertices (bfs_adaptiveFQ_wb_async.cuh:1042-1046), then cuh:1047-1078,
    1114. One entry per level the reference's loop runs (levels 0..depth-2).
    """
    beg = np.asarray(beg, dtype=np.int64)
    lv = np.asarray(levels)
    deg = np.diff(beg)
    depth = int(lv.max()) + 1 if lv.size else 0
    cnt = np.zeros(depth + 1, dtype=np.int64)
    m = lv >= 0
    np.add.at(cnt, lv[m], deg[m])
    E = int(beg[-1])
    INF = 10000
    is_change, td_adaptive, hub_before, hub_after, tag_prev = False, INF, 0, 0, 0
    tags = []
    for L in range(max(depth - 1, 0)):
        c = int(cnt[L])
        cp = int(cnt[L - 1]) if L > 0 else 0
        if not is_change:
            if L == 0 and c >= INF:
                is_change, td_adaptive = True, 1
            elif L > 0 and cp >= INF and c >= INF * 10 and c // cp >= 8:
                is_change, td_adaptive = True, L
            elif (L > 0 and c >= INF * 100) or (L > 0 and 0 < cp < INF and c >= INF * 10 and c // cp >= 1000):
                is_change, td_adaptive = True, L
        ratio = np.float32(c) / np.float32(E if E > 0 else 1)
        a = np.float32(alpha)
        if ratio >= a and tag_prev >= 0:
            hub_before = L
        if ratio < a and tag_prev == -1:
            hub_after = L
        if ratio < a:
            if hub_before == 0 and L < td_adaptive:
                tag = 0
            elif hub_after > 0 and L > hub_after:
                tag = 0
            else:
                tag = 1
        else:
            tag = -1
        tags.append(tag)
        tag_prev = tag
    return tags


def _take(pb, pc, V, E) -> tuple[np.ndarray, np.ndarray]:
    beg = np.ctypeslib.as_array(C.cast(pb, C.POINTER(C.c_int64)), shape=(V.value + 1,)).copy()
    csr = np.ctypeslib.as_array(C.cast(pc, C.POINTER(C.c_int32)), shape=(max(E.value, 1),))[: E.value].copy()
    _lib.oracle_free(pb)
    _lib.oracle_free(pc)
    return beg, csr


def gen_rmat(scale: int, edge_factor: int, seed: int = 1, a: float = 0.57, b: float = 0.19,
             c: float = 0.19) -> tuple[np.ndarray, np.ndarray]:
    """Seeded Graph500 R-MAT CSR (symmetric, deduplicated, no self-loops)."""
    pb, pc, V, E = C.c_void_p(), C.c_void_p(), C.c_int64(), C.c_int64()
    rc = _lib.oracle_gen_rmat(scale, edge_factor, seed, a, b, c, C.byref(pb), C.byref(pc), C.byref(V), C.byref(E))
    if rc != 0:
        raise MemoryError(f"oracle_gen_rmat failed ({rc})") if rc == -2 else ValueError("bad R-MAT arguments")
    return _take(pb, pc, V, E)


def gen_grid(width: int, height: int) -> tuple[np.ndarray, np.ndarray]:
    """2D 4-neighbour grid CSR, vertex r * width + c."""
    pb, pc, V, E = C.c_void_p(), C.c_void_p(), C.c_int64(), C.c_int64()
    rc = _lib.oracle_gen_grid(width, height, C.byref(pb), C.byref(pc), C.byref(V), C.byref(E))
    if rc != 0:
        raise MemoryError(f"oracle_gen_grid failed ({rc})") if rc == -2 else ValueError("bad grid arguments")
    return _take(pb, pc, V, E)


def pick_sources(beg, k: int, seed: int = 1) -> np.ndarray:
    """k seeded sources, uniform over vertices with degree > 0."""
    beg = np.ascontiguousarray(beg, dtype=np.int64)
    out = np.empty(max(k, 1), dtype=np.int32)
    if _lib.oracle_pick_sources(beg.ctypes.data, len(beg) - 1, k, seed, out.ctypes.data) != 0:
        raise ValueError("graph has no edges")
    return out[:k]


def sort_adjacency_degree(beg, csr) -> np.ndarray:
    """The CSR's neighbour lists reordered by descending neighbour degree
    (ties by ascending id); returns a new csr array."""
    beg = np.ascontiguousarray(beg, dtype=np.int64)
    out = np.array(csr, dtype=np.int32, copy=True)
    if _lib.oracle_sort_adjacency_degree(beg.ctypes.data, out.ctypes.data, len(beg) - 1) != 0:
        raise MemoryError("oracle_sort_adjacency_degree failed")
    return out
