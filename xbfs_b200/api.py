"""Python host API over libxbfs.so.

Mirrors the reference's interface for the BFS path:

* the CSR file pair of graph.hpp:4-104 (``Graph.load``),
* the parameters of the reference's command line / BFS_ControlFlow
  (bfs_gpu_update.cu:33-48, bfs_adaptiveFQ_wb_async.cuh:934-935):
  ``alpha``, ``block_dim``, ``grid_dim``, ``padding``, source vertex,
* the per-vertex int32 level array (-1 = unreached) it produces
  (bfs_gpu_update.cu:213-218, 255).

Errors are raised as :class:`XbfsError` carrying the library status code.
Outputs are numpy arrays (host) or, when a CUDA tensor is passed, written in
place on the device.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import BU, TD_QUEUE, TD_SCAN, LevelTrace, Opts, Stats, XbfsError, check, lib

POLICIES = {"heuristic": _lib.POLICY_HEURISTIC, "mlp": _lib.POLICY_MLP,
            "forced": _lib.POLICY_FORCED, "beamer": _lib.POLICY_BEAMER}
STRATEGIES = {"td_queue": TD_QUEUE, "td_scan": TD_SCAN, "bu": BU}

RMAT_A, RMAT_B, RMAT_C = 0.57, 0.19, 0.19  # Graph500 Kronecker parameters


def _ptr(a) -> int:
    """Data pointer of a numpy array or torch tensor (host or device)."""
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a.data_ptr())


@dataclass
class BfsOptions:
    """Per-call options (xbfs_opts). ``policy``: heuristic | mlp | forced | beamer."""
    policy: str = "heuristic"
    alpha: float = 0.1
    block_dim: int = 0
    grid_dim: int = 0
    async_bu: bool = True
    small_max: int = 32
    medium_max: int = 256
    forced: Optional[Sequence[int]] = None
    trace: bool = False
    padding: int = 1
    beamer_alpha: float = 14.0
    beamer_beta: float = 24.0
    stream: int = 0
    bu_mode: int = 0   # bottom-up probe shape (xbfs_opts.bu_probe): 0 = by density (default), 5 = word-parallel, 6 = word-parallel over head records, 1-4 list-based
    wait_timeout_us: int = 0     # bound of device-side waits; 0 = 10 s
    test_absent_block: int = 0   # failure-detection test hook (xbfs_opts.test_absent_block)
    _keep: list = field(default_factory=list, repr=False)

    def to_c(self) -> Opts:
        o = Opts()
        lib.xbfs_opts_init(C.byref(o))
        o.policy = POLICIES[self.policy] if isinstance(self.policy, str) else int(self.policy)
        o.alpha = float(self.alpha)
        o.block_dim = int(self.block_dim)
        o.grid_dim = int(self.grid_dim)
        o.async_bu = 1 if self.async_bu else 0
        o.small_max = int(self.small_max)
        o.medium_max = int(self.medium_max)
        o.trace = 1 if self.trace else 0
        o.padding = int(self.padding)
        o.beamer_alpha = float(self.beamer_alpha)
        o.beamer_beta = float(self.beamer_beta)
        o.stream = self.stream or None
        o.bu_probe = int(self.bu_mode)
        o.wait_timeout_us = int(self.wait_timeout_us)
        o.test_absent_block = int(self.test_absent_block)
        if self.forced is not None:
            vals = [STRATEGIES[s] if isinstance(s, str) else int(s) for s in self.forced]
            arr = (C.c_int8 * max(1, len(vals)))(*vals)
            self._keep = [arr]
            o.forced = C.cast(arr, C.POINTER(C.c_int8))
            o.n_forced = len(vals)
        return o


@dataclass
class BfsResult:
    levels: object
    parents: object
    depth: int
    reached: int
    edges_mc: int
    device_ms: float
    total_ms: float
    kernel_ms: float
    strategies: dict
    n_async: int
    trace: Optional[list] = None

    @property
    def gteps(self) -> float:
        return self.edges_mc / (self.device_ms * 1e-3) / 1e9 if self.device_ms > 0 else 0.0


class Graph:
    """A CSR graph resident on one GPU (xbfs_graph handle)."""

    def __init__(self, handle: int, device: int):
        self._h = C.c_void_p(handle)
        self.device = device
        V, E, md, ni = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        check(lib.xbfs_graph_info(self._h, C.byref(V), C.byref(E), C.byref(md), C.byref(ni)))
        self.V, self.E, self.max_degree, self.n_isolated = V.value, E.value, md.value, ni.value

    # -- construction ------------------------------------------------------
    @classmethod
    def load(cls, beg_path: str, csr_path: str, device: int = 0) -> "Graph":
        h = C.c_void_p()
        check(lib.xbfs_graph_load(beg_path.encode(), csr_path.encode(), device, C.byref(h)))
        return cls(h.value, device)

    @classmethod
    def from_csr(cls, beg: np.ndarray, csr: np.ndarray, device: int = 0) -> "Graph":
        beg = np.ascontiguousarray(beg, dtype=np.int64)
        csr = np.ascontiguousarray(csr, dtype=np.int32)
        h = C.c_void_p()
        check(lib.xbfs_graph_upload(beg.ctypes.data, csr.ctypes.data if csr.size else None,
                                    len(beg) - 1, len(csr), device, C.byref(h)))
        return cls(h.value, device)

    @classmethod
    def rmat(cls, scale: int, edge_factor: int, seed: int = 1, a: float = RMAT_A, b: float = RMAT_B,
             c: float = RMAT_C, device: int = 0) -> "Graph":
        h = C.c_void_p()
        check(lib.xbfs_gen_rmat(scale, edge_factor, seed, a, b, c, device, C.byref(h)))
        return cls(h.value, device)

    @classmethod
    def grid(cls, width: int, height: int, device: int = 0) -> "Graph":
        h = C.c_void_p()
        check(lib.xbfs_gen_grid(width, height, device, C.byref(h)))
        return cls(h.value, device)

    @classmethod
    def er(cls, n: int, mean_degree: float = 8.0, seed: int = 1, device: int = 0) -> "Graph":
        h = C.c_void_p()
        check(lib.xbfs_gen_er(n, mean_degree, seed, device, C.byref(h)))
        return cls(h.value, device)

    # -- lifetime ------------------------------------------------------------
    def free(self) -> None:
        if self._h:
            lib.xbfs_graph_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.free()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # -- data ------------------------------------------------------------------
    def offsets(self) -> np.ndarray:
        beg = np.empty(self.V + 1, dtype=np.int64)
        check(lib.xbfs_graph_download(self._h, beg.ctypes.data, None))
        return beg

    def download(self) -> tuple[np.ndarray, np.ndarray]:
        beg = np.empty(self.V + 1, dtype=np.int64)
        csr = np.empty(max(self.E, 1), dtype=np.int32)
        check(lib.xbfs_graph_download(self._h, beg.ctypes.data, csr.ctypes.data))
        return beg, csr[: self.E]

    def save(self, beg_path: str, csr_path: str) -> None:
        check(lib.xbfs_graph_save(self._h, beg_path.encode(), csr_path.encode()))

    # -- traversal -------------------------------------------------------------
    def bfs(self, src: int, levels=None, parents=None, want_parents: bool = False,
            opts: Optional[BfsOptions] = None, **kw) -> BfsResult:
        """Single-source BFS. ``levels``/``parents`` may be preallocated numpy
        arrays or CUDA tensors of V int32; otherwise numpy arrays are returned."""
        if opts is None:
            opts = BfsOptions(**kw)
        elif kw:
            raise TypeError("pass either opts or keyword options")
        if levels is None:
            levels = np.empty(self.V, dtype=np.int32)
        if parents is None and want_parents:
            parents = np.empty(self.V, dtype=np.int32)
        o = opts.to_c()
        st = Stats()
        st.struct_size = C.sizeof(Stats)
        check(lib.xbfs_bfs(self._h, int(src), _ptr(levels), _ptr(parents) if parents is not None else None,
                           C.byref(o), C.byref(st)))
        trace = self.last_trace() if opts.trace else None
        return BfsResult(levels=levels, parents=parents, depth=st.depth, reached=st.reached,
                         edges_mc=st.edges_mc, device_ms=st.device_ms, total_ms=st.total_ms,
                         kernel_ms=st.kernel_ms,
                         strategies={"td_queue": st.n_td_queue, "td_scan": st.n_td_scan, "bu": st.n_bu},
                         n_async=st.n_async, trace=trace)

    def sort_adjacency(self, order: str = "degree") -> None:
        """Reorder neighbours within each CSR segment: "degree" (descending
        neighbour degree, fewer bottom-up probes) or "id" (ascending ids)."""
        check(lib.xbfs_graph_sort_adjacency(self._h, {"id": 0, "degree": 1}[order]))

    def bfs_many(self, srcs, levels=None, opts: Optional[BfsOptions] = None, **kw) -> BfsResult:
        """One single-source traversal per source, pipelined with the copies of
        their level arrays (xbfs_bfs_many): levels[i] belongs to srcs[i] (n x V
        int32, numpy or CUDA tensor)."""
        if opts is None:
            opts = BfsOptions(**kw)
        elif kw:
            raise TypeError("pass either opts or keyword options")
        srcs = np.ascontiguousarray(srcs, dtype=np.int32)
        n = len(srcs)
        if levels is None:
            levels = np.empty((n, self.V), dtype=np.int32)
        o = opts.to_c()
        st = Stats()
        st.struct_size = C.sizeof(Stats)
        check(lib.xbfs_bfs_many(self._h, srcs.ctypes.data, n, _ptr(levels), C.byref(o), C.byref(st)))
        return BfsResult(levels=levels, parents=None, depth=st.depth, reached=st.reached, edges_mc=st.edges_mc,
                         device_ms=st.device_ms, total_ms=st.total_ms, kernel_ms=st.kernel_ms,
                         strategies={"td_queue": st.n_td_queue, "td_scan": st.n_td_scan, "bu": st.n_bu},
                         n_async=st.n_async)

    def bfs_batch(self, srcs, levels=None, words_per_vertex: int = 0, direction: Optional[str] = None,
                  alpha: float = 0.0, stream: int = 0) -> BfsResult:
        """Multi-source BFS: levels[i] is the level array of srcs[i] (n x V int32,
        numpy or CUDA tensor). ``direction``: None (switch by alpha), "td", "bu"."""
        srcs = np.ascontiguousarray(srcs, dtype=np.int32)
        n = len(srcs)
        if levels is None:
            levels = np.empty((n, self.V), dtype=np.int32)
        opts = BfsOptions(alpha=alpha, stream=stream)
        if direction is not None:
            opts.policy = "forced"
            opts.forced = ["bu" if direction == "bu" else "td_queue"]
        o = opts.to_c()
        st = Stats()
        st.struct_size = C.sizeof(Stats)
        check(lib.xbfs_bfs_batch_w(self._h, srcs.ctypes.data, n, _ptr(levels), C.byref(o), C.byref(st),
                                   int(words_per_vertex)))
        return BfsResult(levels=levels, parents=None, depth=st.depth, reached=st.reached, edges_mc=st.edges_mc,
                         device_ms=st.device_ms, total_ms=st.total_ms, kernel_ms=st.kernel_ms,
                         strategies={"td_queue": st.n_td_queue, "td_scan": 0, "bu": st.n_bu}, n_async=0)

    def last_trace(self) -> list[dict]:
        n = C.c_int32(0)
        check(lib.xbfs_last_trace(self._h, None, 0, C.byref(n)))
        buf = (LevelTrace * max(1, n.value))()
        check(lib.xbfs_last_trace(self._h, buf, n.value, C.byref(n)))
        return [{"level": t.level, "strategy": _lib.STRATEGY_NAMES.get(t.strategy, t.strategy),
                 "n_f": t.n_f, "m_f": t.m_f, "n_u": t.n_u, "m_u": t.m_u, "us": t.us}
                for t in buf[: n.value]]


# ---------------------------------------------------------------------------
# Host-side generators (no GPU needed); identical output to the device ones.
# ---------------------------------------------------------------------------
def _take_host(pb, pc, V, E) -> tuple[np.ndarray, np.ndarray]:
    beg = np.ctypeslib.as_array(pb, shape=(V.value + 1,)).copy()
    csr = np.ctypeslib.as_array(pc, shape=(max(E.value, 1),))[: E.value].copy()
    lib.xbfs_free_host(C.cast(pb, C.c_void_p))
    lib.xbfs_free_host(C.cast(pc, C.c_void_p))
    return beg, csr


def gen_rmat_host(scale: int, edge_factor: int, seed: int = 1, a: float = RMAT_A, b: float = RMAT_B,
                  c: float = RMAT_C) -> tuple[np.ndarray, np.ndarray]:
    pb, pc = C.POINTER(C.c_int64)(), C.POINTER(C.c_int32)()
    V, E = C.c_int64(), C.c_int64()
    check(lib.xbfs_gen_rmat_host(scale, edge_factor, seed, a, b, c, C.byref(pb), C.byref(pc),
                                 C.byref(V), C.byref(E)))
    return _take_host(pb, pc, V, E)


def gen_grid_host(width: int, height: int) -> tuple[np.ndarray, np.ndarray]:
    pb, pc = C.POINTER(C.c_int64)(), C.POINTER(C.c_int32)()
    V, E = C.c_int64(), C.c_int64()
    check(lib.xbfs_gen_grid_host(width, height, C.byref(pb), C.byref(pc), C.byref(V), C.byref(E)))
    return _take_host(pb, pc, V, E)


def gen_er_host(n: int, mean_degree: float = 8.0, seed: int = 1) -> tuple[np.ndarray, np.ndarray]:
    pb, pc = C.POINTER(C.c_int64)(), C.POINTER(C.c_int32)()
    V, E = C.c_int64(), C.c_int64()
    check(lib.xbfs_gen_er_host(n, mean_degree, seed, C.byref(pb), C.byref(pc), C.byref(V), C.byref(E)))
    return _take_host(pb, pc, V, E)


def pick_sources(beg: np.ndarray, k: int, seed: int = 1) -> np.ndarray:
    beg = np.ascontiguousarray(beg, dtype=np.int64)
    out = np.empty(max(k, 1), dtype=np.int32)
    check(lib.xbfs_pick_sources(beg.ctypes.data, len(beg) - 1, k, seed, out.ctypes.data))
    return out[:k]


def convert_edge_list(text_path: str, out_prefix: str, reverse: bool = True, skip_lines: int = 0,
                      dedupe: bool = True, drop_self_loops: bool = True, weights: bool = False) -> tuple[int, int]:
    """Edge-list text -> CSR file pair (int64 offsets, int32 neighbours)."""
    V, E = C.c_int64(), C.c_int64()
    check(lib.xbfs_convert_edge_list(text_path.encode(), int(reverse), int(skip_lines), int(dedupe),
                                     int(drop_self_loops), int(weights), out_prefix.encode(), C.byref(V), C.byref(E)))
    return V.value, E.value


def write_csr(beg: np.ndarray, csr: np.ndarray, beg_path: str, csr_path: str) -> None:
    """Write the reference's file pair: raw int64 beg_pos, raw int32 csr."""
    np.ascontiguousarray(beg, dtype="<i8").tofile(beg_path)
    np.ascontiguousarray(csr, dtype="<i4").tofile(csr_path)


def read_csr(beg_path: str, csr_path: str) -> tuple[np.ndarray, np.ndarray]:
    beg = np.fromfile(beg_path, dtype="<i8")
    csr = np.fromfile(csr_path, dtype="<i4")
    return beg, csr[: int(beg[-1])]


class MultiGraph:
    """Many graphs on one device, one source each, one persistent launch
    (xbfs_multi_*). Levels come back concatenated; ``split`` cuts them."""

    def __init__(self, graphs: Sequence[Graph], device: int = 0):
        arr = (C.c_void_p * len(graphs))(*[g.handle.value for g in graphs])
        h = C.c_void_p()
        check(lib.xbfs_multi_create(arr, len(graphs), device, C.byref(h)))
        self._h = h
        self.graphs = list(graphs)  # keep the handles alive
        self.n = len(graphs)
        tv, te = C.c_int64(), C.c_int64()
        offs = np.empty(self.n, dtype=np.int64)
        check(lib.xbfs_multi_info(h, C.byref(tv), C.byref(te), offs.ctypes.data))
        self.total_V, self.total_E, self.offsets = tv.value, te.value, offs

    def bfs(self, srcs, levels=None) -> BfsResult:
        srcs = np.ascontiguousarray(srcs, dtype=np.int32)
        if levels is None:
            levels = np.empty(self.total_V, dtype=np.int32)
        st = Stats()
        st.struct_size = C.sizeof(Stats)
        check(lib.xbfs_multi_bfs(self._h, srcs.ctypes.data, _ptr(levels), None, C.byref(st)))
        return BfsResult(levels=levels, parents=None, depth=0, reached=0, edges_mc=st.edges_mc,
                         device_ms=st.device_ms, total_ms=st.total_ms, kernel_ms=st.kernel_ms,
                         strategies={}, n_async=0)

    def split(self, levels) -> list:
        return [levels[o:o + g.V] for o, g in zip(self.offsets, self.graphs)]

    def tune(self, srcs, reps: int = 2) -> dict:
        srcs = np.ascontiguousarray(srcs, dtype=np.int32)
        b, t, a, ms = C.c_int32(), C.c_int32(), C.c_float(), C.c_float()
        check(lib.xbfs_multi_tune(self._h, srcs.ctypes.data, reps, C.byref(b), C.byref(t), C.byref(a), C.byref(ms)))
        return {"block": b.value, "thread_max": t.value, "alpha": a.value, "best_ms": ms.value}

    def set_config(self, block: int, thread_max: int, alpha: float) -> None:
        check(lib.xbfs_multi_set_config(self._h, block, thread_max, alpha))

    def free(self) -> None:
        if self._h:
            lib.xbfs_multi_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Server:
    """Continuous-batching BFS server over device-resident graphs (xbfs_serve_*)."""

    def __init__(self, graphs: Sequence[Graph], device: int = 0, hbm_budget_bytes: int = 0):
        arr = (C.c_void_p * len(graphs))(*[g.handle.value for g in graphs])
        h = C.c_void_p()
        check(lib.xbfs_serve_create(arr, len(graphs), device, int(hbm_budget_bytes), C.byref(h)))
        self._h = h
        self.graphs = list(graphs)
        self._host = {}

    def run(self, graph_ids, srcs, arrival_us, keep_outputs: bool = False, to_host: bool = False) -> dict:
        """Replay a request trace. ``keep_outputs``: return device level arrays
        (``levels_dev``, read with fetch()); ``to_host``: each finished request's
        levels are copied to a host array (``levels``) and its device memory freed."""
        g = np.ascontiguousarray(graph_ids, dtype=np.int32)
        s = np.ascontiguousarray(srcs, dtype=np.int32)
        a = np.ascontiguousarray(arrival_us, dtype=np.float64)
        n = len(g)
        admit = np.zeros(n, dtype=np.float64)
        fin = np.zeros(n, dtype=np.float64)
        mc = np.zeros(n, dtype=np.int64)
        ptrs = (C.c_void_p * max(n, 1))()
        mode = 2 if to_host else (1 if keep_outputs else 0)
        host = []
        if to_host:
            host = [np.empty(self.graphs[int(gi)].V, dtype=np.int32) for gi in g]
            for i, h in enumerate(host):
                ptrs[i] = h.ctypes.data
        wall = C.c_double(0)
        check(lib.xbfs_serve_run(self._h, n, g.ctypes.data, s.ctypes.data, a.ctypes.data, mode,
                                 admit.ctypes.data, fin.ctypes.data, mc.ctypes.data,
                                 C.cast(ptrs, C.c_void_p) if mode else None, C.byref(wall)))
        lat = fin - a
        out = {"admit_us": admit, "finish_us": fin, "latency_us": lat, "edges_mc": mc, "wall_us": wall.value,
               "p50_us": float(np.percentile(lat, 50)) if n else 0.0,
               "p99_us": float(np.percentile(lat, 99)) if n else 0.0,
               "gteps": float(mc.sum() / (wall.value * 1e-6) / 1e9) if wall.value > 0 else 0.0}
        if mode == 1:
            out["levels_dev"] = [ptrs[i] for i in range(n)]
        if mode == 2:
            out["levels"] = host
        return out

    # -- online mode -----------------------------------------------------------
    OUTPUTS = {"none": 0, "device": 1, "host": 2}

    def start(self) -> None:
        """Run the engine in the server's own thread; requests come from submit()."""
        check(lib.xbfs_serve_start(self._h))
        self._host = {}

    def submit(self, graph: int, src: int, output: str = "none", levels: Optional[np.ndarray] = None) -> int:
        """Queue one request; returns its ticket at once. ``output``: "none"
        (edge count and times only), "device" (kept level array, see poll /
        fetch), "host" (copied into ``levels`` or a new array before done)."""
        mode = self.OUTPUTS[output]
        if mode == 2 and levels is None:
            levels = np.empty(self.graphs[graph].V, dtype=np.int32)
        t = C.c_int64(0)
        check(lib.xbfs_serve_submit(self._h, int(graph), int(src), mode,
                                    levels.ctypes.data if mode == 2 else None, C.byref(t)))
        if mode == 2:
            self._host[t.value] = levels
        return t.value

    def poll(self, ticket: int, wait_us: int = 0) -> Optional[dict]:
        """The request's result when done (None while it waits or runs);
        ``wait_us`` < 0 waits until done."""
        r = _lib.ServeResult()
        r.struct_size = C.sizeof(_lib.ServeResult)
        st = lib.xbfs_serve_poll(self._h, int(ticket), int(wait_us), C.byref(r))
        if st == _lib.XBFS_ERR_BUSY:
            return None
        check(st)
        out = {"submit_us": r.submit_us, "admit_us": r.admit_us, "finish_us": r.finish_us,
               "latency_us": r.finish_us - r.submit_us, "edges_mc": r.edges_mc}
        if r.levels_dev:
            out["levels_dev"] = r.levels_dev
        if ticket in self._host:
            out["levels"] = self._host.pop(ticket)
        return out

    def stop(self) -> None:
        check(lib.xbfs_serve_stop(self._h))

    def fetch(self, ptr: int, V: int) -> np.ndarray:
        """Copy one kept device level array to the host and release it."""
        host = np.empty(V, dtype=np.int32)
        check(lib.xbfs_serve_fetch(self._h, C.c_void_p(ptr), V, host.ctypes.data))
        return host

    def free(self) -> None:
        if self._h:
            lib.xbfs_serve_free(self._h)   # stops the online thread first
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
