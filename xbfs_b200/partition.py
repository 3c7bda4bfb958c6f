"""1D-partitioned single-source BFS over several GPUs (one process per GPU).

No counterpart in the reference, which runs one source on one GPU
(bfs_gpu_update.cu:138). The vertex range is cut into ``world`` contiguous
slices of equal, 32-aligned size (the last one shorter); rank r holds the
CSR rows of its slice, read straight from the reference's file pair, and the
levels of its own vertices. Every level is host-driven, identically on all
ranks:

* the four frontier statistics (n_f, m_f, n_u, m_u) are summed across ranks
  and the direction is chosen from the sums (Beamer's alpha/beta rule; only
  top-down on a directed CSR);
* top-down: each rank marks the neighbours of its frontier in a byte per
  vertex over all V vertices, the arrays are combined with a MAX all-reduce,
  and each rank claims the unvisited marked vertices of its slice;
* bottom-up: each rank writes its frontier into its words of a V-bit
  bitmap, the words are all-gathered (V/8 bytes in total), and each rank's
  unvisited vertices probe their neighbours in the whole bitmap.

The device steps are CUDA kernels (``DeviceEngine``, xbfs_part_* in
libxbfs.so); the collectives go through ``torch.distributed`` (NCCL over
NVLink between GPUs). Any object with the engine's methods can stand in,
which is how the exchange is tested on CPU ranks with ``gloo``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import check, lib


def slice_words(V: int, world: int) -> int:
    """32-bit words per rank slice (every slice but the last has exactly this many)."""
    words = (V + 31) // 32
    return max(1, (words + world - 1) // world)


def bounds(V: int, world: int) -> list[int]:
    """Vertex bounds of the slices: rank r owns [b[r], b[r+1])."""
    w = slice_words(V, world)
    return [min(V, 32 * w * r) for r in range(world + 1)]


def local_rows(beg: np.ndarray, csr: np.ndarray, lo: int, hi: int) -> tuple[np.ndarray, np.ndarray]:
    """The CSR rows of vertices [lo, hi): offsets rebased to 0, global neighbour ids."""
    b = np.asarray(beg[lo:hi + 1], dtype=np.int64)
    return b - b[0], np.asarray(csr[b[0]:b[-1]], dtype=np.int32)


class DeviceEngine:
    """The per-rank device steps (CUDA kernels in libxbfs.so), with the
    candidate array and the bitmap in device memory for the collectives."""

    def __init__(self, beg_local, csr_local, V: int, lo: int, hi: int, symmetric: bool, device: int = 0):
        import torch
        self.torch = torch
        self.V, self.lo, self.hi, self.n = V, lo, hi, hi - lo
        self.device = device
        bl = np.ascontiguousarray(beg_local, dtype=np.int64)
        cl = np.ascontiguousarray(csr_local, dtype=np.int32)
        h = C.c_void_p()
        check(lib.xbfs_part_create(bl.ctypes.data, cl.ctypes.data if cl.size else None, V, lo, hi,
                                   1 if symmetric else 0, device, C.byref(h)))
        self._h = h
        dev = torch.device("cuda", device)
        self.cand = torch.zeros(V, dtype=torch.uint8, device=dev)

    def new_bits(self, words: int):
        return self.torch.zeros(words, dtype=self.torch.int32, device=self.cand.device)

    def reset(self, src: int) -> None:
        self.cand.zero_()
        self.torch.cuda.synchronize(self.device)
        check(lib.xbfs_part_reset(self._h, int(src)))

    def stats(self) -> list[int]:
        out = np.zeros(4, dtype=np.int64)
        check(lib.xbfs_part_stats(self._h, out.ctypes.data))
        return out.tolist()

    def td_expand(self) -> None:
        check(lib.xbfs_part_td_expand(self._h, self.cand.data_ptr()))

    def claim(self, next_level: int) -> None:
        check(lib.xbfs_part_claim(self._h, self.cand.data_ptr(), int(next_level)))

    def frontier_bits(self, slice_t) -> None:
        check(lib.xbfs_part_frontier_bits(self._h, slice_t.data_ptr(), slice_t.numel()))

    def bottom_up(self, bits_t, next_level: int) -> None:
        check(lib.xbfs_part_bottom_up(self._h, bits_t.data_ptr(), int(next_level)))

    def levels(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.int32)
        if self.n:
            check(lib.xbfs_part_levels(self._h, out.ctypes.data))
        return out

    def free(self) -> None:
        if self._h:
            lib.xbfs_part_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class TorchComm:
    """The three collectives of the level loop over torch.distributed."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)

    def sum(self, vals, like):
        t = like.new_tensor(vals, dtype=self._i64())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return [int(x) for x in t.tolist()]

    def max_bytes(self, t) -> None:
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX, group=self.group)

    def gather_words(self, out, mine) -> None:
        """out: world * len(mine) words, rank r's words at [r * len(mine), ...)."""
        if hasattr(self.dist, "all_gather_into_tensor") and out.is_cuda:
            self.dist.all_gather_into_tensor(out, mine, group=self.group)
        else:
            parts = list(out.split(mine.numel()))
            self.dist.all_gather(parts, mine, group=self.group)

    def _i64(self):
        import torch
        return torch.int64


@dataclass
class Result:
    levels: np.ndarray   # levels of the rank's own vertices [lo, hi)
    depth: int
    strategies: list     # "td" / "bu" per level


def partitioned_bfs(engine, comm, src: int, symmetric: bool = True, alpha: float = 14.0,
                    beta: float = 24.0) -> Result:
    """The level loop of one rank (all ranks call it with the same src)."""
    V = engine.V
    W = slice_words(V, comm.world)
    mine = engine.new_bits(W)
    everyone = engine.new_bits(W * comm.world)
    engine.reset(src)
    level, bu, sched = 0, False, []
    while True:
        n_f, m_f, n_u, m_u = comm.sum(engine.stats(), everyone)
        if n_f == 0:
            break
        if symmetric:
            if not bu and m_f > m_u / alpha:
                bu = True
            elif bu and n_f < V / beta:
                bu = False
        if bu:
            engine.frontier_bits(mine)
            comm.gather_words(everyone, mine)
            engine.bottom_up(everyone, level + 1)
        else:
            engine.td_expand()
            comm.max_bytes(engine.cand)
            engine.claim(level + 1)
        sched.append("bu" if bu else "td")
        level += 1
    return Result(levels=engine.levels(), depth=level, strategies=sched)
