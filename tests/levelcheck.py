"""Size-independent check of a BFS level array on the GPU (test infrastructure).

On a symmetric CSR an int32 array L is exactly the BFS distance array from
src (-1 for unreached vertices) if and only if

  1. L[src] == 0, and every other entry is -1 or >= 1;
  2. for every edge (u, v) with L[u] >= 0: L[v] >= 0 and L[v] <= L[u] + 1
     (reached sets are closed and levels grow by at most one along an edge);
  3. every reached v != src has a neighbour w with L[w] == L[v] - 1 >= 0.

(3) gives every reached vertex a path of length L[v] back to the only
level-0 vertex, so L[v] >= dist(v); (2) along a shortest path gives
L[v] <= dist(v) and reaches every reachable vertex. The check runs with
plain torch tensor operations, independent of the library's kernels, so it
covers level arrays at sizes where a CPU oracle per source would be slow.
"""
from __future__ import annotations

import numpy as np


class LevelChecker:
    def __init__(self, beg: np.ndarray, csr: np.ndarray, device: str = "cuda:0"):
        import torch
        self.torch = torch
        self.V = len(beg) - 1
        self.beg = torch.from_numpy(np.ascontiguousarray(beg, dtype=np.int64)).to(device)
        self.csr = torch.from_numpy(np.ascontiguousarray(csr, dtype=np.int32)).to(device).long()
        deg = self.beg[1:] - self.beg[:-1]
        self.row = torch.repeat_interleave(torch.arange(self.V, device=device), deg)

    def violations(self, L, src: int) -> dict:
        """Counts of vertices / edges breaking each condition (all 0 = exact)."""
        torch = self.torch
        L = L.to(self.beg.device).long()
        out = {"src": int(L[src].item() != 0)}
        other = torch.ones(self.V, dtype=torch.bool, device=L.device)
        other[src] = False
        out["range"] = int(((L == 0) & other).sum().item() + (L < -1).sum().item())
        Lu = L[self.row]
        Lv = L[self.csr]
        reached_u = Lu >= 0
        out["closure"] = int((reached_u & ((Lv < 0) | (Lv > Lu + 1))).sum().item())
        good = ((Lv == Lu - 1) & (Lv >= 0)).to(torch.int64)
        c = torch.zeros(len(good) + 1, dtype=torch.int64, device=L.device)
        torch.cumsum(good, 0, out=c[1:])
        per_vertex = c[self.beg[1:]] - c[self.beg[:-1]]
        need = (L >= 1) & other
        out["parent"] = int((need & (per_vertex == 0)).sum().item())
        return out

    def exact(self, L, src: int) -> bool:
        return all(v == 0 for v in self.violations(L, src).values())
