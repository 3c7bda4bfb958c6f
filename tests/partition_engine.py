"""CPU stand-in for the per-rank device steps of the partitioned BFS
(xbfs_b200.partition.DeviceEngine), in numpy, for testing the exchange
logic on gloo ranks without a GPU. Test infrastructure only."""
import numpy as np
import torch


class NumpyEngine:
    def __init__(self, beg_local, csr_local, V, lo, hi, symmetric=True):
        self.V, self.lo, self.hi, self.n = V, lo, hi, hi - lo
        self.beg = np.asarray(beg_local, dtype=np.int64)
        self.csr = np.asarray(csr_local, dtype=np.int32)
        self.cand = torch.zeros(V, dtype=torch.uint8)
        self.deg = np.diff(self.beg)

    def new_bits(self, words):
        return torch.zeros(words, dtype=torch.int32)

    def reset(self, src):
        self.cand.zero_()
        self.lv = np.full(self.n, -1, dtype=np.int32)
        self.front = np.zeros(0, dtype=np.int64)
        if self.lo <= src < self.hi:
            self.lv[src - self.lo] = 0
            self.front = np.array([src - self.lo])

    def stats(self):
        un = (self.lv < 0) & (self.deg > 0)
        return [len(self.front), int(self.deg[self.front].sum()), int(un.sum()), int(self.deg[un].sum())]

    def td_expand(self):
        c = self.cand.numpy()
        for u in self.front:
            c[self.csr[self.beg[u]:self.beg[u + 1]]] = 1

    def claim(self, next_level):
        c = self.cand.numpy()
        new = np.nonzero((c[self.lo:self.hi] != 0) & (self.lv < 0))[0]
        self.lv[new] = next_level
        self.front = new
        c[:] = 0

    def frontier_bits(self, mine):
        w = mine.numpy().view(np.uint32)
        w[:] = 0
        for v in self.front:
            w[v >> 5] |= np.uint32(1 << (v & 31))

    def bottom_up(self, everyone, next_level):
        bits = everyone.numpy().view(np.uint32)
        new = []
        for i in np.nonzero(self.lv < 0)[0]:
            nb = self.csr[self.beg[i]:self.beg[i + 1]]
            if np.any((bits[nb >> 5] >> (nb & 31).astype(np.uint32)) & 1):
                new.append(i)
        new = np.array(new, dtype=np.int64)
        self.lv[new] = next_level
        self.front = new

    def levels(self):
        return self.lv.copy()
