"""The size-independent exactness check (tests/levelcheck.py) on the CPU:
oracle level arrays pass it, and every kind of planted mistake in an oracle
array is caught. CPU only (torch on the CPU device)."""
import numpy as np

import oracle
from tests.levelcheck import LevelChecker
from xbfs_b200 import gen_grid_host, gen_rmat_host, pick_sources


def test_oracle_levels_pass_and_planted_mistakes_fail():
    for beg, csr in (gen_rmat_host(12, 16, 3), gen_grid_host(40, 30)):
        chk = LevelChecker(beg, csr, device="cpu")
        import torch
        for s in pick_sources(beg, 3, 2):
            s = int(s)
            ref = oracle.bfs_queue(beg, csr, s)
            assert chk.exact(torch.from_numpy(ref), s)
            reached = np.nonzero((ref >= 1))[0]
            v = int(reached[len(reached) // 2])
            for bad_value in (ref[v] + 1, ref[v] - 1, -1, 0):
                bad = ref.copy()
                bad[v] = bad_value
                if bad_value == ref[v]:
                    continue
                assert not chk.exact(torch.from_numpy(bad), s), (s, v, bad_value)
            bad = ref.copy()
            bad[s] = 1
            assert not chk.exact(torch.from_numpy(bad), s)
            # a whole level shifted up by one (consistent among themselves)
            bad = ref.copy()
            bad[ref == ref.max()] += 1
            assert not chk.exact(torch.from_numpy(bad), s)
