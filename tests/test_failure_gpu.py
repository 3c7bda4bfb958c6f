"""Failure detection on the GPU without a fault: every device-side wait of
the traversal kernel is bounded in time. One CTA is told to leave before its
first grid barrier (xbfs_opts.test_absent_block), so the barrier can never
complete; the others give up after wait_timeout_us, the call returns
XBFS_ERR_DEVICE_TIMEOUT, and the same context and graph handle then traverse
normally."""
import time

import numpy as np
import pytest

import oracle
from xbfs_b200 import Graph, XbfsError, gen_rmat_host, pick_sources
from xbfs_b200._lib import XBFS_ERR_DEVICE_TIMEOUT

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("absent", [1, 7])
def test_missing_block_ends_in_a_timeout_status(absent):
    beg, csr = gen_rmat_host(14, 16, 3)
    g = Graph.from_csr(beg, csr)
    s = int(pick_sources(beg, 1, 2)[0])
    t0 = time.perf_counter()
    with pytest.raises(XbfsError) as e:
        g.bfs(s, wait_timeout_us=20000, test_absent_block=absent)
    assert e.value.status == XBFS_ERR_DEVICE_TIMEOUT
    assert time.perf_counter() - t0 < 5.0   # bounded by the 20 ms limit, not the 10 s default
    # the context and the handle are still usable
    for _ in range(2):
        r = g.bfs(s, want_parents=True)
        assert np.array_equal(r.levels, oracle.bfs_queue(beg, csr, s))
        assert oracle.check_tree(beg, csr, s, r.levels, r.parents) == 0
    g.free()


def test_short_limit_alone_does_not_fire():
    beg, csr = gen_rmat_host(15, 16, 4)
    g = Graph.from_csr(beg, csr)
    s = int(pick_sources(beg, 1, 3)[0])
    r = g.bfs(s, wait_timeout_us=200000)
    assert np.array_equal(r.levels, oracle.bfs_queue(beg, csr, s))
    g.free()
