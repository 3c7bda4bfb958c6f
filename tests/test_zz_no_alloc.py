"""xbfs_bfs_noalloc: the allocation-free single-source traversal (workspace in
a fixed static device array). Checked against the ordinary entry point
xbfs_bfs on two calls in a row, plus the tree check of the oracle, and that
repeated calls leave the device's free memory unchanged. This file is named
to be collected last and does not depend on any other test's state."""
import ctypes as C

import numpy as np
import pytest

import oracle
from xbfs_b200 import Graph, gen_grid_host, gen_rmat_host, pick_sources
from xbfs_b200._lib import (XBFS_ERR_INVALID_ARG, XBFS_ERR_UNSUPPORTED, Opts, Stats, XbfsError, check, lib)
from xbfs_b200.api import BfsOptions

pytestmark = pytest.mark.gpu


def noalloc(g, src, levels, parents=None, opts=None):
    """One xbfs_bfs_noalloc call; levels/parents are CUDA tensors."""
    o = (opts or BfsOptions()).to_c()
    st = Stats()
    st.struct_size = C.sizeof(Stats)
    check(lib.xbfs_bfs_noalloc(g._h, int(src), levels.data_ptr(),
                               parents.data_ptr() if parents is not None else None, C.byref(o), C.byref(st)))
    return st


def free_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info(0)[0]


@pytest.mark.parametrize("kind", ["rmat", "grid"])
def test_two_calls_in_a_row_match_xbfs_bfs(kind):
    import torch
    if kind == "rmat":
        beg, csr = gen_rmat_host(15, 16, 21)
    else:
        beg, csr = gen_grid_host(300, 200)
    g = Graph.from_csr(beg, csr)
    srcs = [int(s) for s in pick_sources(beg, 2, 4)]
    lv = torch.empty(g.V, dtype=torch.int32, device="cuda:0")
    pa = torch.empty(g.V, dtype=torch.int32, device="cuda:0")
    noalloc(g, srcs[0], lv, pa)  # first call on the device: set-up
    f0 = free_bytes()
    got = []
    for s in srcs:
        st = noalloc(g, s, lv, pa)
        got.append((lv.cpu().numpy().copy(), pa.cpu().numpy().copy(), st.depth, st.reached))
    assert free_bytes() == f0
    for s, (levels, parents, depth, reached) in zip(srcs, got):
        r = g.bfs(s, want_parents=True)
        assert np.array_equal(levels, r.levels)
        assert depth == r.depth and reached == r.reached
        assert np.array_equal(levels, oracle.bfs_queue(beg, csr, s))
        assert oracle.check_tree(beg, csr, s, levels, parents) == 0
    g.free()


def test_policies_and_levels_only():
    import torch
    from xbfs_b200 import learned
    beg, csr = gen_rmat_host(14, 16, 5)
    g = Graph.from_csr(beg, csr)
    s = int(pick_sources(beg, 1, 9)[0])
    ref = oracle.bfs_queue(beg, csr, s)
    lv = torch.empty(g.V, dtype=torch.int32, device="cuda:0")
    w, _ = learned.load(learned.DEFAULT_WEIGHTS)
    learned.install(w, device=0)   # the learned switch stages its weights in shared memory
    try:
        for opts in (BfsOptions(policy="heuristic"), BfsOptions(policy="beamer"), BfsOptions(async_bu=False),
                     BfsOptions(policy="forced", forced=["td_queue", "td_scan", "bu", "bu", "td_scan"]),
                     BfsOptions(policy="mlp")):
            noalloc(g, s, lv, None, opts)
            assert np.array_equal(lv.cpu().numpy(), ref)
            assert np.array_equal(g.bfs(s, opts=opts).levels, ref)
    finally:
        learned.install(None, device=0)
    g.free()


def test_callers_stream():
    """opts.stream: the traversal runs on the caller's stream."""
    import torch
    beg, csr = gen_rmat_host(13, 16, 8)
    g = Graph.from_csr(beg, csr)
    st = torch.cuda.Stream()
    lv = torch.empty(g.V, dtype=torch.int32, device="cuda:0")
    for s in pick_sources(beg, 2, 3):
        with torch.cuda.stream(st):
            noalloc(g, int(s), lv, None, BfsOptions(stream=st.cuda_stream))
        st.synchronize()
        assert np.array_equal(lv.cpu().numpy(), oracle.bfs_queue(beg, csr, int(s)))
    g.free()


def test_bounded_wait_and_the_next_call():
    """wait_timeout_us bounds the device-side waits as in xbfs_bfs: one CTA
    leaves before its first grid barrier (test_absent_block), the others give
    up after 20 ms, the call returns XBFS_ERR_DEVICE_TIMEOUT, and the next
    call on the same array is correct (it clears what it reads first)."""
    import time

    import torch
    from xbfs_b200._lib import XBFS_ERR_DEVICE_TIMEOUT
    beg, csr = gen_rmat_host(14, 16, 3)
    g = Graph.from_csr(beg, csr)
    s = int(pick_sources(beg, 1, 2)[0])
    lv = torch.empty(g.V, dtype=torch.int32, device="cuda:0")
    t0 = time.perf_counter()
    with pytest.raises(XbfsError) as e:
        noalloc(g, s, lv, None, BfsOptions(wait_timeout_us=20000, test_absent_block=3))
    assert e.value.status == XBFS_ERR_DEVICE_TIMEOUT
    assert time.perf_counter() - t0 < 5.0   # the 20 ms bound, not the 10 s default
    pa = torch.empty(g.V, dtype=torch.int32, device="cuda:0")
    noalloc(g, s, lv, pa)
    levels = lv.cpu().numpy()
    assert np.array_equal(levels, oracle.bfs_queue(beg, csr, s))
    assert oracle.check_tree(beg, csr, s, levels, pa.cpu().numpy()) == 0
    g.free()


def test_largest_fitting_graph_and_refusal_beyond():
    import torch
    g = Graph.rmat(20, 16, 3)  # about 45 MiB of workspace: fits
    lv = torch.empty(g.V, dtype=torch.int32, device="cuda:0")
    noalloc(g, 1, lv)
    assert np.array_equal(lv.cpu().numpy(), g.bfs(1).levels)
    g.free()
    del lv
    g = Graph.rmat(21, 16, 3)  # about 89 MiB: refused with the size in the message
    lv = torch.empty(g.V, dtype=torch.int32, device="cuda:0")
    with pytest.raises(XbfsError) as e:
        noalloc(g, 1, lv)
    assert e.value.status == XBFS_ERR_UNSUPPORTED and "bytes of traversal scratch" in e.value.detail
    g.free()


def test_host_buffers_and_trace_are_refused():
    import torch
    beg, csr = gen_rmat_host(10, 8, 1)
    g = Graph.from_csr(beg, csr)
    host = np.empty(g.V, dtype=np.int32)
    st = Stats()
    st.struct_size = C.sizeof(Stats)
    o = BfsOptions().to_c()
    assert lib.xbfs_bfs_noalloc(g._h, 0, host.ctypes.data, None, C.byref(o), C.byref(st)) == XBFS_ERR_INVALID_ARG
    lv = torch.empty(g.V, dtype=torch.int32, device="cuda:0")
    with pytest.raises(XbfsError) as e:
        noalloc(g, 0, lv, None, BfsOptions(trace=True))
    assert e.value.status == XBFS_ERR_UNSUPPORTED
    g.free()
