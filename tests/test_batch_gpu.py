"""Batched multi-source BFS (64 sources per uint64 word): every per-source
level array bit-exact against the serial CPU BFS, for every word width,
direction choice, duplicate sources, deep graphs (two-byte level rows) and
host or device output."""
import numpy as np
import pytest

import oracle
from tests.conftest import hand_graphs
from xbfs_b200 import Graph, gen_er_host, gen_grid_host, gen_rmat_host, pick_sources

pytestmark = pytest.mark.gpu


def check_batch(g, beg, csr, srcs, **kw):
    r = g.bfs_batch(srcs, **kw)
    mc = 0
    for i, s in enumerate(srcs):
        ref = oracle.bfs_queue(beg, csr, int(s))
        assert np.array_equal(r.levels[i], ref), f"source #{i} ({s}) differs at {np.nonzero(r.levels[i] != ref)[0][:8]}"
        mc += int(np.diff(beg)[ref >= 0].sum())
    assert r.edges_mc == mc // 2  # Graph500 m_c summed over sources
    return r


@pytest.mark.parametrize("words", [1, 2, 4, 8])
@pytest.mark.parametrize("direction", [None, "td", "bu"])
def test_rmat_all_widths_and_directions(words, direction):
    beg, csr = gen_rmat_host(12, 16, 3)
    g = Graph.from_csr(beg, csr)
    srcs = pick_sources(beg, 64 * words - 7, 3)  # a partial last word
    check_batch(g, beg, csr, srcs, words_per_vertex=words, direction=direction)


def test_512_sources_multiple_passes_and_duplicates():
    beg, csr = gen_rmat_host(13, 8, 5)
    g = Graph.from_csr(beg, csr)
    srcs = np.concatenate([pick_sources(beg, 300, 5), pick_sources(beg, 300, 5)[:40]])  # duplicates
    check_batch(g, beg, csr, srcs, words_per_vertex=2)   # 5 passes of 128
    check_batch(g, beg, csr, srcs[:512])                 # auto width


def test_hand_graphs_including_isolated_sources():
    for name, (beg, csr) in hand_graphs().items():
        g = Graph.from_csr(beg, csr)
        n = len(beg) - 1
        srcs = np.arange(n, dtype=np.int32) if n <= 64 else np.arange(0, n, max(1, n // 60), dtype=np.int32)
        check_batch(g, beg, csr, srcs, words_per_vertex=1)


def test_deep_grid_uses_wide_level_rows():
    beg, csr = gen_grid_host(300, 3)   # diameter ~ 301 > 254
    g = Graph.from_csr(beg, csr)
    check_batch(g, beg, csr, np.array([0, 450, 899, 1], dtype=np.int32), words_per_vertex=1)


def test_er_and_device_output():
    import torch
    beg, csr = gen_er_host(30000, 8.0, 2)
    g = Graph.from_csr(beg, csr)
    srcs = pick_sources(beg, 200, 2)
    out = torch.empty((len(srcs), g.V), dtype=torch.int32, device="cuda:0")
    g.bfs_batch(srcs, levels=out)
    torch.cuda.synchronize()
    lv = out.cpu().numpy()
    for i in (0, 57, 199):
        assert np.array_equal(lv[i], oracle.bfs_queue(beg, csr, int(srcs[i])))
