"""The CPU oracle against independent answers: networkx on tiny graphs, the
serial FIFO BFS vs the restated reference sweep vs the OpenMP DO-BFS, and
the reference-schedule replay. CPU only."""
import numpy as np
import pytest

import oracle
from xbfs_b200 import gen_er_host, gen_grid_host, gen_rmat_host, pick_sources


def nx_levels(beg, csr, src):
    import networkx as nx
    G = nx.DiGraph()
    n = len(beg) - 1
    G.add_nodes_from(range(n))
    for u in range(n):
        for e in range(beg[u], beg[u + 1]):
            G.add_edge(u, int(csr[e]))
    d = nx.single_source_shortest_path_length(G, src)
    out = np.full(n, -1, dtype=np.int32)
    for k, v in d.items():
        out[k] = v
    return out


def is_symmetric(beg, csr):
    V = len(beg) - 1
    src = np.repeat(np.arange(V, dtype=np.int64), np.diff(beg))
    a = np.unique(src * V + csr)
    b = np.unique(csr.astype(np.int64) * V + src)
    return np.array_equal(a, b)


def test_hand_graphs_vs_networkx(graphs):
    for name, (beg, csr) in graphs.items():
        n = len(beg) - 1
        for src in sorted({0, n // 2, n - 1}):
            ref = nx_levels(beg, csr, src)
            assert np.array_equal(oracle.bfs_queue(beg, csr, src), ref), name
            sw, k = oracle.bfs_sweep(beg, csr, src)
            assert np.array_equal(sw, ref), name
            assert k == int(ref.max()) + 1, (name, k)  # the reference loop exits after an idle sweep
            if is_symmetric(beg, csr):  # bottom-up reads in-edges through the out-adjacency
                assert np.array_equal(oracle.bfs_do(beg, csr, src, threads=2), ref), name


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_rmat_small_all_oracles_agree(seed):
    beg, csr = gen_rmat_host(10, 16, seed)
    srcs = pick_sources(beg, 8, seed)
    for s in srcs:
        q = oracle.bfs_queue(beg, csr, s)
        assert np.array_equal(q, nx_levels(beg, csr, int(s)))
        assert np.array_equal(oracle.bfs_sweep(beg, csr, s)[0], q)
        assert np.array_equal(oracle.bfs_sweep(beg, csr, s, threads=4)[0], q)
        assert np.array_equal(oracle.bfs_do(beg, csr, s, threads=4), q)


def test_parallel_sweep_and_do_on_larger_graphs():
    for beg, csr in (gen_rmat_host(14, 16, 7), gen_grid_host(64, 48), gen_er_host(5000, 8.0, 3)):
        for s in pick_sources(beg, 3, 11):
            q = oracle.bfs_queue(beg, csr, s)
            assert np.array_equal(oracle.bfs_sweep(beg, csr, s, threads=8)[0], q)
            assert np.array_equal(oracle.bfs_do(beg, csr, s, threads=8), q)


def test_tree_check_accepts_valid_and_rejects_planted_errors():
    beg, csr = gen_rmat_host(9, 8, 5)
    src = int(pick_sources(beg, 1, 5)[0])
    lv = oracle.bfs_queue(beg, csr, src)
    # build a valid parent array on the CPU
    par = np.full(len(lv), -1, dtype=np.int32)
    par[src] = src
    for v in range(len(lv)):
        if lv[v] > 0:
            for e in range(beg[v], beg[v + 1]):
                if lv[csr[e]] == lv[v] - 1:
                    par[v] = csr[e]
                    break
    assert oracle.check_tree(beg, csr, src, lv, par) == 0
    # planted mistakes (in the oracle's input, on the CPU)
    reached = np.nonzero(lv > 1)[0]
    bad = par.copy()
    bad[reached[0]] = src if lv[reached[0]] > 1 else bad[reached[0]]
    assert oracle.check_tree(beg, csr, src, lv, bad) != 0
    bad = par.copy()
    unreached = np.nonzero(lv < 0)[0]
    if len(unreached):
        bad[unreached[0]] = src
        assert oracle.check_tree(beg, csr, src, lv, bad) == unreached[0] + 1


def test_reference_schedule_shapes():
    beg, csr = gen_rmat_host(14, 16, 1)
    src = int(pick_sources(beg, 1, 1)[0])
    lv = oracle.bfs_queue(beg, csr, src)
    tags = oracle.reference_schedule(beg, lv, 0.1)
    assert len(tags) == lv.max()
    assert set(tags) <= {0, 1, -1}
    assert -1 in tags  # a scale-14 R-MAT has a level above 10% of the edges
    assert tags[0] == 0


def test_edges_mc():
    beg, csr = gen_rmat_host(10, 8, 2)
    lv = oracle.bfs_queue(beg, csr, int(pick_sources(beg, 1, 2)[0]))
    deg = np.diff(beg)
    assert oracle.edges_mc(beg, lv) == int(deg[lv >= 0].sum()) // 2
