"""Parity at the sizes the throughput numbers are quoted on.

Each benchmark configuration, built with the same generators, seeds and
sources as bench.py, is traversed through the C ABI and compared with the
CPU oracle: the serial FIFO BFS where it finishes in seconds, else the
OpenMP direction-optimising BFS (itself pinned to the FIFO BFS by
tests/test_oracle.py and cross-checked against it here on one source).
Where a CPU answer per row would take too long (512 batched sources), every
row also passes the size-independent exactness check of tests/levelcheck.py.

  * plain single-source BFS, R-MAT scale 16 edge factor 16, all 64 sources;
  * R-MAT scale 23 edge factor 32 (the headline graph), 8 sources, with
    parents tree-checked, through xbfs_bfs and the pipelined xbfs_bfs_many;
  * the 4096 x 4096 grid, 2 sources, heuristic and learned switch;
  * batched: 512 sources on R-MAT scale 22 edge factor 16 (8 uint64 words per
    vertex, 8.6 GB of output), 16 rows against the oracle across all words
    and every row through the exactness check;
  * the 256-graph uneven multi-graph launch, every graph;
  * the serving loop over the 8 serving graphs (R-MAT scales 20-24, grids up
    to 8192 x 2048), 48 requests with Poisson arrivals, every answer.
"""
import numpy as np
import pytest

import oracle
from tests.levelcheck import LevelChecker
from xbfs_b200 import BfsOptions, Graph, MultiGraph, pick_sources

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def oracle_levels(beg, csr, src, serial=False):
    return oracle.bfs_queue(beg, csr, int(src)) if serial else oracle.bfs_do(beg, csr, int(src))


def test_rmat_s16_ef16_all_64_sources():
    g = Graph.rmat(16, 16, 1)
    beg, csr = g.download()
    srcs = pick_sources(beg, 64, 1)
    rows = g.bfs_many(srcs).levels
    for i, s in enumerate(srcs):
        ref = oracle.bfs_queue(beg, csr, int(s))
        assert np.array_equal(rows[i], ref), f"source {s}"
        r = g.bfs(int(s), want_parents=True)
        assert np.array_equal(r.levels, ref)
        assert oracle.check_tree(beg, csr, int(s), r.levels, r.parents) == 0
        assert r.edges_mc == oracle.edges_mc(beg, ref)
    g.free()


def test_rmat_s23_ef32_headline_graph():
    import torch
    g = Graph.rmat(23, 32, 1)
    beg, csr = g.download()
    assert g.E < (1 << 32) and g.E > (1 << 28)  # bins' 32-bit edge offsets are exercised near their range
    srcs = pick_sources(beg, 8, 1)
    rows = torch.empty((len(srcs), g.V), dtype=torch.int32, device="cuda:0")
    g.bfs_many(srcs, levels=rows)
    torch.cuda.synchronize()
    pa = np.empty(g.V, dtype=np.int32)
    for i, s in enumerate(srcs):
        ref = oracle_levels(beg, csr, s, serial=(i == 0))
        if i == 0:
            assert np.array_equal(ref, oracle.bfs_do(beg, csr, int(s)))
        assert np.array_equal(rows[i].cpu().numpy(), ref), f"bfs_many row {i} (source {s})"
        r = g.bfs(int(s), parents=pa)
        assert np.array_equal(r.levels, ref), f"xbfs_bfs source {s}"
        assert oracle.check_tree(beg, csr, int(s), r.levels, pa) == 0
        assert r.edges_mc == oracle.edges_mc(beg, ref)
    g.free()


def test_grid_4096_squared_two_sources():
    from xbfs_b200 import learned
    g = Graph.grid(4096, 4096)
    beg, csr = g.download()
    assert g.E == 67_092_480
    w, _ = learned.load(learned.DEFAULT_WEIGHTS)
    learned.install(w, device=0)
    try:
        for s in pick_sources(beg, 2, 1):
            ref = oracle.bfs_queue(beg, csr, int(s))
            for pol in ("heuristic", "mlp"):
                r = g.bfs(int(s), opts=BfsOptions(policy=pol))
                assert np.array_equal(r.levels, ref), f"source {s}, policy {pol}"
                assert r.depth == int(ref.max()) + 1
    finally:
        learned.install(None, device=0)
    g.free()


def test_batched_512_sources_rmat_s22_ef16():
    import torch
    g = Graph.rmat(22, 16, 1)
    beg, csr = g.download()
    srcs = pick_sources(beg, 512, 1)
    out = torch.empty((512, g.V), dtype=torch.int32, device="cuda:0")
    r = g.bfs_batch(srcs, levels=out)
    torch.cuda.synchronize()
    # two rows in each of the 8 words: first lane and a middle/last lane
    sample = sorted({64 * w + k for w in range(8) for k in (0, 37 + w)} | {511})
    for i in sample:
        ref = oracle_levels(beg, csr, srcs[i])
        assert np.array_equal(out[i].cpu().numpy(), ref), f"row {i} (source {srcs[i]})"
    chk = LevelChecker(beg, csr)
    bad = [i for i in range(512) if not chk.exact(out[i], int(srcs[i]))]
    assert not bad, f"rows failing the exactness check: {bad[:10]}"
    # Graph500 edge count summed over the sources, from the rows themselves
    deg = torch.from_numpy(np.diff(beg)).to("cuda:0")
    mc = sum(int(deg[out[i] >= 0].sum().item()) for i in range(512)) // 2
    assert r.edges_mc == mc
    del out
    g.free()


def test_multi_graph_256_uneven_graphs():
    rng = np.random.default_rng(1)
    graphs = [Graph.rmat(int(rng.integers(10, 19)), int(rng.integers(8, 33)), 100 + i) for i in range(128)]
    graphs += [Graph.er(int(rng.integers(1000, 200001)), 8.0, 300 + i) for i in range(128)]
    cpu = [g.download() for g in graphs]
    srcs = np.array([int(pick_sources(b, 1, 7 + i)[0]) for i, (b, _) in enumerate(cpu)], dtype=np.int32)
    mg = MultiGraph(graphs)
    mg.tune(srcs, reps=1)
    for rep in range(2):  # first launch and a CUDA-graph replay
        r = mg.bfs(srcs)
        mc = 0
        for k, ((b, c), s, lv) in enumerate(zip(cpu, srcs, mg.split(r.levels))):
            ref = oracle.bfs_queue(b, c, int(s))
            assert np.array_equal(lv, ref), f"graph {k} (V={len(b) - 1}), replay {rep}"
            mc += oracle.edges_mc(b, ref)
        assert r.edges_mc == mc
    mg.free()
    for g in graphs:
        g.free()


def test_serving_graphs_every_answer():
    from xbfs_b200.api import Server
    specs = [("rmat", s) for s in (20, 21, 22, 23, 24)] + [("grid", 2048, 2048), ("grid", 4096, 4096),
                                                           ("grid", 8192, 2048)]
    graphs = [Graph.rmat(sp[1], 16, 1 + sp[1]) if sp[0] == "rmat" else Graph.grid(sp[1], sp[2]) for sp in specs]
    cpu = [g.download() for g in graphs]
    rng = np.random.default_rng(5)
    n = 48
    gid = rng.integers(0, len(graphs), size=n).astype(np.int32)
    gid[:8] = np.arange(8)  # every graph at least once
    src = np.array([pick_sources(cpu[k][0], 1, 1000 + i)[0] for i, k in enumerate(gid)], dtype=np.int32)
    arr = np.cumsum(rng.exponential(1e6 / 1e3, size=n))
    srv = Server(graphs)
    res = srv.run(gid, src, arr, to_host=True)
    for i, (k, s) in enumerate(zip(gid, src)):
        b, c = cpu[k]
        ref = oracle_levels(b, c, s, serial=(specs[k][0] == "grid"))
        assert np.array_equal(res["levels"][i], ref), f"request {i} (graph {k}, source {s})"
        assert res["edges_mc"][i] == oracle.edges_mc(b, ref)
    srv.free()
    for g in graphs:
        g.free()
