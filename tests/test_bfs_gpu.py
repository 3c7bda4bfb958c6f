"""Single-source BFS on the GPU through the C ABI, bit-exact against the CPU
oracle (serial FIFO BFS), on hand graphs, R-MAT, grids and ER graphs, under
every policy, forced strategy schedules, bin thresholds and with parents
checked as a BFS tree."""
import itertools

import numpy as np
import pytest

import oracle
from tests.conftest import hand_graphs
from xbfs_b200 import BfsOptions, Graph, XbfsError, gen_er_host, gen_grid_host, gen_rmat_host, pick_sources
from xbfs_b200 import _lib

pytestmark = pytest.mark.gpu


def run_and_check(g, beg, csr, src, **kw):
    want_parents = kw.pop("want_parents", True)
    r = g.bfs(int(src), want_parents=want_parents, **kw)
    ref = oracle.bfs_queue(beg, csr, src)
    assert np.array_equal(r.levels, ref), f"levels differ at {np.nonzero(r.levels != ref)[0][:10]}"
    if want_parents:
        assert oracle.check_tree(beg, csr, src, r.levels, r.parents) == 0
    assert r.depth == int(ref.max()) + 1
    assert r.reached == int((ref >= 0).sum())
    assert r.edges_mc == oracle.edges_mc(beg, ref)
    return r


def test_hand_graphs_all_sources():
    for name, (beg, csr) in hand_graphs().items():
        g = Graph.from_csr(beg, csr)
        n = len(beg) - 1
        for src in range(n) if n <= 40 else [0, 1, n // 2, n - 1]:
            for policy in ("heuristic", "beamer"):
                run_and_check(g, beg, csr, src, policy=policy)
        g.free()


@pytest.mark.parametrize("scale,ef,seed", [(10, 16, 1), (12, 8, 2), (14, 16, 3), (16, 16, 4)])
def test_rmat_heuristic_and_beamer(scale, ef, seed):
    beg, csr = gen_rmat_host(scale, ef, seed)
    g = Graph.from_csr(beg, csr)
    for s in pick_sources(beg, 8, seed):
        run_and_check(g, beg, csr, s, policy="heuristic")
        run_and_check(g, beg, csr, s, policy="beamer", want_parents=False)
        run_and_check(g, beg, csr, s, policy="heuristic", async_bu=False, want_parents=False)


def test_every_forced_schedule_prefix_gives_identical_levels():
    beg, csr = gen_rmat_host(12, 16, 9)
    g = Graph.from_csr(beg, csr)
    srcs = pick_sources(beg, 2, 9)
    for sched in itertools.product(["td_queue", "td_scan", "bu"], repeat=4):
        for tail in ("td_queue", "td_scan", "bu"):
            for s in srcs:
                run_and_check(g, beg, csr, s, policy="forced", forced=list(sched) + [tail],
                              want_parents=(tail == "bu"))


@pytest.mark.parametrize("seed", range(6))
def test_random_schedules_larger(seed):
    rng = np.random.default_rng(seed)
    beg, csr = gen_rmat_host(16, 16, 100 + seed)
    g = Graph.from_csr(beg, csr)
    for s in pick_sources(beg, 4, seed):
        sched = rng.integers(0, 3, size=12).tolist()
        run_and_check(g, beg, csr, s, policy="forced", forced=sched, async_bu=bool(seed % 2))


@pytest.mark.parametrize("small_max,medium_max", [(1, 1), (4, 16), (32, 256), (64, 64), (1024, 4096)])
def test_bin_thresholds(small_max, medium_max):
    beg, csr = gen_rmat_host(14, 32, 5)
    g = Graph.from_csr(beg, csr)
    for s in pick_sources(beg, 4, 5):
        run_and_check(g, beg, csr, s, small_max=small_max, medium_max=medium_max,
                      policy="forced", forced=["td_queue"])
        run_and_check(g, beg, csr, s, small_max=small_max, medium_max=medium_max)


def test_grid_long_diameter():
    for W, H in [(64, 64), (300, 7), (1, 500), (257, 129)]:
        beg, csr = gen_grid_host(W, H)
        g = Graph.from_csr(beg, csr)
        for s in [0, (W * H) // 2, W * H - 1]:
            run_and_check(g, beg, csr, s)
            run_and_check(g, beg, csr, s, policy="forced", forced=["td_scan", "bu", "td_queue"],
                          want_parents=False)


def test_er_and_small_grid_count():
    beg, csr = gen_er_host(20000, 8.0, 4)
    g = Graph.from_csr(beg, csr)
    for s in pick_sources(beg, 6, 4):
        run_and_check(g, beg, csr, s)


def test_asymmetric_graph_never_uses_bottom_up():
    graphs = hand_graphs()
    beg, csr = graphs["directed_chain"]
    g = Graph.from_csr(beg, csr)
    r = run_and_check(g, beg, csr, 0, policy="forced", forced=["bu"])
    assert r.strategies["bu"] == 0


def test_device_generators_match_host():
    for args in [(10, 16, 3), (13, 8, 4)]:
        b, c = gen_rmat_host(*args)
        g = Graph.rmat(*args)
        gb, gc = g.download()
        assert np.array_equal(gb, b) and np.array_equal(gc, c)
    b, c = gen_grid_host(37, 19)
    gb, gc = Graph.grid(37, 19).download()
    assert np.array_equal(gb, b) and np.array_equal(gc, c)
    b, c = gen_er_host(4000, 8.0, 2)
    gb, gc = Graph.er(4000, 8.0, 2).download()
    assert np.array_equal(gb, b) and np.array_equal(gc, c)


def test_device_output_buffers_and_reuse():
    import torch
    beg, csr = gen_rmat_host(13, 16, 8)
    g = Graph.from_csr(beg, csr)
    lv = torch.empty(g.V, dtype=torch.int32, device="cuda:0")
    pa = torch.empty(g.V, dtype=torch.int32, device="cuda:0")
    for s in pick_sources(beg, 5, 8):
        g.bfs(int(s), levels=lv, parents=pa)
        torch.cuda.synchronize()
        ref = oracle.bfs_queue(beg, csr, s)
        assert np.array_equal(lv.cpu().numpy(), ref)
        assert oracle.check_tree(beg, csr, s, ref, pa.cpu().numpy()) == 0


def test_heuristic_trace_matches_reference_schedule():
    beg, csr = gen_rmat_host(16, 16, 21)
    g = Graph.from_csr(beg, csr)
    for s in pick_sources(beg, 6, 21):
        r = g.bfs(int(s), trace=True)
        ref = oracle.bfs_queue(beg, csr, s)
        tags = oracle.reference_schedule(beg, ref, 0.1)
        mine = [t["strategy"] for t in r.trace][: len(tags)]
        expect = ["bu" if t == -1 else ("td_scan" if t == 1 else "td_queue") for t in tags]
        assert mine == expect
        assert all(t["us"] >= 0 for t in r.trace)
        assert [t["n_f"] for t in r.trace] == [int((ref == L).sum()) for L in range(len(r.trace))]


def test_invalid_arguments():
    beg, csr = gen_rmat_host(8, 4, 1)
    g = Graph.from_csr(beg, csr)
    with pytest.raises(XbfsError) as e:
        g.bfs(g.V)
    assert e.value.status == _lib.XBFS_ERR_INVALID_ARG
    with pytest.raises(XbfsError) as e:
        g.bfs(0, padding=2)
    assert e.value.status == _lib.XBFS_ERR_INVALID_ARG
    with pytest.raises(XbfsError):
        g.bfs(0, policy="forced", forced=[])


def test_load_file_pair_and_malformed_inputs(tmp_path):
    from xbfs_b200 import write_csr
    beg, csr = gen_rmat_host(11, 8, 6)
    write_csr(beg, csr, str(tmp_path / "g_beg_pos.bin"), str(tmp_path / "g_csr.bin"))
    g = Graph.load(str(tmp_path / "g_beg_pos.bin"), str(tmp_path / "g_csr.bin"))
    assert g.V == len(beg) - 1 and g.E == len(csr)
    s = int(pick_sources(beg, 1, 6)[0])
    run_and_check(g, beg, csr, s)
    # non-monotone offsets
    bad = beg.copy()
    bad[5], bad[6] = bad[6] + 1, bad[5]
    write_csr(bad, csr, str(tmp_path / "b_beg.bin"), str(tmp_path / "b_csr.bin"))
    with pytest.raises(XbfsError) as e:
        Graph.load(str(tmp_path / "b_beg.bin"), str(tmp_path / "b_csr.bin"))
    assert e.value.status == _lib.XBFS_ERR_FORMAT
    # out-of-range neighbour
    badc = csr.copy()
    badc[7] = len(beg) + 5
    write_csr(beg, badc, str(tmp_path / "c_beg.bin"), str(tmp_path / "c_csr.bin"))
    with pytest.raises(XbfsError) as e:
        Graph.load(str(tmp_path / "c_beg.bin"), str(tmp_path / "c_csr.bin"))
    assert e.value.status == _lib.XBFS_ERR_FORMAT


def _path_graph(n):
    beg = np.zeros(n + 1, dtype=np.int64)
    deg = np.full(n, 2, dtype=np.int64)
    deg[0] = deg[-1] = 1
    beg[1:] = np.cumsum(deg)
    csr = np.empty(beg[-1], dtype=np.int32)
    for u in range(n):
        nb = [v for v in (u - 1, u + 1) if 0 <= v < n]
        csr[beg[u]:beg[u + 1]] = nb
    return beg, csr


@pytest.mark.gpu
@pytest.mark.parametrize("out,kind", [("host", "rmat"), ("device", "rmat"), ("host", "grid"), ("host", "path")])
def test_many_sources_pipelined_equal_single_calls(out, kind):
    """xbfs_bfs_many: n traversals with the level copies overlapped; every row
    equals the oracle for its source. Host rows travel as 8-bit levels (R-MAT,
    < 256 levels), 16-bit (a grid with ~500 levels) or full width (a path of
    70,000 levels)."""
    import torch
    if kind == "rmat":
        beg, csr = gen_rmat_host(15, 16, 31)
    elif kind == "grid":
        beg, csr = gen_grid_host(300, 200)
    else:
        beg, csr = _path_graph(70000)
    g = Graph.from_csr(beg, csr)
    srcs = pick_sources(beg, 7, 5) if kind != "path" else np.array([0, 69999], dtype=np.int32)
    lv = None if out == "host" else torch.empty((len(srcs), g.V), dtype=torch.int32, device="cuda:0")
    r = g.bfs_many(srcs, levels=lv)
    rows = r.levels if out == "host" else r.levels.cpu().numpy()
    mc = 0
    for i, s in enumerate(srcs):
        ref = oracle.bfs_queue(beg, csr, int(s))
        assert np.array_equal(rows[i], ref), i
        mc += oracle.edges_mc(beg, ref)
    assert r.edges_mc == mc
    g.free()


@pytest.mark.gpu
@pytest.mark.parametrize("bu_mode", [0, 1, 2, 3, 4, 5, 6])
def test_bottom_up_probe_modes(bu_mode):
    """Every bottom-up probe shape gives the oracle's levels and a valid tree
    (R-MAT with async bottom-up on and off, and a forced all-bottom-up run);
    modes 0 and 6 read the head records, the others the CSR offsets only."""
    beg, csr = gen_rmat_host(16, 16, 23)
    g = Graph.from_csr(beg, csr)
    for s in pick_sources(beg, 3, 8):
        ref = oracle.bfs_queue(beg, csr, int(s))
        for kw in ({}, {"async_bu": False}, {"policy": "forced", "forced": ["td_queue", "bu"]}):
            r = g.bfs(int(s), want_parents=True, bu_mode=bu_mode, **kw)
            assert np.array_equal(r.levels, ref), (bu_mode, kw)
            assert oracle.check_tree(beg, csr, int(s), r.levels, r.parents) == 0
    g.free()


@pytest.mark.gpu
@pytest.mark.parametrize("schedule", [["td_queue", "td_queue", "td_scan", "bu"],
                                      ["td_queue", "td_scan", "td_scan", "td_scan"],
                                      ["td_scan"]])
def test_top_down_levels_with_many_fresh_targets(schedule):
    """Top-down levels with bitmap output and many unvisited vertices mark
    their targets and finalize them after a barrier (small-bin claims may
    take some of them in the same level): levels equal the oracle's, parents
    form a valid tree, on degree-ordered R-MAT (hub frontiers) and a grid."""
    for beg, csr in (gen_rmat_host(17, 16, 5), gen_grid_host(300, 200)):
        g = Graph.from_csr(beg, csr)
        g.sort_adjacency("degree")
        b2, c2 = g.download()
        for s in pick_sources(b2, 3, 9):
            ref = oracle.bfs_queue(b2, c2, int(s))
            r = g.bfs(int(s), want_parents=True, policy="forced", forced=schedule)
            assert np.array_equal(r.levels, ref), schedule
            assert oracle.check_tree(b2, c2, int(s), r.levels, r.parents) == 0
            r2 = g.bfs(int(s), policy="forced", forced=schedule)
            assert np.array_equal(r2.levels, ref), schedule
        g.free()


@pytest.mark.gpu
@pytest.mark.parametrize("grid_dim", [1, 2, 7])
def test_few_ctas_large_shares(grid_dim):
    """With the grid capped to a few CTAs every CTA owns tens of thousands of
    vertices: bottom-up steps defer more vertices than the shared-memory queue
    holds (the rest go to the CTA's part of the list area), the warp-level
    top-down loops and the two-phase levels walk long shares; levels equal the
    oracle's and parents form a valid tree in every schedule."""
    beg, csr = gen_rmat_host(16, 16, 31)
    g = Graph.from_csr(beg, csr)
    g.sort_adjacency("degree")
    b2, c2 = g.download()
    for s in pick_sources(b2, 3, 12):
        ref = oracle.bfs_queue(b2, c2, int(s))
        for kw in ({}, {"policy": "forced", "forced": ["td_queue", "bu"]},
                   {"policy": "forced", "forced": ["td_queue", "td_queue", "td_scan", "bu", "td_scan"]}):
            for par in (True, False):
                r = g.bfs(int(s), want_parents=par, grid_dim=grid_dim, **kw)
                assert np.array_equal(r.levels, ref), (grid_dim, kw, par)
                if par:
                    assert oracle.check_tree(b2, c2, int(s), r.levels, r.parents) == 0
    g.free()


def _directed_rmat(scale, ef, seed):
    """An asymmetric CSR from an R-MAT graph: edge u->v kept when u < v or
    u + v is even (so many edges exist one way only)."""
    beg, csr = gen_rmat_host(scale, ef, seed)
    src = np.repeat(np.arange(len(beg) - 1, dtype=np.int64), np.diff(beg))
    keep = (src < csr) | (((src + csr) & 1) == 0)
    src, dst = src[keep], csr[keep]
    nb = np.zeros(len(beg), dtype=np.int64)
    np.add.at(nb, src + 1, 1)
    return np.cumsum(nb), dst.astype(np.int32)


@pytest.mark.gpu
def test_directed_power_law_top_down_paths():
    """A directed power-law CSR (bottom-up never allowed): the warp-level
    sweeps over head records, the two-phase levels (their degree counts come
    from head records, claims stay) and the queue levels (counts published,
    not taken from the bins, since a reached vertex may have no out-edge)
    give the oracle's levels and a valid tree."""
    beg, csr = _directed_rmat(15, 16, 8)
    g = Graph.from_csr(beg, csr)
    g.sort_adjacency("degree")
    b2, c2 = g.download()
    for s in pick_sources(b2, 3, 2):
        ref = oracle.bfs_queue(b2, c2, int(s))
        for kw in ({}, {"policy": "forced", "forced": ["td_queue", "td_scan"]},
                   {"policy": "forced", "forced": ["td_scan"]}):
            r = g.bfs(int(s), want_parents=True, **kw)
            assert np.array_equal(r.levels, ref), kw
            assert oracle.check_tree(b2, c2, int(s), r.levels, r.parents) == 0
            assert r.strategies["bu"] == 0
            r2 = g.bfs(int(s), **kw)
            assert np.array_equal(r2.levels, ref), kw
    g.free()


@pytest.mark.gpu
def test_bottom_up_probe_mode_out_of_range_is_refused():
    beg, csr = gen_rmat_host(10, 8, 2)
    g = Graph.from_csr(beg, csr)
    for m in (-1, 7):
        with pytest.raises(XbfsError):
            g.bfs(0, bu_mode=m)
    g.free()


@pytest.mark.gpu
@pytest.mark.parametrize("order", ["degree", "id"])
def test_head_records_follow_the_neighbour_order(order):
    """The head records are rewritten when the neighbour order changes: an
    all-bottom-up traversal after each re-order (probes start from the head
    record, scans continue at the fourth CSR entry) matches the oracle on
    the re-ordered CSR, in both word-parallel and list-based probing."""
    beg, csr = gen_rmat_host(14, 8, 77)
    g = Graph.from_csr(beg, csr)
    g.sort_adjacency("degree")
    if order == "id":
        g.sort_adjacency("id")
    b2, c2 = g.download()
    for s in pick_sources(b2, 4, 5):
        ref = oracle.bfs_queue(b2, c2, int(s))
        for mode in (0, 6):
            r = g.bfs(int(s), want_parents=True, bu_mode=mode, policy="forced", forced=["td_queue", "bu"])
            assert np.array_equal(r.levels, ref), (order, mode)
            assert oracle.check_tree(b2, c2, int(s), r.levels, r.parents) == 0
    g.free()


@pytest.mark.gpu
def test_degree_sorted_adjacency_keeps_levels():
    """xbfs_graph_sort_adjacency: segments become degree-descending
    permutations of themselves, traversal levels stay the oracle's (parents
    stay a valid tree), and sorting by id restores the generator's CSR."""
    beg, csr = gen_rmat_host(15, 16, 41)
    g = Graph.from_csr(beg, csr)
    g.sort_adjacency("degree")
    b2, c2 = g.download()
    assert np.array_equal(b2, beg)
    deg = np.diff(beg)
    for u in np.random.default_rng(0).integers(0, len(beg) - 1, size=300):
        seg, seg2 = csr[beg[u]:beg[u + 1]], c2[beg[u]:beg[u + 1]]
        assert np.array_equal(np.sort(seg), np.sort(seg2))
        assert np.all(np.diff(deg[seg2]) <= 0)
    # the same order as the oracle side builds for the reference arm (ties by id)
    assert np.array_equal(c2, oracle.sort_adjacency_degree(beg, csr))
    for s in pick_sources(beg, 4, 3):
        r = g.bfs(int(s), want_parents=True)
        assert np.array_equal(r.levels, oracle.bfs_queue(beg, csr, int(s)))
        assert oracle.check_tree(beg, csr, int(s), r.levels, r.parents) == 0
    g.sort_adjacency("id")
    assert np.array_equal(g.download()[1], csr)
    g.free()
