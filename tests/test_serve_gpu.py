"""Serving loop: requests arriving while others run join the 64-slot batches
of their graph; every result must equal the same request run alone
(xbfs_bfs) and the CPU oracle, whatever the arrival pattern, slot pressure
or HBM budget. Latencies are reported."""
import numpy as np
import pytest

import oracle
from xbfs_b200 import Graph, gen_er_host, gen_grid_host, gen_rmat_host, pick_sources
from xbfs_b200.api import Server

pytestmark = pytest.mark.gpu


def setup(seed=0):
    cpu = [gen_rmat_host(12, 16, 40 + seed), gen_rmat_host(14, 8, 41 + seed), gen_er_host(20000, 8.0, 42 + seed),
           gen_grid_host(64, 48)]
    graphs = [Graph.from_csr(b, c) for b, c in cpu]
    return cpu, graphs


def trace(cpu, n, rate_per_s, seed):
    rng = np.random.default_rng(seed)
    gid = rng.integers(0, len(cpu), size=n).astype(np.int32)
    src = np.array([pick_sources(cpu[g][0], 1, int(seed * 1000 + i))[0] for i, g in enumerate(gid)], dtype=np.int32)
    arr = np.cumsum(rng.exponential(1e6 / rate_per_s, size=n))
    return gid, src, arr


def check_all(srv, cpu, graphs, gid, src, res):
    for i, (g, s) in enumerate(zip(gid, src)):
        V = graphs[g].V
        lv = srv.fetch(res["levels_dev"][i], V)
        alone = graphs[g].bfs(int(s)).levels
        ref = oracle.bfs_queue(cpu[g][0], cpu[g][1], int(s))
        assert np.array_equal(lv, ref), f"request {i} (graph {g}, source {s}) differs in the mix"
        assert np.array_equal(alone, ref)
        assert res["edges_mc"][i] == oracle.edges_mc(cpu[g][0], ref)


@pytest.mark.parametrize("rate", [2e3, 5e4, 1e7])
def test_results_in_the_mix_equal_results_alone(rate):
    cpu, graphs = setup(0)
    gid, src, arr = trace(cpu, 150, rate, 1)
    srv = Server(graphs)
    res = srv.run(gid, src, arr, keep_outputs=True)
    assert np.all(res["finish_us"] >= res["admit_us"]) and np.all(res["admit_us"] >= arr - 1)
    print(f"rate {rate:g}/s: p50 {res['p50_us']:.0f} us, p99 {res['p99_us']:.0f} us, {res['gteps']:.2f} GTEPS")
    check_all(srv, cpu, graphs, gid, src, res)


def test_more_requests_than_slots_and_a_tight_memory_budget():
    """More than 64 requests per graph at once, and an HBM budget for three
    level arrays at a time: requests wait for slots and memory, results are
    delivered to host arrays as they finish (freeing their device memory)."""
    cpu, graphs = setup(1)
    gid, src, arr = trace(cpu, 300, 1e8, 2)   # everything arrives at once: > 64 per graph
    budget = 3 * max(g.V for g in graphs) * 4   # room for three outputs at a time
    srv = Server(graphs, hbm_budget_bytes=budget)
    res = srv.run(gid, src, arr, to_host=True)
    assert len(set(res["admit_us"].tolist())) > 1   # admission waited for memory
    for i, (g, s) in enumerate(zip(gid, src)):
        ref = oracle.bfs_queue(cpu[g][0], cpu[g][1], int(s))
        assert np.array_equal(res["levels"][i], ref), f"request {i} (graph {g}, source {s}) differs"
        assert res["edges_mc"][i] == oracle.edges_mc(cpu[g][0], ref)


def test_kept_outputs_that_fill_the_budget_are_an_error():
    """Device-kept outputs hold their memory until released: when they block
    a waiting request the run stops with XBFS_ERR_OOM instead of waiting."""
    from xbfs_b200._lib import XBFS_ERR_OOM, XbfsError
    cpu, graphs = setup(1)
    gid, src, arr = trace(cpu, 20, 1e8, 5)
    budget = 3 * max(g.V for g in graphs) * 4
    srv = Server(graphs, hbm_budget_bytes=budget)
    with pytest.raises(XbfsError) as e:
        srv.run(gid, src, arr, keep_outputs=True)
    assert e.value.status == XBFS_ERR_OOM and "fill the HBM budget" in e.value.detail


def test_run_without_keeping_outputs_reports_edges():
    cpu, graphs = setup(2)
    gid, src, arr = trace(cpu, 100, 1e5, 3)
    srv = Server(graphs)
    res = srv.run(gid, src, arr, keep_outputs=False)
    for i, (g, s) in enumerate(zip(gid, src)):
        assert res["edges_mc"][i] == oracle.edges_mc(cpu[g][0], oracle.bfs_queue(cpu[g][0], cpu[g][1], int(s)))
    assert res["p99_us"] >= res["p50_us"] > 0


def test_directed_graph_and_isolated_sources():
    """A directed CSR (bottom-up ticks are invalid there and must stay off), a
    directed R-MAT-like graph and sources without edges: every answer equals
    the oracle's."""
    from tests.conftest import hand_graphs
    hg = hand_graphs()
    beg, csr = gen_rmat_host(12, 16, 7)
    # drop the reverse of every third edge to make it directed
    keep = np.ones(len(csr), dtype=bool)
    src_of = np.repeat(np.arange(len(beg) - 1), np.diff(beg))
    keep[(src_of > csr) & (np.arange(len(csr)) % 3 == 0)] = False
    dbeg = np.concatenate([[0], np.cumsum(np.bincount(src_of[keep], minlength=len(beg) - 1))]).astype(np.int64)
    dcsr = csr[keep].astype(np.int32)
    cpu = [hg["directed_chain"], (dbeg, dcsr), hg["isolated_src"]]
    graphs = [Graph.from_csr(b, c) for b, c in cpu]
    gid = np.array([0, 1, 1, 2, 2, 1, 0], dtype=np.int32)
    src = np.array([0, 5, 17, 0, 1, 100, 3], dtype=np.int32)
    srv = Server(graphs)
    res = srv.run(gid, src, np.zeros(len(gid)), to_host=True)
    for i, (g, s) in enumerate(zip(gid, src)):
        assert np.array_equal(res["levels"][i], oracle.bfs_queue(cpu[g][0], cpu[g][1], int(s))), i


def test_staggered_joins_on_one_power_law_graph():
    """Requests on one R-MAT graph arriving a few microseconds apart join the
    batch at different ticks, so ticks where some slots have large frontiers
    (advanced bottom-up) and others small ones (advanced top-down in the same
    tick) are the common case; every answer equals the oracle's."""
    beg, csr = gen_rmat_host(15, 16, 9)
    g = Graph.from_csr(beg, csr)
    srcs = pick_sources(beg, 96, 11).astype(np.int32)
    arr = np.arange(len(srcs), dtype=np.float64) * 15.0
    srv = Server([g])
    res = srv.run(np.zeros(len(srcs), dtype=np.int32), srcs, arr, to_host=True)
    assert len(set(res["admit_us"].tolist())) > 1
    for i, s in enumerate(srcs):
        ref = oracle.bfs_queue(beg, csr, int(s))
        assert np.array_equal(res["levels"][i], ref), f"request {i} (source {s}) differs"
        assert res["edges_mc"][i] == oracle.edges_mc(beg, ref)


def test_online_submit_while_rounds_run_and_poll():
    """Online mode: requests submitted from two host threads while earlier
    ones run (the grid's traversal is hundreds of level steps long), with all
    three output modes; every answer equals the oracle's, and a trace replay
    is refused while the server runs online."""
    import threading
    import time

    from xbfs_b200._lib import XBFS_ERR_BUSY, XbfsError
    cpu, graphs = setup(3)
    cpu.append(gen_grid_host(400, 300))
    graphs.append(Graph.from_csr(*cpu[-1]))
    srv = Server(graphs)
    srv.start()
    with pytest.raises(XbfsError) as e:
        srv.run(np.zeros(1, dtype=np.int32), np.zeros(1, dtype=np.int32), np.zeros(1))
    assert e.value.status == XBFS_ERR_BUSY
    rng = np.random.default_rng(4)
    subs, lock = [], threading.Lock()

    def submitter(seed, n):
        r = np.random.default_rng(seed)
        for i in range(n):
            g = int(r.integers(0, len(graphs)))
            s = int(pick_sources(cpu[g][0], 1, seed * 100 + i)[0])
            out = ("none", "device", "host")[i % 3]
            t = srv.submit(g, s, output=out)
            with lock:
                subs.append((t, g, s, out))
            time.sleep(float(r.exponential(2e-4)))

    first = srv.submit(len(graphs) - 1, 0, output="host")   # a long traversal in flight
    subs.append((first, len(graphs) - 1, 0, "host"))
    assert srv.poll(first) is None   # still running right after submission
    ths = [threading.Thread(target=submitter, args=(k + 1, 40)) for k in range(2)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    seen_overlap = False
    for t, g, s, out in subs:
        res = srv.poll(t, wait_us=-1)
        ref = oracle.bfs_queue(cpu[g][0], cpu[g][1], s)
        assert res["edges_mc"] == oracle.edges_mc(cpu[g][0], ref), (t, g, s)
        assert res["finish_us"] >= res["admit_us"] >= res["submit_us"] - 1
        if out == "host":
            assert np.array_equal(res["levels"], ref), (t, g, s)
        elif out == "device":
            assert np.array_equal(srv.fetch(res["levels_dev"], graphs[g].V), ref), (t, g, s)
        if t != first and res["admit_us"] < srv.poll(first)["finish_us"]:
            seen_overlap = True   # admitted while the long traversal was running
    assert seen_overlap
    srv.stop()
    # after stop, a trace replay on the same server works again
    gid, src, arr = trace(cpu[:4], 20, 1e5, 9)
    res = srv.run(gid, src, arr, to_host=True)
    for i, (g, s) in enumerate(zip(gid, src)):
        assert np.array_equal(res["levels"][i], oracle.bfs_queue(cpu[g][0], cpu[g][1], int(s)))
    srv.free()
