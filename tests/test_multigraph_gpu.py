"""Multi-graph persistent launch: many uneven graphs (R-MAT and ER, plus
hand graphs), one source each, one launch replayed from a CUDA graph; every
graph's levels bit-exact against the CPU oracle, before and after autotuning,
for every configuration candidate, and across repeated replays."""
import numpy as np
import pytest

import oracle
from tests.conftest import hand_graphs
from xbfs_b200 import Graph, MultiGraph, gen_er_host, gen_rmat_host, pick_sources

pytestmark = pytest.mark.gpu


def make_set(seed=0, n_rmat=10, n_er=10, smax=14):
    rng = np.random.default_rng(seed)
    cpu = []
    for i in range(n_rmat):
        cpu.append(gen_rmat_host(int(rng.integers(6, smax + 1)), int(rng.integers(8, 33)), 1000 + i))
    for i in range(n_er):
        cpu.append(gen_er_host(int(rng.integers(1000, 20000)), 8.0, 2000 + i))
    for name, (b, c) in hand_graphs().items():
        if name not in ("directed_chain",):
            cpu.append((b, c))
    return cpu


def check(mg, cpu, srcs, r):
    for (beg, csr), s, lv in zip(cpu, srcs, mg.split(r.levels)):
        assert np.array_equal(lv, oracle.bfs_queue(beg, csr, int(s)))
    mc = sum(int(np.diff(b)[oracle.bfs_queue(b, c, int(s)) >= 0].sum()) // 2 for (b, c), s in zip(cpu, srcs))
    assert r.edges_mc == mc


def pick(cpu, seed):
    out = []
    for i, (b, c) in enumerate(cpu):
        deg = np.diff(b)
        out.append(int(pick_sources(b, 1, seed + i)[0]) if deg.max() > 0 else 0)
    return np.array(out, dtype=np.int32)


def test_multi_graph_levels_and_replay():
    cpu = make_set(0)
    graphs = [Graph.from_csr(b, c) for b, c in cpu]
    mg = MultiGraph(graphs)
    for rep in range(3):
        srcs = pick(cpu, 10 * rep)
        check(mg, cpu, srcs, mg.bfs(srcs))


@pytest.mark.parametrize("block", [256, 512, 1024])
@pytest.mark.parametrize("thread_max", [0, 32, 100000])
@pytest.mark.parametrize("alpha", [0.001, 4.0, 1e9])
def test_every_configuration_is_exact(block, thread_max, alpha):
    cpu = make_set(1, n_rmat=5, n_er=5, smax=12)
    mg = MultiGraph([Graph.from_csr(b, c) for b, c in cpu])
    mg.set_config(block, thread_max, alpha)
    srcs = pick(cpu, 3)
    check(mg, cpu, srcs, mg.bfs(srcs))


def test_autotune_then_run_and_device_output():
    import torch
    cpu = make_set(2)
    mg = MultiGraph([Graph.from_csr(b, c) for b, c in cpu])
    srcs = pick(cpu, 7)
    cfg = mg.tune(srcs, reps=1)
    assert cfg["block"] in (256, 512, 1024) and cfg["best_ms"] > 0
    out = torch.empty(mg.total_V, dtype=torch.int32, device="cuda:0")
    r = mg.bfs(srcs, levels=out)
    torch.cuda.synchronize()
    r.levels = out.cpu().numpy()
    check(mg, cpu, srcs, r)


def test_graph_larger_than_shared_bitmaps():
    cpu = [gen_rmat_host(19, 4, 5), gen_er_host(3000, 8.0, 1)]
    mg = MultiGraph([Graph.from_csr(b, c) for b, c in cpu])
    srcs = pick(cpu, 1)
    check(mg, cpu, srcs, mg.bfs(srcs))
