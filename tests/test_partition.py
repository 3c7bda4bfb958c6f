"""1D-partitioned multi-GPU BFS (xbfs_b200/partition.py). The exchange
logic runs on world-size 2 and 3 ``gloo`` ranks on the CPU with a numpy
stand-in for the device steps; the device steps (xbfs_part_* kernels) run
on one GPU, as one rank and as ranks emulated by threads of one process
(the ranks' kernels never wait on each other: every exchange is a host
collective between launches). Levels are compared with the CPU oracle."""
import os
import socket
import sys
import threading

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import oracle
from xbfs_b200 import gen_grid_host, gen_rmat_host, pick_sources
from xbfs_b200.partition import bounds, local_rows, partitioned_bfs, slice_words

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def graph(kind):
    if kind == "rmat":
        return gen_rmat_host(12, 16, 5), True
    if kind == "grid":
        return gen_grid_host(70, 50), True
    beg, csr = gen_rmat_host(11, 8, 6)   # directed: drop the reverse of every third edge
    V = len(beg) - 1
    src_of = np.repeat(np.arange(V), np.diff(beg))
    keep = ~((src_of > csr) & (np.arange(len(csr)) % 3 == 0))
    dbeg = np.concatenate([[0], np.cumsum(np.bincount(src_of[keep], minlength=V))]).astype(np.int64)
    return (dbeg, csr[keep].astype(np.int32)), False


def test_bounds_tile_the_vertex_range_in_whole_words():
    for V in (1, 31, 32, 33, 1000, 4096, 100003):
        for world in (1, 2, 3, 8):
            b = bounds(V, world)
            assert b[0] == 0 and b[-1] == V and all(x <= y for x, y in zip(b, b[1:]))
            assert all(x % 32 == 0 or x == V for x in b[:-1])   # empty trailing slices start at V
            W = slice_words(V, world)
            assert all(y - x <= 32 * W for x, y in zip(b, b[1:]))
            assert W * world * 32 >= V


def _rank(rank, world, port, kind, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    from tests.partition_engine import NumpyEngine
    from xbfs_b200.partition import TorchComm
    dist.init_process_group("gloo", rank=rank, world_size=world)
    (beg, csr), sym = graph(kind)
    V = len(beg) - 1
    b = bounds(V, world)
    bl, cl = local_rows(beg, csr, b[rank], b[rank + 1])
    eng = NumpyEngine(bl, cl, V, b[rank], b[rank + 1], sym)
    comm = TorchComm()
    out = []
    for s in pick_sources(beg, 3, 2):
        r = partitioned_bfs(eng, comm, int(s), symmetric=sym, alpha=2.0, beta=24.0)
        out.append((int(s), r.levels, r.depth, r.strategies))
    q.put((rank, b[rank], out))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("kind", ["rmat", "grid", "directed"])
def test_gloo_ranks_give_the_oracle_levels(world, kind):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, kind, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (beg, csr), sym = graph(kind)
    for k in range(3):
        s = res[0][2][k][0]
        full = np.concatenate([r[2][k][1] for r in res])
        assert np.array_equal(full, oracle.bfs_queue(beg, csr, s)), (kind, world, s)
        scheds = {tuple(r[2][k][3]) for r in res}
        assert len(scheds) == 1   # every rank took the same steps
        if kind != "directed" and kind == "rmat":
            assert "bu" in next(iter(scheds))   # both exchanges were used
        if kind == "directed":
            assert "bu" not in next(iter(scheds))


class ThreadComm:
    """Ranks emulated by threads of one process: the collectives meet at a
    barrier and combine on the host. Test infrastructure."""

    def __init__(self, world):
        self.world = world
        self.bar = threading.Barrier(world)
        self.slots = [None] * world

    def view(self, rank):
        outer = self

        class V:
            world = outer.world

            def sum(self_, vals, like):
                outer.slots[rank] = list(vals)
                outer.bar.wait()
                tot = [sum(x) for x in zip(*outer.slots)]
                outer.bar.wait()
                return tot

            def max_bytes(self_, t):
                torch.cuda.synchronize()
                outer.slots[rank] = t
                outer.bar.wait()
                if rank == 0:
                    m = outer.slots[0].clone()
                    for o in outer.slots[1:]:
                        torch.maximum(m, o, out=m)
                    outer.result = m
                outer.bar.wait()
                t.copy_(outer.result)
                torch.cuda.synchronize()
                outer.bar.wait()

            def gather_words(self_, out, mine):
                torch.cuda.synchronize()
                outer.slots[rank] = mine
                outer.bar.wait()
                out.copy_(torch.cat(outer.slots))
                torch.cuda.synchronize()
                outer.bar.wait()
        return V()


@pytest.mark.gpu
@pytest.mark.parametrize("world", [1, 2, 3])
@pytest.mark.parametrize("kind", ["rmat", "grid", "directed"])
def test_device_steps_on_one_gpu(world, kind):
    from xbfs_b200.partition import DeviceEngine
    (beg, csr), sym = graph(kind)
    V = len(beg) - 1
    b = bounds(V, world)
    engines = [DeviceEngine(*local_rows(beg, csr, b[r], b[r + 1]), V, b[r], b[r + 1], sym) for r in range(world)]
    comm = ThreadComm(world)
    for s in pick_sources(beg, 3, 4):
        out = [None] * world

        def run(r):
            out[r] = partitioned_bfs(engines[r], comm.view(r), int(s), symmetric=sym, alpha=2.0)
        ths = [threading.Thread(target=run, args=(r,)) for r in range(world)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        full = np.concatenate([o.levels for o in out])
        assert np.array_equal(full, oracle.bfs_queue(beg, csr, int(s))), (kind, world, int(s))
    for e in engines:
        e.free()
