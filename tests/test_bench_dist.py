"""The N>1 path of bench.py on CPU: world_size-2 ``gloo`` ranks. The
traversal itself needs a GPU; what is checked here is the host side of the
replica scaling — per-rank sources, the job-wide figure (all ranks' edges
over the slowest rank's time) and that only rank 0 prints — and that the
reference arm under torchrun runs on rank 0 alone."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench
    from xbfs_b200 import gen_rmat_host, pick_sources
    w, r, _ = bench.dist_init("gloo")
    beg, _ = gen_rmat_host(10, 8, 1)
    srcs = pick_sources(beg, 4, 1 + r).tolist()        # as run_ours picks them
    edges = [1000.0, 3000.0][r]
    secs = [0.002, 0.004][r]
    gteps, tot, mx = bench.job_rate(edges, secs, w)
    dist.barrier()
    q.put((r, srcs, gteps, tot, mx))
    dist.destroy_process_group()


def test_job_rate_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, s0, g0, t0, m0), (_, s1, g1, t1, m1) = out
    assert t0 == t1 == 4000.0 and m0 == m1 == 0.004
    assert g0 == g1 == pytest.approx(4000.0 / 0.004 / 1e9)
    assert s0 != s1  # each replica traverses its own sources


def test_single_rank_job_rate_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    g, tot, mx = bench.job_rate(500, 0.001, 1)
    assert (g, tot, mx) == (500 / 0.001 / 1e9, 500.0, 0.001)


def test_reference_arm_under_torchrun_prints_once():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "3", "--warmup", "1", "--scale", "12", "--ef", "8",
           "--sources", "4"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] in ("port", "reference") and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["config"]["workload"] == "rmat-s12-ef8 single-source BFS" and d["config"]["sources"] == 4
    assert set(d["config"]) == {"workload", "V", "E", "sources", "policy", "seed", "adjacency", "l2", "parallelism"}
    assert "reference_gpu" in d


def test_reference_arm_loads_no_product_library():
    """The reference arm builds its graph and sources with the oracle's own
    generator: libxbfs.so must not be mapped into its process."""
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--scale', '12', '--ef', '8', "
            "'--steps', '2', '--warmup', '1', '--sources', '4', '--no-reference-gpu']; "
            "runpy.run_path('bench.py', run_name='__main__'); "
            "print('MAPPED', any('libxbfs' in l for l in open('/proc/self/maps')))")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, cwd=ROOT,
                       env=dict(os.environ, CUDA_VISIBLE_DEVICES=""))
    assert r.returncode == 0, r.stderr[-2000:]
    assert "MAPPED False" in r.stdout
    d = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][0])
    assert d["config"]["E"] > 0 and d["config"]["policy"] == "heuristic" and "reference_gpu" not in d
