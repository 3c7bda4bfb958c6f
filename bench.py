#!/usr/bin/env python
"""Benchmark: single-source BFS (the XBFS hot path) on one or more B200s.

Default workload: Graph500 R-MAT scale 23, edge factor 32 (a=.57 b=.19
c=.19, symmetrised, deduplicated, seeded), 64 sources drawn uniformly from
non-isolated vertices; a step is one BFS from one source (sources cycle).
Metric: GTEPS (Graph500 m_c / time), with the achieved HBM GB/s of the
traversal kernel in ``roofline``.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

``--impl reference`` times the reference's own CPU BFS (the level-synchronous
sweep of bfs_gpu_update.cu:105-127, restated in oracle/ and run with all host
threads) on the same graph and sources. Multi-GPU runs are replicas (every
rank traverses its own copy of the graph from its own sources; no exchange).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GTEPS + HBM GB/s at R-MAT s23 on 1 B200; batched/learned vs plain; serve p99"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=256)
    ap.add_argument("--warmup", type=int, default=8)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["rmat", "grid"], default="rmat")
    ap.add_argument("--scale", type=int, default=23)
    ap.add_argument("--ef", type=int, default=32)
    ap.add_argument("--grid-w", type=int, default=4096)
    ap.add_argument("--grid-h", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--sources", type=int, default=64)
    ap.add_argument("--policy", default="heuristic")
    ap.add_argument("--adjacency", choices=["degree", "file"], default="degree",
                    help="neighbour order prepared before timing: descending neighbour degree (default) or as "
                         "generated (ascending ids); levels are the same either way")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-flush", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=32)
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="budget of the cpu_baseline sample")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="reference arm: skip timing the reference's own GPU BFS beside its CPU BFS")
    ap.add_argument("--reference-gpu-sources", type=int, default=4)
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle check of the timed rows")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the learned / batched / multi-graph / serving comparison sections")
    return ap.parse_args()


# ---------------------------------------------------------------------------
class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while running."""

    REASONS = {
        "hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
        "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80, "sync_boost": 0x10,
    }

    def __init__(self, device: int, period_s: float = 0.0005):
        self.device, self.period = device, period_s
        self.samples: list[tuple[int, int]] = []
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.samples.append((mhz, rs, time.perf_counter()))
            except Exception:
                pass
            time.sleep(self.period)

    def __enter__(self):
        if self.nv:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join()

    def summary(self, t0: float | None = None, t1: float | None = None) -> dict:
        """Samples taken in [t0, t1] (perf_counter seconds; all when None)."""
        sel = [x for x in self.samples if (t0 is None or x[2] >= t0) and (t1 is None or x[2] <= t1)]
        if not sel:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0}
        mask = 0
        for x in sel:
            mask |= x[1]
        reasons = [k for k, v in self.REASONS.items() if mask & v]
        return {"sm_mhz": statistics.median(x[0] for x in sel), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(sel)}


def peak_hbm() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(workload_tag: str):
    """dram bytes per launch of the traversal kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", f"k_bfs_{workload_tag}.txt")
    try:
        for line in open(p):
            if line.startswith("dram_bytes_per_launch:"):
                return float(line.split(":")[1].split()[0])
    except Exception:
        pass
    return None


# ---------------------------------------------------------------------------
def dist_init(backend: str = "nccl"):
    """One process per GPU under torchrun; the process group only carries the
    scalar reductions of the job-wide figures (no data-path collective: every
    rank traverses its own replica of the graph). ``gloo`` serves CPU tests."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def allreduce(vals, op):
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor(vals, dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return t.tolist()


def job_rate(edges: float, my_seconds: float, world: int):
    """Whole-job GTEPS of independent replicas: the edges of all ranks over the
    slowest rank's time. Returns (gteps, total edges, max seconds)."""
    if world > 1:
        import torch.distributed as dist
        edges, = allreduce([float(edges)], dist.ReduceOp.SUM)
        my_seconds, = allreduce([float(my_seconds)], dist.ReduceOp.MAX)
    return float(edges) / my_seconds / 1e9, float(edges), float(my_seconds)


def barrier(world):
    import torch
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()


def make_graph(args, device):
    from xbfs_b200 import Graph
    if args.workload == "rmat":
        g = Graph.rmat(args.scale, args.ef, args.seed, device=device)
        name = f"rmat-s{args.scale}-ef{args.ef}"
    else:
        g = Graph.grid(args.grid_w, args.grid_h, device=device)
        name = f"grid-{args.grid_w}x{args.grid_h}"
    return g, name


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_sample(beg, csr, srcs, budget_s, kind="serial"):
    """A CPU BFS of the oracle on a bounded sample of sources: the serial FIFO
    BFS ("serial") or the OpenMP direction-optimising BFS on all host threads
    ("openmp"). Returns (GTEPS, sources done, seconds, threads)."""
    import oracle
    threads = len(os.sched_getaffinity(0)) if kind == "openmp" else 1
    done, edges, t_total = [], 0, 0.0
    for s in srcs:
        t0 = time.perf_counter()
        lv = oracle.bfs_queue(beg, csr, s) if kind == "serial" else oracle.bfs_do(beg, csr, s, threads)
        t_total += time.perf_counter() - t0
        edges += oracle.edges_mc(beg, lv)
        done.append(int(s))
        if t_total > budget_s:
            break
    return edges / t_total / 1e9, done, t_total, threads


def check_parity(g, beg, par_src, par_rows, e2e_par, world):
    """Level rows the timed region and the e2e leg produced, compared with
    the OpenMP oracle (and the serial FIFO oracle on the first source) on the
    same graph. Every rank checks its own rows; counts are summed."""
    import oracle
    _, csr = g.download()
    cache = {}

    def ref(s):
        if s not in cache:
            cache[s] = oracle.bfs_do(beg, csr, s)
        return cache[s]
    checked = mism = 0
    for s, row in list(zip(par_src, par_rows if par_rows is not None else [])) + list(e2e_par):
        checked += 1
        mism += int(not np.array_equal(row, ref(s)))
    if par_src:
        checked += 1
        mism += int(not np.array_equal(par_rows[0], oracle.bfs_queue(beg, csr, par_src[0])))
    del csr
    if world > 1:
        import torch.distributed as dist
        checked, mism = allreduce([float(checked), float(mism)], dist.ReduceOp.SUM)
    return {"checked": int(checked), "mismatches": int(mism),
            "rows": "levels of the last timed chunk (up to 16 sources) and of the first e2e host rows",
            "oracle": "OpenMP direction-optimising BFS per source, plus the serial FIFO BFS on the first"}


# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist

    from xbfs_b200 import BfsOptions, pick_sources
    world, rank, local = dist_init()
    torch.cuda.set_device(local)
    dev = local
    g, wname = make_graph(args, dev)
    V, E = g.V, g.E
    if args.adjacency == "degree":
        # graph preparation, untimed: hubs first in every neighbour list, so
        # bottom-up probes find a frontier parent sooner (levels unchanged)
        g.sort_adjacency("degree")
    beg = g.offsets()
    srcs = pick_sources(beg, args.sources, args.seed + rank)
    # a dedicated stream: the library launches on it, and the events, the L2
    # flush and the output tensor all live on it too
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    opts = BfsOptions(policy=args.policy, stream=stream.cuda_stream)
    lv = torch.empty(V, dtype=torch.int32, device="cuda")
    # L2 flush between steps (untimed): write a 256 MB buffer (> 126 MB L2),
    # then read another one so the dirty lines are written back before the
    # next timed step instead of inside it.
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    flush_rd = torch.ones(64 << 20, dtype=torch.int32, device="cuda")

    def step(i, timed_events=None):
        if not args.no_flush:
            flush.fill_(i & 0xFF)
            flush_rd.sum()
        if timed_events is not None:
            timed_events[0].record(stream)
        r = g.bfs(int(srcs[i % len(srcs)]), levels=lv, opts=opts)
        if timed_events is not None:
            timed_events[1].record(stream)
        return r

    # ---- timed region: args.steps traversals back to back on the device
    # (xbfs_bfs_many, level rows in HBM, no host round trip between steps);
    # the CSR (2 GB at scale 23) is far larger than the 126 MB L2
    chunk = min(64, args.steps)
    rows = torch.empty((chunk, V), dtype=torch.int32, device="cuda")
    plan = [np.array([srcs[(i0 + j) % len(srcs)] for j in range(min(chunk, args.steps - i0))], dtype=np.int32)
            for i0 in range(0, args.steps, chunk)]
    # clocks are sampled from the warm-up through the per-call figures below
    # (the GPU is busy throughout); the line reports the timed region's
    # samples and those of the whole busy window
    clk = ClockSampler(dev).__enter__()
    for i in range(args.warmup):
        g.bfs_many(np.array([srcs[i % len(srcs)]], dtype=np.int32), levels=rows[:1], opts=opts)
    barrier(world)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    edges, strat = 0, {"td_queue": 0, "td_scan": 0, "bu": 0}
    t_wall0 = time.perf_counter()
    ev0.record(stream)
    for src_chunk in plan:
        r = g.bfs_many(src_chunk, levels=rows[:len(src_chunk)], opts=opts)
        edges += r.edges_mc
        for k in strat:
            strat[k] += r.strategies[k]
    ev1.record(stream)
    barrier(world)
    t_wall1 = time.perf_counter()
    t_wall = t_wall1 - t_wall0
    value, tot_edges, max_s = job_rate(edges, ev0.elapsed_time(ev1) * 1e-3, world)
    max_ms = max_s * 1e3
    # level rows of the last timed chunk, kept for the oracle check below
    n_par = 0 if args.no_parity else min(16, len(plan[-1]))
    par_src = [int(x) for x in plan[-1][:n_par]]
    par_rows = rows[:n_par].cpu().numpy() if n_par else None
    # the same timed path on the neighbour order as generated, for reference
    file_order = None
    if args.adjacency == "degree":
        g.sort_adjacency("id")
        g.bfs_many(plan[0][:2], levels=rows[:2], opts=opts)
        fe0, fe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        fedges = 0
        fe0.record(stream)
        for src_chunk in plan:
            fedges += g.bfs_many(src_chunk, levels=rows[:len(src_chunk)], opts=opts).edges_mc
        fe1.record(stream)
        torch.cuda.synchronize()
        fms = fe0.elapsed_time(fe1)
        file_order = {"gteps": round(fedges / (fms * 1e-3) / 1e9, 3), "ms_per_step": round(fms / args.steps, 5),
                      "note": "same sources and timed path, neighbours in generator order"}
        g.sort_adjacency("degree")
    del rows

    # ---- one xbfs_bfs call per step with the L2 flushed before each (the
    # traversal kernel's own duration, for the roofline)
    pc_steps = min(args.steps, 64)
    for i in range(3):
        step(i)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(pc_steps)]
    results = [step(3 + i, evs[i]) for i in range(pc_steps)]
    torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    kernel_ms = [r.kernel_ms for r in results]
    clk.__exit__()
    pc_gteps = sum(r.edges_mc for r in results) / (sum(step_ms) * 1e-3) / 1e9

    # ---- end to end through the public API with host buffers
    e2e = None
    e2e_par = []
    if not args.no_e2e:
        # xbfs_bfs_many: one public call for all e2e steps, each step's int32[V]
        # level array copied to pinned host memory while the next traversal runs
        nstep = args.e2e_steps
        host_rows = torch.empty((nstep, V), dtype=torch.int32, pin_memory=True).numpy()
        e_src = np.array([srcs[i % len(srcs)] for i in range(nstep)], dtype=np.int32)
        g.bfs_many(e_src[:2], levels=host_rows[:2], opts=opts)
        barrier(world)
        t0 = time.perf_counter()
        r = g.bfs_many(e_src, levels=host_rows, opts=opts)
        barrier(world)
        e_gteps, _, _ = job_rate(r.edges_mc, time.perf_counter() - t0, world)
        e2e_par = [(int(e_src[i]), host_rows[i].copy()) for i in range(min(4, nstep))] if not args.no_parity else []
        single = host_rows[0]
        t1 = time.perf_counter()
        e1 = 0
        for i in range(min(nstep, 16)):
            e1 += g.bfs(int(e_src[i]), levels=single, opts=opts).edges_mc
        t1 = time.perf_counter() - t1
        e2e = {"value": round(e_gteps, 3), "unit": "GTEPS",
               "h2d_bytes_per_step": 4, "d2h_bytes_per_step": 4 * V,
               "note": f"xbfs_bfs_many over {nstep} sources into pinned host memory: per step the source id "
                       "goes host to device and the int32[V] level array device to host, the copy of step i "
                       "overlapping the traversal of step i+1; graph resident in HBM",
               "one_call_per_source_gteps": round(e1 / t1 / 1e9, 3)}
        del host_rows

    # ---- roofline of the traversal kernel
    b_alg = 8 * (V + 1) + 4 * E + 4 * V
    mean_k = statistics.mean(kernel_ms)
    achieved = b_alg / (mean_k * 1e-3) / 1e9
    peak, peak_kind = peak_hbm()
    tag = f"rmat_s{args.scale}_ef{args.ef}" if args.workload == "rmat" else f"grid_{args.grid_w}x{args.grid_h}"
    traffic = ncu_traffic(tag)
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": peak_kind,
                "kernel": "k_bfs (persistent cooperative level loop)",
                "algorithmic_bytes_per_launch": b_alg,
                "mean_launch_ms": round(mean_k, 5)}
    if traffic:
        # what DRAM actually moved per launch (ncu) over the same launch time
        roofline["dram_gbs_ncu"] = round(traffic / (mean_k * 1e-3) / 1e9, 1)
        roofline["dram_frac_ncu"] = round(traffic / (mean_k * 1e-3) / 1e9 / peak, 4)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        _, csr = g.download()
        gteps, done, secs, _ = cpu_sample(beg, csr, srcs, args.cpu_seconds)
        cpu = {"value": round(gteps, 4), "unit": "GTEPS", "cores": 1, "kind": "port",
               "sample": f"serial FIFO BFS (oracle) from {len(done)} of the {len(srcs)} sources, {secs:.1f} s"}
        og, odone, osecs, othr = cpu_sample(beg, csr, srcs, args.cpu_seconds / 3, kind="openmp")
        cpu["openmp_do_bfs"] = {"value": round(og, 4), "unit": "GTEPS", "cores": othr,
                                "cpu": cpu_model(),
                                "sample": f"OpenMP direction-optimising BFS (oracle) from {len(odone)} sources, "
                                          f"{osecs:.1f} s"}
        del csr
    parity = None
    if not args.no_parity:
        parity = check_parity(g, beg, par_src, par_rows, e2e_par, world)
    del par_rows
    depth = statistics.median(r.depth for r in results)
    out = {
        "metric": METRIC, "value": round(value, 3), "unit": "GTEPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(max_ms / args.steps, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded Graph500 R-MAT generated on the device)" if args.workload == "rmat"
        else "synthetic (2D 4-neighbour grid)",
        "config": workload_config(args, V, E, len(srcs), world),
        "timed_region": "xbfs_bfs_many over the steps' sources, level rows in HBM; the per-call figures flush "
                        "L2 (256 MB write + 256 MB read, untimed) before each call",
        "median_depth": depth, "levels_by_strategy": strat, "parity": parity,
        "adjacency_generator_order": file_order,
        "per_call_l2_flushed": {"gteps": round(pc_gteps, 3), "steps": pc_steps,
                                "ms_per_step": round(sum(step_ms) / pc_steps, 5),
                                "kernel_ms_mean": round(statistics.mean(kernel_ms), 5)},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
        # one k_bfs launch per traversal (it sets up its own state); the
        # control blocks are zeroed by one memset per xbfs_bfs_many call
        "clocks": dict(clk.summary(t_wall0, t_wall1), busy_window=clk.summary()), "gpu_launches": args.steps,
        "wall_s_timed_region": round(t_wall, 4),
        "hbm_gbs_algorithmic_per_step": round(b_alg * args.steps / (max_ms * 1e-3) / 1e9, 1),
    }
    if not args.no_extras and args.workload == "rmat":
        out["learned"] = extra_learned(args, g, srcs, opts, lv, stream, flush, flush_rd, value)
        out["batched_same_graph"] = extra_batched_same_graph(args, g, beg, value, wname)
        g.free()
        g = None
        torch.cuda.empty_cache()
        out["batched"] = extra_batched(args, value)
        out["multi_graph"] = extra_multigraph(args)
        out["serve"] = extra_serve(args)
    if world > 1:
        # every rank ran the same sections; report the job-wide sums / maxima
        for key in ("learned", "batched", "multi_graph"):
            sec = out.get(key)
            if isinstance(sec, dict) and "gteps" in sec:
                tot, = allreduce([float(sec["gteps"])], dist.ReduceOp.SUM)
                sec["gteps_all_ranks"] = round(tot, 3)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if g is not None:
        g.free()
    if world > 1:
        dist.destroy_process_group()


def _timed_steps(fn, steps):
    import torch
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    res = []
    for i in range(steps):
        res.append(fn(i, evs[i]))
    torch.cuda.synchronize()
    return res, [a.elapsed_time(b) for a, b in evs]


def extra_learned(args, g, srcs, opts, lv, stream, flush, flush_rd, plain_gteps):
    """Same graph and sources with the learned switch (shipped weights)."""
    from xbfs_b200 import learned
    path = learned.DEFAULT_WEIGHTS
    if not os.path.exists(path):
        return {"unavailable": "no trained weights shipped"}
    w, meta = learned.load(path)
    learned.install(w, device=g.device)
    import dataclasses
    o2 = dataclasses.replace(opts, policy="mlp")
    beamer = dataclasses.replace(opts, policy="beamer")

    import torch
    plan = np.array(srcs[:64], dtype=np.int32)
    rows = torch.empty((len(plan), g.V), dtype=torch.int32, device="cuda")

    def run(o):
        # the timed region of the plain form: back-to-back traversals, rows in HBM
        g.bfs_many(plan[:2], levels=rows[:2], opts=o)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = g.bfs_many(plan, levels=rows, opts=o)
        e1.record(stream)
        torch.cuda.synchronize()
        return r.edges_mc / (e0.elapsed_time(e1) * 1e-3) / 1e9
    g_plain = run(opts)
    g_mlp = run(o2)
    g_beamer = run(beamer)
    del rows
    out = {"gteps": round(g_mlp, 3), "policy": "mlp", "vs_plain": round(g_mlp / g_plain, 4),
           "plain_same_sources_gteps": round(g_plain, 3), "beamer_gteps": round(g_beamer, 3),
           "train_meta": {k: meta[k] for k in ("samples", "train_accuracy")}}
    # the second graph of the comparison: the 4096 x 4096 grid (diameter ~8190)
    import torch
    from xbfs_b200 import BfsOptions, Graph, pick_sources
    gg = Graph.grid(4096, 4096, device=g.device)
    gsrc = pick_sources(gg.offsets(), 4, args.seed)
    glv = torch.empty(gg.V, dtype=torch.int32, device="cuda")
    per = {}
    for pol in ("heuristic", "mlp", "beamer"):
        go = BfsOptions(policy=pol, stream=stream.cuda_stream)
        gg.bfs(int(gsrc[0]), levels=glv, opts=go)
        ms, mc = 0.0, 0
        for s_ in gsrc:
            r = gg.bfs(int(s_), levels=glv, opts=go)
            ms += r.kernel_ms
            mc += r.edges_mc
        per[pol] = {"gteps": round(mc / (ms * 1e-3) / 1e9, 4), "ms_per_source": round(ms / len(gsrc), 3)}
    out["grid-4096x4096"] = dict(per, mlp_vs_plain=round(per["heuristic"]["ms_per_source"] /
                                                         per["mlp"]["ms_per_source"], 4))
    del glv
    gg.free()
    learned.install(None, device=g.device)
    return out


def batched_roofline(V, E, n, ms):
    """Batched algorithmic bytes: one pass over the CSR pair per group of 64
    sources plus the n int32[V] level rows, over the device time."""
    groups = (n + 63) // 64
    b_alg = groups * (8 * (V + 1) + 4 * E) + 4 * V * n
    peak, peak_kind = peak_hbm()
    ach = b_alg / (ms * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4),
            "peak_source": peak_kind, "algorithmic_bytes_per_call": b_alg,
            "kernel": "ms::k_msbfs + ms::k_ms_transpose (device time of the call)"}


def extra_batched_same_graph(args, g, beg, plain_gteps, wname):
    """512 sources in one batched pass (8 uint64 words per vertex) on the
    bench's own graph, against the plain form's timed value on it."""
    import torch
    from xbfs_b200 import pick_sources
    srcs = pick_sources(beg, 512, args.seed + 7)
    out = torch.empty((512, g.V), dtype=torch.int32, device="cuda")
    best = None
    for _ in range(3):
        r = g.bfs_batch(srcs, levels=out)
        if best is None or r.device_ms < best.device_ms:
            best = r
    del out
    torch.cuda.empty_cache()
    gteps = best.edges_mc / (best.device_ms * 1e-3) / 1e9
    return {"workload": f"{wname}, 512 sources", "gteps": round(gteps, 3), "ms": round(best.device_ms, 3),
            "vs_plain": round(gteps / plain_gteps, 3), "roofline": batched_roofline(g.V, g.E, 512, best.device_ms)}


def extra_batched(args, plain_ref):
    """512 sources on R-MAT scale 22 ef16 (8 groups of 64 per uint64 word) vs
    single-source on the same graph; outputs are n x V int32 in HBM."""
    import torch
    from xbfs_b200 import Graph, pick_sources
    g = Graph.rmat(22, 16, args.seed)
    beg = g.offsets()
    srcs = pick_sources(beg, 512, args.seed)
    out = torch.empty((512, g.V), dtype=torch.int32, device="cuda")
    g.bfs_batch(srcs, levels=out)  # warm-up
    best = None
    for _ in range(3):
        r = g.bfs_batch(srcs, levels=out)
        if best is None or r.device_ms < best.device_ms:
            best = r
    lv = torch.empty(g.V, dtype=torch.int32, device="cuda")
    ms, mc = 0.0, 0
    for s in srcs[:64]:
        r1 = g.bfs(int(s), levels=lv)
        ms += r1.kernel_ms
        mc += r1.edges_mc
    single = mc / (ms * 1e-3) / 1e9
    res = {"workload": "rmat-s22-ef16, 512 sources", "gteps": round(best.edges_mc / (best.device_ms * 1e-3) / 1e9, 3),
           "ms": round(best.device_ms, 3), "single_source_gteps_same_graph": round(single, 3)}
    res["vs_single_source"] = round(res["gteps"] / single, 3)
    res["roofline"] = batched_roofline(g.V, g.E, 512, best.device_ms)
    del out
    g.free()
    torch.cuda.empty_cache()
    return res


def extra_multigraph(args):
    """256 uneven graphs (128 R-MAT scale 10..18 ef 8..32 + 128 ER n 1e3..2e5,
    mean degree 8), one source each, one persistent launch replayed from a
    CUDA graph, configuration picked by the autotuner; vs one xbfs_bfs call
    per graph."""
    import torch
    from xbfs_b200 import Graph, MultiGraph, pick_sources
    rng = np.random.default_rng(args.seed)
    graphs = [Graph.rmat(int(rng.integers(10, 19)), int(rng.integers(8, 33)), 100 + i) for i in range(128)]
    graphs += [Graph.er(int(rng.integers(1000, 200001)), 8.0, 300 + i) for i in range(128)]
    srcs = np.array([int(pick_sources(g.offsets(), 1, 7 + i)[0]) for i, g in enumerate(graphs)], dtype=np.int32)
    mg = MultiGraph(graphs)
    cfg = mg.tune(srcs, reps=2)
    out = torch.empty(mg.total_V, dtype=torch.int32, device="cuda")
    best = min((mg.bfs(srcs, levels=out) for _ in range(5)), key=lambda r: r.device_ms)
    t_one, mc1 = 0.0, 0
    for g, s in zip(graphs, srcs):
        r = g.bfs(int(s))
        t_one += r.device_ms
        mc1 += r.edges_mc
    b_alg = sum(8 * (g.V + 1) + 4 * g.E + 4 * g.V for g in graphs)
    peak, peak_kind = peak_hbm()
    ach = b_alg / (best.device_ms * 1e-3) / 1e9
    res = {"workload": "256 graphs (128 R-MAT s10-18, 128 ER 1e3-2e5)", "gteps": round(best.edges_mc / (best.device_ms * 1e-3) / 1e9, 3),
           "roofline": {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                        "frac": round(ach / peak, 4), "peak_source": peak_kind,
                        "algorithmic_bytes_per_launch": b_alg, "kernel": "mg::k_multi",
                        "note": "sum over graphs of size(beg) + size(csr) + 4V, over the device time of the "
                                "replayed launch; the whole arena (about 1.2 GB) partly fits the 126 MB L2"},
           "ms": round(best.device_ms, 3), "tuned": cfg, "one_call_per_graph_ms": round(t_one, 3),
           "speedup_vs_one_call_per_graph": round(t_one / best.device_ms, 2)}
    mg.free()
    for g in graphs:
        g.free()
    del out
    torch.cuda.empty_cache()
    return res


def extra_serve(args):
    """Serving: Poisson arrivals over 8 device-resident graphs (R-MAT scales
    20-24 ef16 and grids 2048x2048, 4096x4096, 8192x2048), continuous batching
    into 64-source slots, admission by free HBM; p50 / p99 latency and
    aggregate GTEPS per arrival rate."""
    import torch
    from xbfs_b200 import Graph, pick_sources
    from xbfs_b200.api import Server
    specs = [("rmat", s) for s in (20, 21, 22, 23, 24)] + [("grid", 2048, 2048), ("grid", 4096, 4096), ("grid", 8192, 2048)]
    graphs = [Graph.rmat(sp[1], 16, args.seed + sp[1]) if sp[0] == "rmat" else Graph.grid(sp[1], sp[2]) for sp in specs]
    begs = [g.offsets() for g in graphs]
    srv = Server(graphs)
    res = {"graphs": ["rmat-s%d-ef16" % sp[1] if sp[0] == "rmat" else "grid-%dx%d" % sp[1:] for sp in specs], "rates": []}
    rng = np.random.default_rng(args.seed)
    is_grid = np.array([sp[0] == "grid" for sp in specs])
    for rate in (1e2, 1e3, 1e4, 1e5):
        # two independent traces per rate; latencies pooled (a single trace of
        # a few hundred requests over 8 very different graphs is noisy)
        n = int(min(400, max(40, rate * 2)))
        lat, kinds, mc, wall = [], [], 0, 0.0
        for rep in range(2):
            gid = rng.integers(0, len(graphs), size=n).astype(np.int32)
            src = np.array([pick_sources(begs[gi], 1, int(rate) + 1000 * rep + i)[0] for i, gi in enumerate(gid)],
                           dtype=np.int32)
            arr = np.cumsum(rng.exponential(1e6 / rate, size=n))
            r = srv.run(gid, src, arr, keep_outputs=False)
            lat.append(r["latency_us"])
            kinds.append(is_grid[gid])
            mc += int(r["edges_mc"].sum())
            wall += r["wall_us"]
        lat, kinds = np.concatenate(lat) / 1e3, np.concatenate(kinds)
        pct = lambda a, q: round(float(np.percentile(a, q)), 3) if len(a) else None
        res["rates"].append({"rate_per_s": rate, "requests": 2 * n, "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99),
                             "rmat_p50_ms": pct(lat[~kinds], 50), "rmat_p99_ms": pct(lat[~kinds], 99),
                             "grid_p50_ms": pct(lat[kinds], 50), "grid_p99_ms": pct(lat[kinds], 99),
                             "gteps": round(mc / (wall * 1e-6) / 1e9, 3), "wall_s": round(wall / 1e6, 3)})
    srv.free()
    for g in graphs:
        g.free()
    torch.cuda.empty_cache()
    return res


def workload_config(args, V, E, n_sources, world):
    """The config block both arms print (same keys and values for the same
    command line): the workload, its sizes and seeds, and how L2 is kept out
    of the timed steps."""
    if args.workload == "rmat":
        wname = f"rmat-s{args.scale}-ef{args.ef}"
    else:
        wname = f"grid-{args.grid_w}x{args.grid_h}"
    adjacency = ("neighbours of each vertex in descending degree order (untimed preparation)"
                 if args.adjacency == "degree" else "neighbours in generator order (ascending ids)")
    return {"workload": f"{wname} single-source BFS", "V": int(V), "E": int(E), "sources": int(n_sources),
            "policy": args.policy, "seed": args.seed, "adjacency": adjacency,
            "l2": "inputs larger than L2 (CSR of E int32 entries) in the timed steps",
            "parallelism": f"replicas x{world}"}


def reference_gpu_leg(beg, csr, srcs, k, alpha=0.1):
    """The reference's own GPU BFS (BFS_ControlFlow, compiled unmodified from
    the reference sources into oracle/_ref/xbfs_ref_harness by oracle/Makefile)
    on the same graph and sources, one harness process per source. The
    harness refuses (exit 3, nothing launched) the inputs on which the
    reference has known out-of-bounds accesses. GTEPS from the reference's
    own TD/BU phase timers and from the wall time of its BFS_ControlFlow
    call (which includes its per-level host work); levels compared with the
    OpenMP oracle."""
    import subprocess
    import tempfile

    import oracle
    if not os.path.exists(oracle.REF_HARNESS):
        return {"unavailable": "oracle/_ref/xbfs_ref_harness not built (it needs the reference sources at build time)"}
    rows = []
    with tempfile.TemporaryDirectory() as d:
        bp, cp = os.path.join(d, "g_beg_pos.bin"), os.path.join(d, "g_csr.bin")
        np.ascontiguousarray(beg, dtype="<i8").tofile(bp)
        np.ascontiguousarray(csr, dtype="<i4").tofile(cp)
        for s in srcs[:k]:
            out = os.path.join(d, "lv.bin")
            try:
                r = subprocess.run([oracle.REF_HARNESS, bp, cp, str(int(s)), out, str(alpha), "256", "256"],
                                   capture_output=True, text=True, timeout=300)
            except Exception as e:  # timed out or could not start
                rows.append({"src": int(s), "error": str(e)[:200]})
                continue
            try:
                info = json.loads(r.stderr.strip().splitlines()[-1])
            except (ValueError, IndexError):  # no record: e.g. no CUDA device
                rows.append({"src": int(s), "rc": r.returncode, "error": (r.stderr + r.stdout)[-200:]})
                continue
            info["rc"] = r.returncode
            rec = {"src": int(s), "rc": info["rc"]}
            if info["rc"] == 0 and "kernel_s" in info:
                lv = np.fromfile(out, dtype="<i4")
                rec.update(kernel_s=info["kernel_s"], wall_s=info["wall_s"], depth=info.get("levels"),
                           edges_mc=oracle.edges_mc(beg, lv),
                           levels_equal_oracle=bool(np.array_equal(lv, oracle.bfs_do(beg, csr, int(s)))))
            else:
                rec["skipped"] = info.get("skipped") or info.get("error") or "no result"
            rows.append(rec)
    ok = [r for r in rows if "kernel_s" in r]
    res = {"impl": "BFS_ControlFlow of the reference, unmodified, 256 x 256, alpha 0.1, padding 1",
           "sources_tried": len(rows), "sources_timed": len(ok)}
    if ok:
        mc = sum(r["edges_mc"] for r in ok)
        res["gteps_phase_timers"] = round(mc / sum(r["kernel_s"] for r in ok) / 1e9, 3)
        res["gteps_wall"] = round(mc / sum(r["wall_s"] for r in ok) / 1e9, 4)
        res["ms_phase_timers_per_source"] = round(sum(r["kernel_s"] for r in ok) / len(ok) * 1e3, 3)
        res["all_levels_equal_oracle"] = all(r["levels_equal_oracle"] for r in ok)
    res["per_source"] = rows
    return res


def run_reference(args):
    """The reference's CPU BFS (sweep, bfs_gpu_update.cu:105-127), all host
    threads, on the same graph and sources as the other arm. The graph and
    sources come from the oracle's own generator (oracle/gen.c), so this arm
    loads no product library; the reference's GPU BFS is timed beside it."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    threads = len(os.sched_getaffinity(0))
    if args.workload == "rmat":
        beg, csr = oracle.gen_rmat(args.scale, args.ef, args.seed)
    else:
        beg, csr = oracle.gen_grid(args.grid_w, args.grid_h)
    srcs = oracle.pick_sources(beg, args.sources, args.seed)
    if args.adjacency == "degree":
        csr = oracle.sort_adjacency_degree(beg, csr)   # the same graph preparation as the other arm
    for i in range(args.warmup):
        oracle.bfs_sweep(beg, csr, srcs[i % len(srcs)], threads)
    t_total, edges = 0.0, 0
    steps = args.steps
    budget = 120.0
    done = 0
    for i in range(steps):
        s = srcs[i % len(srcs)]
        t0 = time.perf_counter()
        lv, _ = oracle.bfs_sweep(beg, csr, s, threads)
        t_total += time.perf_counter() - t0
        edges += oracle.edges_mc(beg, lv)
        done += 1
        if t_total > budget:
            break
    value = edges / t_total / 1e9
    out = {
        "metric": METRIC, "value": round(value, 4), "unit": "GTEPS", "n_gpus": world, "steps": done,
        "warmup": args.warmup, "ms_per_step": round(t_total / done * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "impl": "reference",
        "data": "synthetic (seeded Graph500 R-MAT)" if args.workload == "rmat" else "synthetic (2D 4-neighbour grid)",
        "config": workload_config(args, len(beg) - 1, int(beg[-1]), len(srcs), world),
        "timed_region": f"the reference's CPU sweep BFS (bfs_gpu_update.cu:105-127) restated, one source per step, "
                        f"{threads} threads",
        "cpu_baseline": {"value": round(value, 4), "unit": "GTEPS", "cores": threads, "kind": "port",
                         "sample": f"reference sweep BFS (bfs_gpu_update.cu:105-127) restated, {done} sources, "
                                   f"{threads} threads"},
        "e2e": {"value": round(value, 4), "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_reference_gpu:
        out["reference_gpu"] = reference_gpu_leg(beg, csr, srcs, args.reference_gpu_sources)
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
