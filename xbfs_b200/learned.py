"""Learned direction/strategy switch: data collection, GPU training,
evaluation and installation of the 8 -> 32 -> 32 -> 3 MLP used by
XBFS_POLICY_MLP.

The reference chooses the per-level strategy with fixed thresholds
(bfs_adaptiveFQ_wb_async.cuh:946-1078, 1114). Here every level of a set of
training traversals is run once with each strategy from the same snapshot
(`xbfs_level_costs`, each followed by the cheapest next level, because a
strategy also decides the form of the next frontier), the cheapest is the
label, levels are weighted by what a wrong choice costs, and the network is trained
on the device by the library's own forward/backward/SGD kernels
(`xbfs_mlp_train`). The heuristic stays the fallback: without installed
weights XBFS_POLICY_MLP behaves as XBFS_POLICY_HEURISTIC. Strategies change
speed only; levels are identical under every schedule.

    python -m xbfs_b200.learned train --out xbfs_b200/switch_mlp.npz
    python -m xbfs_b200.learned eval  --weights xbfs_b200/switch_mlp.npz
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import time
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import LevelTrace, check, lib
from .api import Graph, pick_sources

N_IN, N_H, N_OUT = 8, 32, 3
N_PACKED = 16 + N_H * N_IN + N_H + N_H * N_H + N_H + N_OUT * N_H + N_OUT  # 1459
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "switch_mlp.npz")


def _flog(x: float) -> np.float32:
    return np.float32(np.log1p(max(float(x), 0.0)))


def features_from_trace(trace: list[dict]) -> np.ndarray:
    """Per-level features exactly as the traversal kernel forms them:
    log1p of n_f, m_f, n_u, m_u, level; previous strategy; log growth of the
    frontier; log1p of the frontier's mean degree."""
    out = np.zeros((len(trace), N_IN), dtype=np.float32)
    prev_s, n_prev = 0, 1
    for i, t in enumerate(trace):
        n_f, m_f = t["n_f"], t["m_f"]
        out[i] = [_flog(n_f), _flog(m_f), _flog(t["n_u"]), _flog(t["m_u"]), _flog(t["level"]),
                  np.float32(prev_s),
                  np.float32(np.log(n_f + 1.0) - np.log(n_prev + 1.0)),
                  _flog(m_f / n_f if n_f > 0 else 0.0)]
        prev_s, n_prev = t["strategy_id"], n_f
    return out


def level_costs(g: Graph, src: int, follow: int = 0, cap: int = 16384) -> tuple[list[dict], np.ndarray]:
    """Runs xbfs_level_costs; returns (trace, costs[levels, 3] in us)."""
    costs = np.zeros((cap, 3), dtype=np.float32)
    tr = (LevelTrace * cap)()
    n = C.c_int32(0)
    check(lib.xbfs_level_costs(g.handle, int(src), int(follow), cap, costs.ctypes.data, tr, C.byref(n)))
    trace = [{"level": t.level, "strategy_id": t.strategy, "n_f": t.n_f, "m_f": t.m_f, "n_u": t.n_u,
              "m_u": t.m_u, "us": t.us} for t in tr[: n.value]]
    return trace, costs[: n.value].copy()


@dataclass
class Dataset:
    feats: np.ndarray   # (N, 8) float32
    labels: np.ndarray  # (N,) int32, argmin of costs
    costs: np.ndarray   # (N, 3) us

    def __len__(self):
        return len(self.labels)


def collect(graph_specs: list[tuple], sources: int = 4, seed: int = 1, follows=(0, 1),
            device: int = 0, log=print) -> Dataset:
    feats, labels, costs = [], [], []
    for spec in graph_specs:
        g = make_graph(spec, device)
        beg = g.offsets()
        # a grid spec may carry its own source count (long-diameter grids are
        # costly to step level by level); those follow the cheapest path only
        n_src = spec[3] if spec[0] == "grid" and len(spec) > 3 else sources
        fol = follows if n_src == sources else (0,)
        for s in pick_sources(beg, n_src, seed):
            for f in fol:
                tr, c = level_costs(g, int(s), follow=f)
                if not tr:
                    continue
                feats.append(features_from_trace(tr))
                c = tie_adjusted(c)
                labels.append(np.argmin(c, axis=1).astype(np.int32))
                costs.append(c)
        log(f"collected {spec}: {sum(len(x) for x in labels)} samples so far")
        g.free()
    return Dataset(np.concatenate(feats), np.concatenate(labels), np.concatenate(costs))


def make_graph(spec: tuple, device: int = 0, sort: bool = True) -> Graph:
    """The graph of a spec, neighbours in descending degree order by default
    (the preparation the bench applies: the per-level costs the switch is
    trained on should be those of the graphs it runs on)."""
    kind = spec[0]
    if kind == "rmat":
        g = Graph.rmat(spec[1], spec[2], spec[3] if len(spec) > 3 else 1, device=device)
    elif kind == "grid":
        g = Graph.grid(spec[1], spec[2], device=device)
    elif kind == "er":
        g = Graph.er(spec[1], spec[2], spec[3] if len(spec) > 3 else 1, device=device)
    else:
        raise ValueError(spec)
    if sort:
        g.sort_adjacency("degree")
    return g


def init_weights(feats: np.ndarray, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    mean = feats.mean(axis=0).astype(np.float32)
    std = np.maximum(feats.std(axis=0), 1e-3).astype(np.float32)
    W1 = rng.normal(0, np.sqrt(2.0 / N_IN), (N_H, N_IN))
    W2 = rng.normal(0, np.sqrt(2.0 / N_H), (N_H, N_H))
    W3 = rng.normal(0, np.sqrt(1.0 / N_H), (N_OUT, N_H))
    parts = [mean, std, W1.ravel(), np.zeros(N_H), W2.ravel(), np.zeros(N_H), W3.ravel(), np.zeros(N_OUT)]
    w = np.concatenate([np.asarray(p, dtype=np.float32).ravel() for p in parts])
    assert w.size == N_PACKED == lib.xbfs_mlp_num_params()
    return w


# Stepped per-level costs of two strategies are often within the noise of
# each other (long runs of tiny top-down levels); a label picked from such a
# tie is a coin flip, and on larger graphs than the training ones the
# scan-based strategies then pay for sweeps the small graphs did not show.
# Costs are therefore compared with the scan and bottom-up strategies charged
# 10% + 1 us extra: the network leaves the queue-based top-down only where
# another strategy is clearly cheaper.
TIE_SCALE = np.array([1.0, 1.1, 1.1])
TIE_ADD_US = np.array([0.0, 1.0, 1.0])


def tie_adjusted(costs: np.ndarray) -> np.ndarray:
    return np.asarray(costs, dtype=np.float64) * TIE_SCALE + TIE_ADD_US


def regret(costs: np.ndarray) -> np.ndarray:
    """Per level: what choosing the second-cheapest strategy instead of the
    cheapest would cost (us)."""
    c = np.sort(np.asarray(costs, dtype=np.float64), axis=1)
    return c[:, 1] - c[:, 0]


def train(ds: Dataset, epochs: int = 3000, lr: float = 0.05, momentum: float = 0.9, seed: int = 0,
          device: int = 0, weighted: bool = False) -> tuple[np.ndarray, np.ndarray]:
    """Full-batch SGD on the device (the library's own kernels). With
    ``weighted``, the batch is a resample of the levels in proportion to
    their regret, so a level where the choice is worth 300 us counts more
    than one where all strategies cost the same (plain cross-entropy on the
    argmin labels would be dominated by the thousands of near-tied levels of
    long-diameter graphs)."""
    w = init_weights(ds.feats, seed)
    losses = np.zeros(epochs, dtype=np.float32)
    feats, labels = ds.feats, ds.labels
    if weighted:
        r = regret(ds.costs)
        if r.sum() > 0:
            prob = r + 0.05 * r.mean()
            prob /= prob.sum()
            idx = np.random.default_rng(seed).choice(len(r), size=max(len(r), 20000), p=prob)
            feats, labels = feats[idx], labels[idx]
    feats = np.ascontiguousarray(feats, dtype=np.float32)
    labels = np.ascontiguousarray(labels, dtype=np.int32)
    check(lib.xbfs_mlp_train(device, w.ctypes.data, feats.ctypes.data, labels.ctypes.data, len(labels), epochs,
                             lr, momentum, losses.ctypes.data))
    return w, losses


def logits(w: np.ndarray, feats: np.ndarray, device: int = 0) -> np.ndarray:
    out = np.zeros((len(feats), N_OUT), dtype=np.float32)
    f = np.ascontiguousarray(feats, dtype=np.float32)
    check(lib.xbfs_mlp_logits(device, w.ctypes.data, f.ctypes.data, len(f), out.ctypes.data))
    return out


def install(w: np.ndarray | None, device: int = 0) -> None:
    if w is None:
        check(lib.xbfs_mlp_set_weights(device, None, 0))
    else:
        w = np.ascontiguousarray(w, dtype=np.float32)
        check(lib.xbfs_mlp_set_weights(device, w.ctypes.data, w.size))


def save(path: str, w: np.ndarray, meta: dict) -> None:
    np.savez(path, weights=w, meta=np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8))


def load(path: str = DEFAULT_WEIGHTS) -> tuple[np.ndarray, dict]:
    d = np.load(path)
    return d["weights"].astype(np.float32), json.loads(bytes(d["meta"]).decode())


def evaluate(graph_specs: list[tuple], sources: int = 8, seed: int = 99, reps: int = 3, device: int = 0,
             policies=("heuristic", "beamer", "mlp")) -> dict:
    """Traversal time per policy (min of reps per source, kernel time),
    levels checked identical across policies."""
    import torch
    res = {}
    for spec in graph_specs:
        g = make_graph(spec, device)
        beg = g.offsets()
        lv = {p: torch.empty(g.V, dtype=torch.int32, device=f"cuda:{device}") for p in policies}
        per = {p: [] for p in policies}
        mc = 0
        for s in pick_sources(beg, sources, seed):
            for p in policies:
                best = 1e30
                for _ in range(reps):
                    r = g.bfs(int(s), levels=lv[p], policy=p)
                    best = min(best, r.kernel_ms)
                per[p].append(best)
                if p == policies[0]:
                    mc += r.edges_mc
            torch.cuda.synchronize()
            for p in policies[1:]:
                if not torch.equal(lv[p], lv[policies[0]]):
                    raise AssertionError(f"levels differ between policies on {spec} source {s}")
        res[str(spec)] = {p: {"ms": float(np.sum(per[p])), "gteps": mc / (np.sum(per[p]) * 1e-3) / 1e9}
                          for p in policies}
        g.free()
    return res


TRAIN_SET = [("rmat", 16, 16, 11), ("rmat", 18, 8, 12), ("rmat", 19, 32, 13), ("rmat", 20, 16, 14),
             ("rmat", 21, 32, 15), ("rmat", 22, 16, 16), ("rmat", 20, 8, 21), ("rmat", 22, 32, 22),
             ("er", 200000, 8.0, 17), ("er", 2000000, 16.0, 18), ("er", 1000000, 8.0, 19),
             ("er", 3000000, 4.0, 20), ("er", 6000000, 8.0, 23),
             ("grid", 512, 512), ("grid", 1024, 256), ("grid", 2048, 1024, 1)]
EVAL_SET = [("rmat", 23, 32, 1), ("rmat", 22, 16, 1), ("grid", 1024, 1024), ("er", 4000000, 8.0, 3)]


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train", "eval"])
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--weights", default=DEFAULT_WEIGHTS)
    ap.add_argument("--sources", type=int, default=6)
    ap.add_argument("--epochs", type=int, default=3000)
    ap.add_argument("--report", default=None)
    a = ap.parse_args()
    if a.cmd == "train":
        t0 = time.time()
        ds = collect(TRAIN_SET, sources=a.sources)
        w, losses = train(ds, epochs=a.epochs, weighted=True)
        pred = np.argmax(logits(w, ds.feats), axis=1)
        acc = float((pred == ds.labels).mean())
        chosen = ds.costs[np.arange(len(ds)), pred].sum()
        best = ds.costs.min(axis=1).sum()
        meta = {"samples": len(ds), "epochs": a.epochs, "final_loss": float(losses[-1]), "train_accuracy": acc,
                "labels": "argmin of (level + cheapest next level) device time, scan/bottom-up +10% +1 us; regret-weighted",
                "train_cost_ratio_vs_oracle": float(chosen / best), "label_counts": np.bincount(ds.labels, minlength=3).tolist(),
                "train_set": [list(map(str, s)) for s in TRAIN_SET], "seconds": time.time() - t0}
        save(a.out, w, meta)
        print(json.dumps(meta))
    else:
        w, meta = load(a.weights)
        install(w)
        res = evaluate(EVAL_SET)
        print(json.dumps(res, indent=1))
        if a.report:
            with open(a.report, "w") as f:
                json.dump({"meta": meta, "eval": res}, f, indent=1)


if __name__ == "__main__":
    main()
