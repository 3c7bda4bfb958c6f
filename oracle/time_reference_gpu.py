"""Times the reference's own GPU BFS (BFS_ControlFlow of hpda-lab/XBFS, built
from the reference sources by `make -C oracle ref` into
oracle/_ref/xbfs_ref_harness) beside this library's xbfs_bfs on the same
seeded R-MAT graphs and sources, on one GPU. Measurement tooling for the
reference comparison only; the library never calls it.

    python oracle/time_reference_gpu.py --scale 23 --ef 32 --sources 8

Prints one JSON line per graph: per-source reference times (its own
TD/BU phase timers summed, and the wall time of the BFS_ControlFlow call,
which includes its per-level host work) and this library's kernel and
device times, with the Graph500 edge count of each source.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import REF_HARNESS, edges_mc  # noqa: E402
from xbfs_b200 import Graph, gen_rmat_host, pick_sources, write_csr  # noqa: E402


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=int, default=16)
    ap.add_argument("--ef", type=int, default=16)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--sources", type=int, default=8)
    a = ap.parse_args()
    beg, csr = gen_rmat_host(a.scale, a.ef, a.seed)
    srcs = [int(s) for s in pick_sources(beg, a.sources, a.seed)]
    g = Graph.from_csr(beg, csr)
    rows = []
    with tempfile.TemporaryDirectory() as d:
        bp, cp = os.path.join(d, "g_beg_pos.bin"), os.path.join(d, "g_csr.bin")
        write_csr(beg, csr, bp, cp)
        for s in srcs:
            out = os.path.join(d, "lv.bin")
            r = subprocess.run([REF_HARNESS, bp, cp, str(s), out, "0.1", "256", "256"], capture_output=True,
                               text=True, timeout=1800)
            rec = {"src": s}
            try:
                info = json.loads(r.stderr.strip().splitlines()[-1])
            except (ValueError, IndexError):
                info = {"error": r.stderr[-300:]}
            rec["reference"] = info
            ours = None
            for _ in range(3):
                res = g.bfs(s)
                if ours is None or res.kernel_ms < ours.kernel_ms:
                    ours = res
            rec["ours"] = {"kernel_ms": ours.kernel_ms, "device_ms": ours.device_ms, "depth": ours.depth}
            rec["edges_mc"] = int(edges_mc(beg, ours.levels))
            if "kernel_s" in info:
                ref_lv = np.fromfile(out, dtype=np.int32)
                rec["levels_equal"] = bool(np.array_equal(ref_lv, ours.levels))
            rows.append(rec)
    g.free()
    ok = [r for r in rows if "kernel_s" in r["reference"]]
    summary = {"graph": f"rmat-s{a.scale}-ef{a.ef}", "seed": a.seed, "sources": len(rows), "compared": len(ok)}
    if ok:
        mc = sum(r["edges_mc"] for r in ok)
        summary["reference_gteps_phase_timers"] = mc / sum(r["reference"]["kernel_s"] for r in ok) / 1e9
        summary["reference_gteps_wall"] = mc / sum(r["reference"]["wall_s"] for r in ok) / 1e9
        summary["ours_gteps_kernel"] = mc / sum(r["ours"]["kernel_ms"] * 1e-3 for r in ok) / 1e9
        summary["ours_gteps_device"] = mc / sum(r["ours"]["device_ms"] * 1e-3 for r in ok) / 1e9
        summary["all_levels_equal"] = all(r.get("levels_equal") for r in ok)
    summary["per_source"] = rows
    print(json.dumps(summary), flush=True)


if __name__ == "__main__":
    main()
