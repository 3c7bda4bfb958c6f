"""Generates tests/golden/ref_levels.npz: level arrays produced by the
reference's own GPU BFS (BFS_ControlFlow of hpda-lab/XBFS, built from the
reference sources by oracle/Makefile into oracle/_ref/xbfs_ref_harness) on
small graphs, for pinning the CPU oracle and the new kernels.

Needs a GPU and the prebuilt harness; run on the GPU machine:
    python tests/golden/make_golden.py --out <dir>
then copy <dir>/ref_levels.npz into tests/golden/.

Each entry stores the graph (CSR), the sources, the reference's levels per
source, and the reference's per-level strategy tags (0 scan-free/last-phase
top-down, 1 single-scan top-down, -1 bottom-up). Cases the harness refuses
(its safety gate, see oracle/ref_harness.cu) are recorded as skipped.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import REF_HARNESS  # noqa: E402
from tests.conftest import hand_graphs  # noqa: E402
from xbfs_b200 import gen_er_host, gen_grid_host, gen_rmat_host, pick_sources, write_csr  # noqa: E402


def cases():
    hg = hand_graphs()
    for name in ("path", "star32", "star33", "star256", "star257", "two_components", "isolated_src",
                 "dup_and_loops", "hub_tail"):
        beg, csr = hg[name]
        n = len(beg) - 1
        yield name, beg, csr, sorted({1 % n, n // 2, n - 1})
    for scale, ef, seed in ((10, 16, 1), (11, 8, 2), (12, 16, 3), (13, 32, 4)):
        beg, csr = gen_rmat_host(scale, ef, seed)
        yield f"rmat_s{scale}_ef{ef}_seed{seed}", beg, csr, pick_sources(beg, 4, seed).tolist()
    beg, csr = gen_er_host(3000, 8.0, 5)
    yield "er_3000", beg, csr, pick_sources(beg, 4, 5).tolist()
    beg, csr = gen_grid_host(24, 20)
    yield "grid_24x20", beg, csr, [0, 250, 479]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--harness", default=REF_HARNESS)
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    arrays, meta = {}, {}
    with tempfile.TemporaryDirectory() as td:
        for name, beg, csr, srcs in cases():
            bp, cp = os.path.join(td, name + "_beg_pos.bin"), os.path.join(td, name + "_csr.bin")
            write_csr(beg, csr, bp, cp)
            lv_all, tags_all, info = [], [], []
            for s in srcs:
                outp = os.path.join(td, f"{name}_{s}.lv")
                r = subprocess.run([a.harness, bp, cp, str(s), outp], capture_output=True, text=True, timeout=120)
                line = r.stderr.strip().splitlines()[-1] if r.stderr.strip() else "{}"
                try:
                    j = json.loads(line)
                except json.JSONDecodeError:
                    j = {"raw": line}
                j["rc"] = r.returncode
                info.append(j)
                if r.returncode == 0:
                    lv_all.append(np.fromfile(outp, dtype="<i4"))
                    tags_all.append(j.get("tags", []))
                else:
                    lv_all.append(np.full(len(beg) - 1, -2, dtype=np.int32))
                    tags_all.append([])
                print(name, s, json.dumps(j)[:200], flush=True)
            arrays[f"{name}__beg"] = beg
            arrays[f"{name}__csr"] = csr
            arrays[f"{name}__srcs"] = np.asarray(srcs, dtype=np.int32)
            arrays[f"{name}__levels"] = np.stack(lv_all)
            meta[name] = {"info": info, "tags": tags_all}
    arrays["__meta__"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(a.out, "ref_levels.npz"), **arrays)
    print("wrote", os.path.join(a.out, "ref_levels.npz"))


if __name__ == "__main__":
    main()
