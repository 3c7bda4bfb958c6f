"""In-tree build of the native library and the `bfs` command line.

Compiles every ``csrc/*.cu`` for sm_100a with nvcc into ``xbfs_b200/libxbfs.so``
and links ``xbfs_b200/bin/bfs`` (the reference-compatible command line,
``csrc/bfs_cli.cpp``) against it. Objects go to ``_build/`` at the repository
root; a source is recompiled only when it or a header changed.

Usage: ``python xbfs_b200/build.py [-j N] [--force] [--ptxas-v]`` (run by path: importing
the package loads the library this script builds).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(ROOT, "_build", "xbfs")
LIB = os.path.join(PKG, "libxbfs.so")
CLI = os.path.join(PKG, "bin", "bfs")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp", "-Xcompiler", "-O3",
    "-I" + INCLUDE, "-I" + CSRC,
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers() -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, obj: str, extra: list[str]) -> tuple[str, int, str]:
    cmd = [nvcc()] + NVCC_FLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return src, r.returncode, (r.stdout + r.stderr)


def build(jobs: int | None = None, force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    """Build libxbfs.so and bin/bfs; returns the library path."""
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    heads = _headers()
    todo = []
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if force or _stale(o, [s] + heads):
            todo.append((s, o))
    extra = ["-Xptxas", "-v"] if ptxas_v else []
    if todo:
        jobs = jobs or min(len(todo), os.cpu_count() or 4)
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            futs = [ex.submit(_compile, s, o, extra) for s, o in todo]
            errors = []
            for f in cf.as_completed(futs):
                src, rc, out = f.result()
                if rc != 0:
                    errors.append(f"--- {src}\n{out}")
                elif verbose or ptxas_v:
                    sys.stderr.write(out)
            if errors:
                raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    if force or todo or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + [
            "-Xcompiler", "-fopenmp", "-lgomp", "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    for cli_name, exe in (("bfs_cli.cpp", CLI), ("text_to_bin_cli.cpp", os.path.join(PKG, "bin", "text_to_bin"))):
        cli_src = os.path.join(CSRC, cli_name)
        if os.path.exists(cli_src) and (force or _stale(exe, [cli_src, LIB] + heads)):
            cmd = ["g++", "-O2", "-std=c++17", "-I" + INCLUDE, cli_src, "-o", exe,
                   "-L" + PKG, "-lxbfs", "-Wl,-rpath,$ORIGIN/.."]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"{cli_name} link failed:\n" + r.stdout + r.stderr)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register/smem usage per kernel")
    a = ap.parse_args()
    print(build(a.j, a.force, a.v, a.ptxas_v))


if __name__ == "__main__":
    main()
