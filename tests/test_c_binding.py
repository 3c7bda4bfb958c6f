"""The C ABI used from plain C (no GPU needed): a C99 program includes
include/xbfs.h, links libxbfs.so and calls the host-only entry points
(version, options, error strings, host generation and the CSR writer), the
way a C caller of the reference's interface would switch over."""
import os
import subprocess

import numpy as np

from xbfs_b200 import read_csr

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROG = r"""
#include <stdio.h>
#include <stdlib.h>
#include "xbfs.h"
int main(int argc, char** argv) {
  xbfs_opts o;
  xbfs_opts_init(&o);
  if (o.struct_size != (int32_t)sizeof(xbfs_opts) || o.policy != XBFS_POLICY_HEURISTIC) return 2;
  if (xbfs_version() <= 0) return 3;
  if (!xbfs_strerror(XBFS_ERR_FORMAT)) return 4;
  int64_t *beg = NULL, V = 0, E = 0;
  int32_t* csr = NULL;
  if (xbfs_gen_rmat_host(10, 8, 3, 0.57, 0.19, 0.19, &beg, &csr, &V, &E) != XBFS_OK) return 5;
  FILE* fb = fopen(argv[1], "wb");
  FILE* fc = fopen(argv[2], "wb");
  fwrite(beg, 8, (size_t)V + 1, fb);
  fwrite(csr, 4, (size_t)E, fc);
  fclose(fb);
  fclose(fc);
  printf("%lld %lld\n", (long long)V, (long long)E);
  xbfs_free_host(beg);
  xbfs_free_host(csr);
  return 0;
}
"""


def test_c_program_against_the_header_and_library(tmp_path):
    src = tmp_path / "caller.c"
    src.write_text(PROG)
    exe = tmp_path / "caller"
    lib_dir = os.path.join(ROOT, "xbfs_b200")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe), "-L", lib_dir, "-lxbfs", "-Wl,-rpath," + lib_dir], check=True)
    bp, cp = tmp_path / "g_beg_pos.bin", tmp_path / "g_csr.bin"
    r = subprocess.run([str(exe), str(bp), str(cp)], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stderr)
    V, E = map(int, r.stdout.split())
    beg, csr = read_csr(str(bp), str(cp))
    assert len(beg) == V + 1 and len(csr) == E and beg[-1] == E
    assert np.all(np.diff(beg) >= 0) and csr.min() >= 0 and csr.max() < V
