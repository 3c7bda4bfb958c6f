"""The reference-compatible `bfs` command line (xbfs_b200/bin/bfs): the
reference's 11 positional arguments (bfs_gpu_update.cu:33-48), its timing
line appended to <results> ("workload;td_s;bu_s;total_s",
bfs_gpu_update.cu:282-285), and the added --out / --parents dumps.

CPU tests cover the argument contract (refusals happen before any device
work); the GPU test runs a traversal from a written file pair and compares
the dumped levels with the oracle and the parents with the tree check."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from xbfs_b200 import gen_grid_host, gen_rmat_host, pick_sources, write_csr

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BFS = os.path.join(ROOT, "xbfs_b200", "bin", "bfs")


def run(args, **kw):
    return subprocess.run([BFS] + [str(a) for a in args], capture_output=True, text=True, timeout=600, **kw)


def ref_args(beg_p, csr_p, results, src, padding=1, gpu=0, alpha=0.1, grid=256, workload="graph"):
    # beg csr weight BlockDim GridDim gpu_id results alpha src workload padding
    return [beg_p, csr_p, "x", 256, grid, gpu, results, alpha, src, workload, padding]


def test_wrong_argument_count_is_refused():
    for args in ([], ["a"] * 10, ["a"] * 12):
        r = run(args)
        assert r.returncode == 255 and "Wrong input" in r.stdout   # the reference returns -1


def test_padding_other_than_one_is_refused_before_device_work(tmp_path):
    r = run(ref_args(tmp_path / "missing_beg.bin", tmp_path / "missing_csr.bin", tmp_path / "r.csv", 0, padding=2))
    assert r.returncode == 2 and "padding = 2" in r.stderr
    assert not (tmp_path / "r.csv").exists()


def test_bad_flags_are_refused(tmp_path):
    base = ref_args(tmp_path / "b", tmp_path / "c", tmp_path / "r.csv", 0)
    r = run(base + ["--forced", "td_queue,sideways"])
    assert r.returncode == 2 and "unknown strategy" in r.stderr
    r = run(base + ["--policy", "psychic"])
    assert r.returncode != 0
    r = run(base + ["--out"])
    assert r.returncode == 2 and "needs a value" in r.stderr


def test_missing_files_are_an_error_not_a_crash(tmp_path):
    r = run(ref_args(tmp_path / "none_beg.bin", tmp_path / "none_csr.bin", tmp_path / "r.csv", 0))
    assert r.returncode == 1 and "bfs:" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["rmat", "grid"])
def test_traversal_from_files_levels_parents_and_csv(tmp_path, kind):
    beg, csr = gen_rmat_host(14, 16, 3) if kind == "rmat" else gen_grid_host(200, 150)
    bp, cp = str(tmp_path / "g_beg_pos.bin"), str(tmp_path / "g_csr.bin")
    write_csr(beg, csr, bp, cp)
    results = tmp_path / "results.csv"
    for i, s in enumerate(pick_sources(beg, 3, 5)):
        lv_p, pa_p = tmp_path / f"lv{i}.bin", tmp_path / f"pa{i}.bin"
        r = run(ref_args(bp, cp, results, int(s), workload=f"{kind}{i}") + ["--out", lv_p, "--parents", pa_p])
        assert r.returncode == 0, r.stderr + r.stdout
        levels = np.fromfile(lv_p, dtype="<i4")
        parents = np.fromfile(pa_p, dtype="<i4")
        ref = oracle.bfs_queue(beg, csr, int(s))
        assert np.array_equal(levels, ref)
        assert oracle.check_tree(beg, csr, int(s), levels, parents) == 0
        assert f"Current level = {int(ref.max()) + 1}" in r.stdout
    lines = results.read_text().splitlines()
    assert len(lines) == 3
    for i, ln in enumerate(lines):
        name, td, bu, total = ln.split(";")
        assert name == f"{kind}{i}"
        assert float(td) >= 0 and float(bu) >= 0 and float(total) == pytest.approx(float(td) + float(bu), abs=2e-9)
        assert float(total) > 0


@pytest.mark.gpu
def test_policies_and_forced_schedule_from_the_command_line(tmp_path):
    beg, csr = gen_rmat_host(13, 16, 4)
    bp, cp = str(tmp_path / "g_beg_pos.bin"), str(tmp_path / "g_csr.bin")
    write_csr(beg, csr, bp, cp)
    s = int(pick_sources(beg, 1, 1)[0])
    ref = oracle.bfs_queue(beg, csr, s)
    for extra in (["--policy", "beamer"], ["--forced", "td_scan,bu,td_queue"], ["--no-async", "--trace"]):
        lv_p = tmp_path / "lv.bin"
        r = run(ref_args(bp, cp, tmp_path / "r.csv", s) + ["--out", lv_p] + extra)
        assert r.returncode == 0, r.stderr
        assert np.array_equal(np.fromfile(lv_p, dtype="<i4"), ref), extra


@pytest.mark.gpu
def test_out_of_range_source_is_an_error(tmp_path):
    beg, csr = gen_rmat_host(10, 8, 1)
    bp, cp = str(tmp_path / "g_beg_pos.bin"), str(tmp_path / "g_csr.bin")
    write_csr(beg, csr, bp, cp)
    r = run(ref_args(bp, cp, tmp_path / "r.csv", len(beg) + 5))
    assert r.returncode == 1 and "INVALID" in r.stderr.upper()
