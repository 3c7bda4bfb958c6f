"""Edge-list converter (replacement of CSRGenerator/tuple_text_to_bin.cpp):
the file pair it writes is the BFS reader's format (int64 offsets, int32
neighbours), with the reference converter's options (reverse, skip_lines)
plus dedupe / self-loop removal. CPU only (the GPU load is in the GPU suite)."""
import os
import subprocess

import numpy as np
import pytest

from xbfs_b200 import XbfsError, read_csr
from xbfs_b200.api import convert_edge_list

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def csr_from_pairs(pairs, n, reverse, dedupe, drop_loops):
    es = []
    for u, v in pairs:
        if drop_loops and u == v:
            continue
        es.append((u, v))
        if reverse and u != v:
            es.append((v, u))
    es.sort()
    if dedupe:
        es = sorted(set(es))
    beg = np.zeros(n + 1, dtype=np.int64)
    for u, _ in es:
        beg[u + 1] += 1
    return np.cumsum(beg), np.array([v for _, v in es], dtype=np.int32)


@pytest.mark.parametrize("reverse", [0, 1])
@pytest.mark.parametrize("dedupe", [0, 1])
@pytest.mark.parametrize("drop", [0, 1])
def test_options_match_a_direct_construction(tmp_path, reverse, dedupe, drop):
    rng = np.random.default_rng(reverse * 4 + dedupe * 2 + drop)
    pairs = [(int(a), int(b)) for a, b in rng.integers(0, 200, size=(2000, 2))] + [(5, 5), (7, 9), (7, 9)]
    text = "% matrix-market style header\n% second header line\n" + "".join(f"{u}\t{v}\n" for u, v in pairs)
    text += "# comment line\n\n"
    p = tmp_path / "g.txt"
    p.write_text(text)
    n = max(max(u, v) for u, v in pairs) + 1
    V, E = convert_edge_list(str(p), str(tmp_path / "out"), reverse=reverse, skip_lines=2, dedupe=dedupe,
                             drop_self_loops=drop)
    beg, csr = read_csr(str(tmp_path / "out_beg_pos.bin"), str(tmp_path / "out_csr.bin"))
    rb, rc = csr_from_pairs(pairs, n, reverse, dedupe, drop)
    assert V == n and E == len(rc)
    assert np.array_equal(beg, rb)
    # adjacency order within a vertex is sorted in both
    assert np.array_equal(csr, rc)
    assert os.path.getsize(tmp_path / "out_csr.bin") == 4 * E  # int32 neighbours


def test_cli_keeps_the_reference_argument_order(tmp_path):
    p = tmp_path / "edges.txt"
    p.write_text("header\n0 1\n1 2\n2 0\n3 3\n")
    exe = os.path.join(ROOT, "xbfs_b200", "bin", "text_to_bin")
    r = subprocess.run([exe, str(p), "1", "1", "8"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    beg, csr = read_csr(str(p) + "_beg_pos.bin", str(p) + "_csr.bin")
    assert beg.tolist() == [0, 2, 4, 6, 6] and csr.tolist() == [1, 2, 0, 2, 0, 1]
    r = subprocess.run([exe, str(p), "1", "1", "8", "--weights", "--out", str(tmp_path / "w")],
                       capture_output=True, text=True)
    assert r.returncode == 0
    w = np.fromfile(tmp_path / "w_weight.bin", dtype=np.int32)
    assert len(w) == 6 and w.min() >= 1 and w.max() <= 63


def test_malformed_line_is_an_error(tmp_path):
    p = tmp_path / "bad.txt"
    p.write_text("0 1\n1 x\n")
    with pytest.raises(XbfsError):
        convert_edge_list(str(p), str(tmp_path / "o"))
