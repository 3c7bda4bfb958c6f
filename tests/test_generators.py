"""Host generators: format contract (symmetric, no self-loops, no duplicates,
sorted adjacency, int64/int32), determinism, and grid closed form. CPU only."""
import os

import numpy as np
import pytest

from xbfs_b200 import gen_er_host, gen_grid_host, gen_rmat_host, pick_sources, read_csr, write_csr


def check_csr_contract(beg, csr):
    V = len(beg) - 1
    assert beg.dtype == np.int64 and csr.dtype == np.int32
    assert beg[0] == 0 and beg[-1] == len(csr)
    assert np.all(np.diff(beg) >= 0)
    assert csr.min(initial=0) >= 0 and csr.max(initial=0) < V
    src = np.repeat(np.arange(V, dtype=np.int64), np.diff(beg))
    assert not np.any(src == csr), "self-loop"
    key = src * V + csr
    assert np.all(np.diff(key) > 0), "unsorted or duplicate adjacency"
    rev = csr.astype(np.int64) * V + src
    assert np.array_equal(np.sort(rev), key), "not symmetric"


@pytest.mark.parametrize("scale,ef", [(6, 4), (10, 16), (12, 8)])
def test_rmat_contract_and_determinism(scale, ef):
    b1, c1 = gen_rmat_host(scale, ef, 42)
    check_csr_contract(b1, c1)
    b2, c2 = gen_rmat_host(scale, ef, 42)
    assert np.array_equal(b1, b2) and np.array_equal(c1, c2)
    b3, c3 = gen_rmat_host(scale, ef, 43)
    assert not (len(c1) == len(c3) and np.array_equal(c1, c3))
    assert len(b1) == (1 << scale) + 1
    # skew: R-MAT has a heavy-tailed degree distribution
    deg = np.diff(b1)
    assert deg.max() > 4 * deg.mean()


def test_er_contract():
    b, c = gen_er_host(3000, 8.0, 9)
    check_csr_contract(b, c)
    assert abs(len(c) / 3000 - 8.0) < 0.5


def test_grid_closed_form():
    for W, H in [(1, 1), (1, 7), (5, 1), (4, 3), (64, 64)]:
        b, c = gen_grid_host(W, H)
        check_csr_contract(b, c)
        assert len(c) == 2 * (W - 1) * H + 2 * W * (H - 1)
    b, c = gen_grid_host(4096, 4096)
    assert len(c) == 67_092_480


def test_pick_sources_non_isolated_distinct():
    b, c = gen_rmat_host(12, 4, 1)
    s = pick_sources(b, 64, 5)
    deg = np.diff(b)
    assert len(set(s.tolist())) == 64
    assert np.all(deg[s] > 0)
    assert np.array_equal(s, pick_sources(b, 64, 5))


def test_file_roundtrip(tmp_path):
    b, c = gen_rmat_host(8, 8, 3)
    write_csr(b, c, str(tmp_path / "g_beg_pos.bin"), str(tmp_path / "g_csr.bin"))
    assert os.path.getsize(tmp_path / "g_beg_pos.bin") == 8 * len(b)
    assert os.path.getsize(tmp_path / "g_csr.bin") == 4 * len(c)
    b2, c2 = read_csr(str(tmp_path / "g_beg_pos.bin"), str(tmp_path / "g_csr.bin"))
    assert np.array_equal(b, b2) and np.array_equal(c, c2)


@pytest.mark.parametrize("scale,ef,seed", [(6, 4, 1), (10, 16, 2), (13, 32, 3), (16, 16, 4), (18, 8, 5)])
def test_oracle_side_generator_builds_the_same_rmat(scale, ef, seed):
    """The reference arm of bench.py builds its graph and sources with the
    oracle's own generator (oracle/gen.c: per-vertex buckets, not the
    library's key sort); both builds must give the same CSR and sources."""
    import oracle
    b1, c1 = oracle.gen_rmat(scale, ef, seed)
    b2, c2 = gen_rmat_host(scale, ef, seed)
    assert np.array_equal(b1, b2) and np.array_equal(c1, c2)
    check_csr_contract(b1, c1)
    assert np.array_equal(oracle.pick_sources(b1, 64, seed), pick_sources(b2, 64, seed))


def test_oracle_side_generator_builds_the_same_grid():
    import oracle
    for W, H in [(1, 1), (1, 7), (5, 1), (4, 3), (300, 200)]:
        b1, c1 = oracle.gen_grid(W, H)
        b2, c2 = gen_grid_host(W, H)
        assert np.array_equal(b1, b2) and np.array_equal(c1, c2)
