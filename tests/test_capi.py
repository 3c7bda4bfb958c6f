"""The C-ABI library loads and exports every entry point include/xbfs.h
declares; host-only entry points behave (no GPU calls here)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from xbfs_b200 import _lib
from xbfs_b200._lib import XbfsError, lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(xbfs_[a-z0-9_]+)\s*\(", text))
    return names


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) > 15
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    names = declared_functions()
    unbound = sorted(n for n in names if n not in _lib.SIGNATURES)
    assert not unbound, unbound


def test_strerror_and_version():
    assert lib.xbfs_strerror(0) == b"ok"
    assert lib.xbfs_strerror(_lib.XBFS_ERR_FORMAT) == b"malformed graph"
    assert lib.xbfs_version() >= 10000


def test_opts_init_abi():
    o = _lib.Opts()
    lib.xbfs_opts_init(C.byref(o))
    assert o.struct_size == C.sizeof(_lib.Opts)
    assert abs(o.alpha - 0.1) < 1e-7 and o.padding == 1 and o.small_max == 32 and o.medium_max == 256


def test_device_count_without_gpu_is_zero_or_more():
    n = _lib.device_count()
    assert n >= 0


def test_load_reports_errors_without_exiting(tmp_path):
    h = C.c_void_p()
    st = lib.xbfs_graph_load(str(tmp_path / "missing_beg").encode(), str(tmp_path / "missing_csr").encode(), 0,
                             C.byref(h))
    assert st == _lib.XBFS_ERR_IO
    assert b"missing_beg" in lib.xbfs_last_error()
    # truncated beg file (not a multiple of 8)
    (tmp_path / "b.bin").write_bytes(b"\x00" * 12)
    (tmp_path / "c.bin").write_bytes(b"")
    st = lib.xbfs_graph_load(str(tmp_path / "b.bin").encode(), str(tmp_path / "c.bin").encode(), 0, C.byref(h))
    assert st == _lib.XBFS_ERR_FORMAT
    # csr shorter than beg_pos[V] says
    np.array([0, 2, 3], dtype="<i8").tofile(tmp_path / "b2.bin")
    np.array([1], dtype="<i4").tofile(tmp_path / "c2.bin")
    st = lib.xbfs_graph_load(str(tmp_path / "b2.bin").encode(), str(tmp_path / "c2.bin").encode(), 0, C.byref(h))
    assert st == _lib.XBFS_ERR_FORMAT


def test_null_arguments_rejected():
    assert lib.xbfs_graph_load(None, None, 0, None) == _lib.XBFS_ERR_INVALID_ARG
    assert lib.xbfs_bfs(None, 0, None, None, None, None) == _lib.XBFS_ERR_INVALID_ARG
    n = C.c_int32()
    assert lib.xbfs_last_trace(None, None, 0, C.byref(n)) == _lib.XBFS_ERR_INVALID_ARG


def test_check_raises_with_detail():
    with pytest.raises(XbfsError) as ei:
        _lib.check(lib.xbfs_graph_load(b"/nonexistent/b", b"/nonexistent/c", 0, C.byref(C.c_void_p())))
    assert ei.value.status == _lib.XBFS_ERR_IO
