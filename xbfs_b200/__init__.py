"""xbfs_b200 — B200-native direction-optimising BFS (the XBFS hot path).

The product is the native library ``libxbfs.so`` (C ABI in include/xbfs.h,
kernels in csrc/); this package is its Python host-side mirror.
"""
from ._lib import (BU, TD_QUEUE, TD_SCAN, XbfsError, device_count)  # noqa: F401
from .api import (BfsOptions, BfsResult, Graph, MultiGraph, gen_er_host, gen_grid_host,  # noqa: F401
                  gen_rmat_host, pick_sources, read_csr, write_csr)

__version__ = "0.1.0"
