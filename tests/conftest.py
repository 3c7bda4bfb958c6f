import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: large inputs")


def pytest_collection_modifyitems(config, items):
    # A gpu test on a machine without a device fails loudly instead of silently
    # falling back; selection is by marker (-m gpu / -m "not gpu").
    pass


@pytest.fixture(scope="session")
def lib():
    from xbfs_b200 import _lib
    return _lib


def hand_graphs():
    """Small graphs covering the reference's edge cases (degree bins 32/256,
    isolated source, components, duplicates/self-loops removed by the loader
    contract being the caller's; here they are kept to test robustness)."""
    out = {}

    def from_edges(n, edges, sym=True):
        adj = [[] for _ in range(n)]
        for u, v in edges:
            adj[u].append(v)
            if sym and u != v:
                adj[v].append(u)
        beg = np.zeros(n + 1, dtype=np.int64)
        for i in range(n):
            beg[i + 1] = beg[i] + len(adj[i])
        csr = np.array([x for a in adj for x in a], dtype=np.int32)
        return beg, csr

    out["path"] = from_edges(10, [(i, i + 1) for i in range(9)])
    out["star33"] = from_edges(34, [(0, i) for i in range(1, 34)])          # hub degree 33: medium bin
    out["star32"] = from_edges(33, [(0, i) for i in range(1, 33)])          # degree exactly 32
    out["star257"] = from_edges(258, [(0, i) for i in range(1, 258)])       # large bin
    out["star256"] = from_edges(257, [(0, i) for i in range(1, 257)])       # degree exactly 256
    out["two_components"] = from_edges(8, [(0, 1), (1, 2), (4, 5), (5, 6), (6, 7)])
    out["isolated_src"] = from_edges(5, [(1, 2), (2, 3)])                   # vertex 0 and 4 isolated
    out["single_vertex"] = (np.zeros(2, dtype=np.int64), np.zeros(0, dtype=np.int32))
    out["dup_and_loops"] = from_edges(6, [(0, 1), (0, 1), (1, 1), (1, 2), (2, 3), (3, 3), (3, 4), (4, 5)])
    # directed (asymmetric) CSR is allowed by the file format
    out["directed_chain"] = from_edges(6, [(0, 1), (1, 2), (2, 3), (3, 4), (4, 5)], sym=False)
    # hub + long tail: exercises a top-down tail after bottom-up
    edges = [(0, i) for i in range(1, 600)] + [(599 + i, 600 + i) for i in range(0, 50)]
    out["hub_tail"] = from_edges(650, edges)
    return out


@pytest.fixture(scope="session")
def graphs():
    return hand_graphs()
