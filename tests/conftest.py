"""Shared fixtures. GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run with -m gpu)")


@pytest.fixture(scope="session")
def eb():
    import enterprise_b200
    enterprise_b200.lib()
    return enterprise_b200


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()
    return oracle


def hand_graphs():
    """Small hand-made undirected graphs as (name, V, edge list)."""
    out = []
    out.append(("path8", 8, [(i, i + 1) for i in range(7)]))
    out.append(("star9", 9, [(0, i) for i in range(1, 9)]))
    out.append(("cycle10", 10, [(i, (i + 1) % 10) for i in range(10)]))
    out.append(("two_components", 12, [(0, 1), (1, 2), (2, 3), (5, 6), (6, 7), (7, 5), (8, 9)]))
    out.append(("isolated_tail", 7, [(0, 1), (1, 2)]))
    # self loops and duplicate edges in the input list (removed by the builder)
    out.append(("loops_dups", 6, [(0, 0), (0, 1), (1, 0), (0, 1), (1, 2), (2, 2), (2, 3), (3, 4), (4, 5), (5, 5)]))
    out.append(("complete6", 6, [(i, j) for i in range(6) for j in range(i + 1, 6)]))
    return out


def tier_graph(seed=7):
    """Hits every degree tier: a hub of degree > 1024, mid-degree vertices
    (32..1024) and small ones (< 32), plus a long tail path (many levels)."""
    rng = np.random.default_rng(seed)
    V = 6000
    edges = []
    for v in range(1, 3000):  # hub 0 with degree 2999
        edges.append((0, v))
    for h in range(3000, 3040):  # 40 mid vertices of degree ~100
        for v in rng.choice(np.arange(3040, 5000), size=100, replace=False):
            edges.append((h, int(v)))
        edges.append((h, int(rng.integers(1, 3000))))
    for v in range(3040, 5000):  # small
        edges.append((v, int(rng.integers(3040, 5000))))
    for v in range(5000, 5999):  # tail path off vertex 4999
        edges.append((v, v + 1))
    edges.append((4999, 5000))
    e = np.array(edges, dtype=np.int64)
    return V, e[:, 0], e[:, 1]
