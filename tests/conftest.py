"""Shared fixtures.  GPU tests carry @pytest.mark.gpu and call through the C ABI."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "maximal-kplex-enumeration_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

DATASETS = os.path.join(ROOT, "datasets")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) device")
    config.addinivalue_line("markers", "slow: minutes of CPU time; run with KPLEX_SLOW=1")


def pytest_collection_modifyitems(config, items):
    if os.environ.get("KPLEX_SLOW") == "1":
        return
    skip = pytest.mark.skip(reason="slow oracle pin; set KPLEX_SLOW=1")
    for it in items:
        if "slow" in it.keywords:
            it.add_marker(skip)


def _ensure_built():
    lib = os.path.join(PKG, "libkplex.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", PKG, "-j8"], check=True)
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "-j4"], check=True)


@pytest.fixture(scope="session")
def kp():
    _ensure_built()
    import kplex_b200
    return kplex_b200


@pytest.fixture(scope="session")
def orc():
    _ensure_built()
    import oracle
    return oracle


def dataset(name):
    p = os.path.join(DATASETS, name)
    return p if os.path.exists(p) else None


def big_left_graph(nl=1500, nt=8, nr=5, seed=7):
    """A graph whose roots carry left sets above 1024 vertices.

    Root R (degree nr) is adjacent to nr members of an nt-clique T; nl
    degree-3 vertices L each join 3 members of T (four fifths of them inside
    R's part of T) and nothing else.  The L vertices precede R in the
    degeneracy order, so with k=2, q=4 about 1500 of them pass the 2-hop left
    filter (>= q-2k+3 = 3 neighbours in C1) for root R, while every local
    subgraph stays below 1024 vertices."""
    import numpy as np
    rng = np.random.default_rng(seed)
    R, T, l0 = 0, list(range(1, 1 + nt)), 1 + nt
    edges = set()
    for i in range(nt):
        for j in range(i + 1, nt):
            edges.add((T[i], T[j]))
    for t in T[:nr]:
        edges.add((R, t))
    for i in range(nl):
        part = T[:nr] if i < nl * 4 // 5 else T
        for t in rng.choice(part, 3, replace=False):
            edges.add((int(t), l0 + i))
    n = l0 + nl
    rows = [[] for _ in range(n)]
    for a, b in edges:
        rows[a].append(b)
        rows[b].append(a)
    off = np.zeros(n + 1, np.uint32)
    off[1:] = np.cumsum([len(r) for r in rows])
    adj = np.concatenate([sorted(r) for r in rows]).astype(np.uint32)
    return off, adj
