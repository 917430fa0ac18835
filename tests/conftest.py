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


def big_root_graph(nbig=1100, core=4, extra_p=0.0, seed=0):
    """A graph whose first roots have local subgraphs of more than 1024 vertices.

    C = {0, ..., core-1} is a clique; each of the nbig vertices S = {core, ...,
    core+nbig-1} is adjacent to all of C (and, with extra_p > 0, to other S
    vertices at random with that probability); R = core+nbig is adjacent to all
    of C.  R has the smallest degree and, inserted last, leaves the degeneracy
    order first (its bucket is LIFO), so R's local subgraph is R, C1 = C and
    C2 = S: 1 + core + nbig vertices.  The S vertices that follow each S
    vertex in the order are its C2, so about nbig - 1019 roots exceed 1024
    vertices.

    With core = 4, extra_p = 0, k = 2 and q = 6 the maximal 2-plexes are
    exactly {R} + C + {v} for v in S and C + {v, w} for v != w in S (S is
    independent, so a 2-plex holds at most two S vertices, and R misses every
    S vertex): big_root_expected gives their count and hash."""
    import numpy as np
    rng = np.random.default_rng(seed)
    n = core + nbig + 1
    R = core + nbig
    S = np.arange(core, core + nbig)
    rows = [set() for _ in range(n)]
    for a in range(core):
        rows[a].update(b for b in range(core) if b != a)
        rows[a].update(S.tolist())
        rows[a].add(R)
        rows[R].add(a)
    for v in S:
        rows[v].update(range(core))
    if extra_p > 0:
        iu, iw = np.triu_indices(nbig, 1)
        keep = rng.random(len(iu)) < extra_p
        for a, b in zip(S[iu[keep]], S[iw[keep]]):
            rows[a].add(int(b))
            rows[b].add(int(a))
    off = np.zeros(n + 1, np.uint32)
    off[1:] = np.cumsum([len(r) for r in rows])
    adj = np.concatenate([sorted(r) for r in rows]).astype(np.uint32)
    return off, adj


def oversized_root_graph(nclique=1100, nroot=1000, nouter=1100):
    """A root whose 2-hop subgraph exceeds MAX_LOCAL = 2048 vertices: root 0 is
    adjacent to nroot members of a nclique-clique A, and nouter vertices B are
    adjacent to all of A.  Root 0 has the smallest degree, so it leaves the
    degeneracy order first; C1 = its nroot neighbours and C2 = the rest of A
    and all of B: 1 + nclique + nouter local vertices."""
    import numpy as np
    A = np.arange(1, 1 + nclique)
    B = np.arange(1 + nclique, 1 + nclique + nouter)
    n = 1 + nclique + nouter
    ia, ib = np.triu_indices(nclique, 1)
    s = np.concatenate([np.zeros(nroot, np.int64), A[ia], np.repeat(A, nouter)])
    d = np.concatenate([A[:nroot], A[ib], np.tile(B, nclique)])
    u = np.concatenate([s, d])
    v = np.concatenate([d, s])
    order = np.lexsort((v, u))
    u, v = u[order], v[order]
    off = np.zeros(n + 1, np.uint32)
    off[1:] = np.cumsum(np.bincount(u, minlength=n))
    return off, v.astype(np.uint32)


def _splitmix64(z):
    import numpy as np
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def plex_hash_sum(sets):
    """The project hash (kplex_common.h) of an array of sorted vertex sets, one per row."""
    import numpy as np
    sets = np.asarray(sets, dtype=np.uint64)
    x = _splitmix64(np.full(sets.shape[0], 0x6B706C6578B200 ^ sets.shape[1], dtype=np.uint64))
    for c in range(sets.shape[1]):
        x = _splitmix64(x ^ sets[:, c])
    with np.errstate(over="ignore"):
        return int(np.sum(x, dtype=np.uint64))


def big_root_expected(nbig=1100):
    """Count and hash of big_root_graph(nbig) at k = 2, q = 6, derived by hand."""
    import numpy as np
    S = np.arange(4, 4 + nbig, dtype=np.uint64)
    R = 4 + nbig
    c = np.tile(np.arange(4, dtype=np.uint64), (nbig, 1))
    with_r = np.column_stack([c, S, np.full(nbig, R, np.uint64)])
    iv, iw = np.triu_indices(nbig, 1)
    pairs = np.column_stack([np.tile(np.arange(4, dtype=np.uint64), (len(iv), 1)), S[iv], S[iw]])
    h = (plex_hash_sum(with_r) + plex_hash_sum(pairs)) % (1 << 64)
    return {"count": nbig + nbig * (nbig - 1) // 2, "hash": h}


def dense_request_graph():
    """1,101 vertices, about 480,000 edges: root 0 adjacent to 550 of a 600-clique A,
    and 500 vertices B adjacent to all of A.  Root 0's local subgraph has
    1 + 550 + 550 vertices; a request whose device estimate is far above the
    small batched graphs'."""
    import numpy as np
    A = np.arange(1, 601)
    B = np.arange(601, 1101)
    n = 1101
    ia, ib = np.triu_indices(600, 1)
    s = np.concatenate([np.zeros(550, np.int64), A[ia], np.repeat(A, 500)])
    d = np.concatenate([A[:550], A[ib], np.tile(B, 600)])
    u = np.concatenate([s, d])
    v = np.concatenate([d, s])
    order = np.lexsort((v, u))
    u, v = u[order], v[order]
    off = np.zeros(n + 1, np.uint32)
    off[1:] = np.cumsum(np.bincount(u, minlength=n))
    return off, v.astype(np.uint32)
