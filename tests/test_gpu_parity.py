"""Device path (through the C ABI) against the oracle and the golden fixtures.

Integer work: every comparison is exact — count, the order-independent hash
of the sorted vertex sets, and the number of generated tasks (the device
builds the same search tree as the oracle)."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, dataset

pytestmark = pytest.mark.gpu


def golden():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)


def test_small_workload(kp, orc):
    w = kp.WORKLOADS["small"]
    off, adj = kp.workload_graph("small")
    g = kp.enumerate_csr(off, adj, w["k"], w["q"], w["thres"], w["truss"])
    gold = golden()["workloads"]["small"]
    assert (g["count"], g["hash"], g["tasks"]) == (gold["count"], gold["hash"], gold["tasks"])
    assert g["valid_roots"] == gold["valid_roots"] and g["pn"] == gold["pn"]
    assert g["gpu_launches"] >= 3


def test_golden_random_graphs(kp, orc):
    for c in golden()["random"]:
        off, adj = orc.random_graph(c["n"], c["p"], c["seed"], [tuple(x) for x in c["planted"]])
        g = kp.enumerate_csr(off, adj, c["k"], c["q"], truss=c["truss"])
        assert (g["count"], g["hash"], g["tasks"]) == (c["count"], c["hash"], c["tasks"]), c


@pytest.mark.parametrize("k", [2, 3, 4, 5])
@pytest.mark.parametrize("truss", [0, 1])
def test_random_vs_oracle(kp, orc, k, truss):
    for seed in range(6):
        rng = np.random.default_rng(100 * k + seed)
        n = int(rng.integers(30, 90))
        off, adj = orc.random_graph(n, float(rng.uniform(0.05, 0.2)), seed,
                                    [(int(rng.integers(10, 20)), float(rng.uniform(0.8, 1.0))) for _ in range(3)])
        for q in (2 * k - 1, 2 * k + 1, 2 * k + 4):
            g = kp.enumerate_csr(off, adj, k, q, truss=truss)
            o = orc.enumerate_csr(off, adj, k, q, truss, threads=2)
            assert (g["count"], g["hash"], g["tasks"]) == (o["count"], o["hash"], o["tasks"]), (seed, k, q)


def test_left_sets_beyond_1024(kp, orc):
    from conftest import big_left_graph
    off, adj = big_left_graph()
    g = kp.enumerate_csr(off, adj, 2, 4)
    o = orc.enumerate_csr(off, adj, 2, 4, threads=4)
    assert g["max_left"] == o["max_left"] > 1024
    assert (g["count"], g["hash"], g["tasks"]) == (o["count"], o["hash"], o["tasks"])


def test_big_root_analytic(kp, orc):
    """Roots of 1,105 local vertices (two bitset words per lane): the count and
    hash equal the ones derived by hand for this graph, and the task count the
    oracle's."""
    from conftest import big_root_expected, big_root_graph
    off, adj = big_root_graph(1100)
    g = kp.enumerate_csr(off, adj, 2, 6)
    e = big_root_expected(1100)
    assert g["max_local_n"] == 1105
    assert (g["count"], g["hash"]) == (e["count"], e["hash"])
    o = orc.enumerate_csr(off, adj, 2, 6, threads=4)
    assert g["tasks"] == o["tasks"]


@pytest.mark.parametrize("nbig,core,p,k,q", [(1150, 4, 0.003, 2, 6), (1200, 5, 0.004, 3, 9)])
def test_big_root_random(kp, orc, nbig, core, p, k, q):
    """Roots above 1024 local vertices with random structure among their C2."""
    from conftest import big_root_graph
    off, adj = big_root_graph(nbig, core, p, seed=5)
    g = kp.enumerate_csr(off, adj, k, q)
    o = orc.enumerate_csr(off, adj, k, q, threads=4)
    assert g["max_local_n"] == o["max_n"] > 1024
    assert (g["count"], g["hash"], g["tasks"], g["valid_roots"]) == (o["count"], o["hash"], o["tasks"], o["valid_roots"])


def test_edge_cases(kp):
    # empty graph, no vertex survives the core, graph too small for any root
    off = np.zeros(1, np.uint32)
    adj = np.zeros(0, np.uint32)
    g = kp.enumerate_csr(off, adj, 2, 8)
    assert g["count"] == 0 and g["hash"] == 0 and g["pn"] == 0
    n = 10
    rows = [[j for j in range(n) if j != i] for i in range(n)]
    off = np.zeros(n + 1, np.uint32)
    off[1:] = np.cumsum([len(r) for r in rows])
    adj = np.concatenate(rows).astype(np.uint32)
    g = kp.enumerate_csr(off, adj, 2, 11)      # K10 has no 11-vertex k-plex
    assert g["count"] == 0
    g = kp.enumerate_csr(off, adj, 2, 10)      # exactly the clique
    assert g["count"] == 1 and g["valid_roots"] >= 1


@pytest.mark.parametrize("key", ["soc-epinions.bin:4:30:0", "email-euall.bin:3:12:0", "email-euall.bin:3:12:1"])
def test_shipped_datasets(kp, key):
    fname, k, q, tr = key.split(":")
    p = dataset(fname)
    if not p:
        pytest.skip("dataset not copied (tests/golden/fetch_datasets.sh)")
    g = kp.enumerate_file(p, int(k), int(q), 0.25, int(tr))
    gold = golden()["datasets"][key]
    assert g["count"] == {"soc-epinions.bin": 13172906, "email-euall.bin": 32639016}[fname]   # README.md:142, :144
    assert (g["count"], g["hash"], g["tasks"]) == (gold["count"], gold["hash"], gold["tasks"])


def _subset_keys():
    return sorted(golden().get("subsets", {}))


@pytest.mark.parametrize("key", _subset_keys())
def test_synthetic_subsets(kp, key):
    """Stated root ranges of the full-size synthetic workloads (configs 2 and 3), which
    hold too many maximal k-plexes for the oracle to enumerate whole, against the
    oracle's fixture for the same roots."""
    s = golden()["subsets"][key]
    w = kp.WORKLOADS[s["workload"]]
    off, adj = kp.workload_graph(s["workload"])
    g = kp.enumerate_csr(off, adj, w["k"], w["q"], w["thres"], w["truss"], root_begin=s["root_begin"],
                         root_end=s["root_end"])
    assert (g["count"], g["hash"], g["tasks"], g["valid_roots"]) == (s["count"], s["hash"], s["tasks"], s["valid_roots"])
    assert g["max_local_n"] == s["max_n"]


def test_repeat_and_reuse(kp):
    """Device buffers are cached between calls: repeated searches and a second graph stay exact."""
    off, adj = kp.workload_graph("small")
    prep = kp.prepare(off, adj, 2, 8)
    try:
        a, b = prep.search(), prep.search()
        assert (a["count"], a["hash"], a["tasks"]) == (b["count"], b["hash"], b["tasks"])
    finally:
        prep.release()
    g = golden()["random"][0]
