"""Request server: continuous batching with memory admission.

Every request's count and hash must be the same as a plain call on its graph,
whatever launch it shared; admission must hold requests back when the budget is
taken and refuse one that can never fit; a failing request must not take the
requests batched with it down."""
import time

import numpy as np
import pytest

from conftest import dense_request_graph, oversized_root_graph

pytestmark = pytest.mark.gpu


def _collect(srv, n, timeout_s=300):
    got = {}
    t0 = time.time()
    while len(got) < n and time.time() - t0 < timeout_s:
        for c in srv.poll(64, timeout_ms=200):
            got[c["tag"]] = c
    return got


def test_server_results_match_plain_calls(kp, orc):
    graphs = kp.batch_workload(count=40, seed=11)
    small = kp.workload_graph("small")
    graphs.append((small[0], small[1], 2, 8))
    with kp.Server(slots=2, max_batch=16) as srv:
        for i, (off, adj, k, q) in enumerate(graphs):
            srv.submit(off, adj, k, q, tag=i)
        got = _collect(srv, len(graphs))
        st = srv.stats()
    assert len(got) == len(graphs)
    assert st["completed"] == len(graphs) and st["launches"] >= 2 and st["max_batch_seen"] >= 2
    for i, (off, adj, k, q) in enumerate(graphs):
        one = kp.enumerate_csr(off, adj, k, q)
        c = got[i]
        assert c["status"] == 0
        assert (c["count"], c["hash"], c["valid_roots"]) == (one["count"], one["hash"], one["valid_roots"]), i
        assert c["ms_latency"] >= c["ms_service"] > 0
        if i % 8 == 0:   # and a sample against the oracle, not only against the device
            o = orc.enumerate_csr(off, adj, k, q, threads=4)
            assert (c["count"], c["hash"], c["valid_roots"]) == (o["count"], o["hash"], o["valid_roots"]), i
    assert got[len(graphs) - 1]["count"] == 871


def test_server_split_grid_overlaps(kp):
    graphs = kp.batch_workload(count=24, seed=12)
    with kp.Server(slots=3, max_batch=4, split_grid=True) as srv:
        for i, (off, adj, k, q) in enumerate(graphs):
            srv.submit(off, adj, k, q, tag=i)
        srv.drain(timeout_ms=300_000)
        got = {c["tag"]: c for c in srv.poll(64)}
        st = srv.stats()
    assert st["max_concurrent"] >= 2
    for i, (off, adj, k, q) in enumerate(graphs):
        one = kp.enumerate_csr(off, adj, k, q)
        assert (got[i]["count"], got[i]["hash"]) == (one["count"], one["hash"]), i


def test_server_memory_admission(kp):
    graphs = kp.batch_workload(count=6, seed=13)
    big = dense_request_graph()
    # a budget that holds the largest request's estimate (about 1.75 MB) but not two of
    # them, and no workspace: each request is admitted only when nothing else is in flight
    with kp.Server(slots=2, max_batch=8, mem_budget=1_800_000) as srv:
        with pytest.raises(kp.KplexError) as e:
            srv.submit(big[0], big[1], 2, 20, tag=99)   # its estimate alone exceeds the budget
        assert e.value.status == kp.ERR_NOMEM
        for i, (off, adj, k, q) in enumerate(graphs):
            srv.submit(off, adj, k, q, tag=i)
        srv.drain(timeout_ms=300_000)
        got = {c["tag"]: c for c in srv.poll(64)}
        st = srv.stats()
    assert st["rejected"] == 1 and st["max_batch_seen"] == 1 and st["max_concurrent"] == 1
    for i, (off, adj, k, q) in enumerate(graphs):
        one = kp.enumerate_csr(off, adj, k, q)
        assert (got[i]["count"], got[i]["hash"]) == (one["count"], one["hash"])


def test_server_isolates_failing_request(kp):
    bad = oversized_root_graph(1100, 1000, 1000)
    graphs = kp.batch_workload(count=5, seed=14)
    with kp.Server(slots=1, max_batch=16) as srv:
        with pytest.raises(kp.KplexError):
            srv.submit(bad[0], bad[1], 1, 20, tag=1000)   # k < 2
        srv.submit(bad[0], bad[1], 2, 20, tag=500)
        for i, (off, adj, k, q) in enumerate(graphs):
            srv.submit(off, adj, k, q, tag=i)
        srv.drain(timeout_ms=300_000)
        got = {c["tag"]: c for c in srv.poll(64)}
    assert got[500]["status"] == kp.ERR_CAPACITY
    for i, (off, adj, k, q) in enumerate(graphs):
        one = kp.enumerate_csr(off, adj, k, q)
        assert got[i]["status"] == 0 and (got[i]["count"], got[i]["hash"]) == (one["count"], one["hash"])


def test_server_large_request_runs_alone(kp):
    """A request whose device estimate reaches large_bytes gets a launch of its own:
    with large_bytes = 1 every request is large and runs alone; with the rule off
    (UINT64_MAX) the same queue is batched."""
    graphs = kp.batch_workload(count=8, seed=15)
    for large, want_alone in ((1, True), (2**64 - 1, False)):
        with kp.Server(slots=1, max_batch=16, large_bytes=large) as srv:
            for i, (off, adj, k, q) in enumerate(graphs):
                srv.submit(off, adj, k, q, tag=i)
            srv.drain(timeout_ms=300_000)
            got = {c["tag"]: c for c in srv.poll(64)}
            st = srv.stats()
        assert len(got) == len(graphs)
        if want_alone:
            assert all(c["batch_size"] == 1 for c in got.values()) and st["max_batch_seen"] == 1
        else:
            assert st["max_batch_seen"] >= 2
        for i, (off, adj, k, q) in enumerate(graphs):
            ref = kp.enumerate_csr(off, adj, k, q)
            assert got[i]["status"] == 0 and (got[i]["count"], got[i]["hash"]) == (ref["count"], ref["hash"])
