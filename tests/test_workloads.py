"""Host-side workload generators used by the batched and served benches (no GPU)."""
import numpy as np


def test_batch_graph_matches_batch_workload(kp):
    graphs = kp.batch_workload(count=12, seed=4)
    for i in (0, 5, 11):
        off, adj, k, q = kp.batch_graph(i, 4)
        assert np.array_equal(off, graphs[i][0]) and np.array_equal(adj, graphs[i][1])
        assert (k, q) == graphs[i][2:]


def test_q_floor_keeps_graphs_and_raises_q(kp):
    plain = kp.batch_workload(count=40, seed=4)
    bounded = kp.batch_workload(count=40, seed=4, q_per_k=4)
    for (o1, a1, k1, q1), (o2, a2, k2, q2) in zip(plain, bounded):
        assert np.array_equal(o1, o2) and np.array_equal(a1, a2) and k1 == k2
        assert q2 == max(q1, 4 * k1)
        assert 2 <= k1 <= 4 and 8 <= q1 <= 20 and q2 >= 2 * k2 - 1


def test_batch_graphs_are_valid_csr(kp):
    for off, adj, k, q in kp.batch_workload(count=8, seed=7):
        n = len(off) - 1
        assert off[0] == 0 and off[-1] == len(adj) and np.all(np.diff(off.astype(np.int64)) >= 0)
        for v in range(n):
            row = adj[off[v]:off[v + 1]]
            assert np.all(np.diff(row.astype(np.int64)) > 0) and np.all(row < n) and v not in row


def test_served_stream_is_seeded_and_mixed(kp):
    import bench
    a, name_a = bench.served_requests(rate=50.0, duration=4.0, seed=5)
    b, name_b = bench.served_requests(rate=50.0, duration=4.0, seed=5)
    assert name_a == name_b and len(a) == len(b) > 100
    assert [(r[0], r[3], r[4], r[5]) for r in a] == [(r[0], r[3], r[4], r[5]) for r in b]
    times = [r[0] for r in a]
    assert times == sorted(times) and times[-1] < 4.0
    kinds = [r[5] for r in a]
    assert kinds.count("small") > kinds.count("large") > 0
    assert all(r[4] >= 4 * r[3] for r in a if r[5] == "small")
