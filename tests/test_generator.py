"""The seeded synthetic workload generator."""
import numpy as np


def test_deterministic_and_simple(kp):
    a = kp.workload_graph("small")
    b = kp.workload_graph("small")
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    off, adj = a
    n = len(off) - 1
    for v in range(n):
        nb = adj[off[v]:off[v + 1]]
        assert np.all(np.diff(nb.astype(np.int64)) > 0)
        assert v not in nb
    # symmetric
    src = np.repeat(np.arange(n), np.diff(off))
    fwd = set(zip(src.tolist(), adj.tolist()))
    assert all((w, v) in fwd for v, w in fwd)


def test_exact_base_edges_and_cap(kp):
    spec = dict(seed=7, n=5000, base_edges=20000, exponent=2.1, max_degree=60, groups=0, group_min=0, group_max=0,
                density_min=1.0, density_max=1.0)
    off, adj = kp.generate(spec)
    assert len(adj) == 2 * 20000
    assert np.diff(off).max() <= 60


def test_planted_group_density(kp):
    spec = dict(seed=9, n=300, base_edges=0, exponent=2.5, max_degree=0, groups=1, group_min=40, group_max=40,
                density_min=0.9, density_max=0.9)
    off, adj = kp.generate(spec)
    assert len(adj) == 2 * round(0.9 * 40 * 39 / 2)
