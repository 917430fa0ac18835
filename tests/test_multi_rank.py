"""Multi-GPU host logic on CPU: two gloo ranks shard the roots (r % world == rank),
each enumerates its shard, and bench.py's reduction rebuilds the whole-graph
count and hash.  The per-rank enumeration here is the oracle (CPU); on GPUs the
same partition goes through kplex_params.shard_index/shard_count."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import PKG, ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q, weighted=False):
    import sys
    sys.path[:0] = [ROOT, PKG]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        import kplex_b200 as kp
        import oracle
        off, adj = kp.workload_graph("small")
        if weighted:   # every process computes the same cost-weighted assignment
            owner = kp.partition_roots(kp.preprocess(off, adj, 2, 8, 0), 8, world)
            part = oracle.enumerate_owned(off, adj, 2, 8, 0, owner, rank, threads=2)
        else:
            part = oracle.enumerate_shard(off, adj, 2, 8, 0, rank, world, threads=2)
        c, h, ms = bench.allreduce_results(dist, part["count"], part["hash"], float(rank + 1), "cpu")
        q.put((rank, c, h, ms, part["valid_roots"]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("weighted", [False, True])
def test_two_rank_shards_reduce_to_whole(kp, orc, weighted):
    off, adj = kp.workload_graph("small")
    whole = orc.enumerate_csr(off, adj, 2, 8, 0)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q, weighted)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, c, h, ms, _ in out:
        assert (c, h) == (whole["count"], whole["hash"])
        assert ms == 2.0
    assert sum(o[4] for o in out) == whole["valid_roots"]


def test_weighted_partition_covers_every_root_once_and_balances(kp):
    """kplex_partition_roots: every root gets one owner in [0, shards), the same
    assignment every time, and the estimated loads are close to even."""
    import numpy as np
    off, adj = kp.workload_graph("epinions")
    pre = kp.preprocess(off, adj, 4, 30, 0)
    nroots = pre["pn"] - 30 + 2
    o = pre["off"]
    later = np.array([(pre["dpos"][pre["adj"][o[v]:o[v + 1]]] > pre["dpos"][v]).sum() for v in pre["dseq"][:nroots]])
    cost = (np.minimum(later, 1023) + 1).astype(np.float64) ** 2
    for shards in (2, 3, 8):
        a = kp.partition_roots(pre, 30, shards)
        assert len(a) == nroots and a.max() < shards
        assert (a == kp.partition_roots(pre, 30, shards)).all()
        loads = np.array([cost[a == s].sum() for s in range(shards)])
        assert loads.max() <= 1.05 * loads.mean()
