"""Python view of libkplex.so (include/kplex.h) for tests, the bench and scripting.

The product is the C ABI; this module only marshals numpy arrays into it.  It
mirrors the reference's drop-in surface: `enumerate_file(path, k, q, t, truss)`
is `./main <graph> -k K -q Q -t T -tr TR` (main.cu:11-61) and returns the
values the reference prints (inc/host_funcs.h:1149-1157) plus the 64-bit
count and the plex hash.  There is no CPU fallback: if libkplex.so is missing
or no sm_100 device is present, the calls fail with KplexError.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libkplex.so")

OK, ERR_PARAM, ERR_IO, ERR_FORMAT, ERR_CUDA, ERR_NOMEM, ERR_CAPACITY, ERR_TIMEOUT, ERR_NO_DEVICE, ERR_INTERNAL = range(10)
FLAG_QUIET, FLAG_NO_HASH, FLAG_SPILL_HOST, FLAG_TEST_NO_WAIT, FLAG_SHARD_WEIGHTED = 0x1, 0x2, 0x4, 0x8, 0x10


class KplexError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"kplex status {status}: {message}")
        self.status = status


class Params(ctypes.Structure):
    _fields_ = [("k", ctypes.c_int), ("q", ctypes.c_int), ("thres", ctypes.c_float), ("truss", ctypes.c_int),
                ("flags", ctypes.c_uint32), ("device", ctypes.c_int), ("pool_slots", ctypes.c_uint64),
                ("omp_threads", ctypes.c_uint32), ("shard_index", ctypes.c_uint32), ("shard_count", ctypes.c_uint32),
                ("blocks_per_sm", ctypes.c_uint32), ("stage_after", ctypes.c_int32), ("root_begin", ctypes.c_uint32),
                ("root_end", ctypes.c_uint32)]


class Result(ctypes.Structure):
    _fields_ = [("count", ctypes.c_uint64), ("hash", ctypes.c_uint64), ("valid_roots", ctypes.c_uint64),
                ("tasks", ctypes.c_uint64), ("nodes", ctypes.c_uint64), ("pn", ctypes.c_uint32), ("pm", ctypes.c_uint32),
                ("max_local_n", ctypes.c_uint32), ("max_left", ctypes.c_uint32), ("pauses", ctypes.c_uint32),
                ("spilled", ctypes.c_uint32), ("ms_preprocess", ctypes.c_double), ("ms_device", ctypes.c_double),
                ("ms_ref_region", ctypes.c_double), ("ms_total", ctypes.c_double), ("status", ctypes.c_int),
                ("gpu_launches", ctypes.c_uint32), ("ms_decompose", ctypes.c_double), ("ms_ksearch", ctypes.c_double),
                ("ms_bnb", ctypes.c_double), ("bnb_bytes", ctypes.c_uint64), ("roots_bytes", ctypes.c_uint64),
                ("ks_tasks", ctypes.c_uint64), ("stage_copies", ctypes.c_uint64), ("ks_warp_ms", ctypes.c_double),
                ("bnb_warp_ms", ctypes.c_double), ("idle_warp_ms", ctypes.c_double), ("search_warps", ctypes.c_uint32)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class Graph(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint32), ("m_directed", ctypes.c_uint64),
                ("offsets", ctypes.POINTER(ctypes.c_uint32)), ("neighbors", ctypes.POINTER(ctypes.c_uint32))]


class Job(ctypes.Structure):
    _fields_ = [("offsets", ctypes.POINTER(ctypes.c_uint32)), ("neighbors", ctypes.POINTER(ctypes.c_uint32)),
                ("n", ctypes.c_uint32), ("m_directed", ctypes.c_uint64), ("k", ctypes.c_int), ("q", ctypes.c_int),
                ("truss", ctypes.c_int)]


class GenSpec(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64), ("n", ctypes.c_uint32), ("base_edges", ctypes.c_uint64),
                ("exponent", ctypes.c_double), ("max_degree", ctypes.c_uint32), ("groups", ctypes.c_uint32),
                ("group_min", ctypes.c_uint32), ("group_max", ctypes.c_uint32),
                ("density_min", ctypes.c_double), ("density_max", ctypes.c_double)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("slots", ctypes.c_uint32), ("max_batch", ctypes.c_uint32),
                ("mem_budget", ctypes.c_uint64), ("split_grid", ctypes.c_uint32), ("thres", ctypes.c_float),
                ("flags", ctypes.c_uint32), ("pool_slots", ctypes.c_uint64), ("large_bytes", ctypes.c_uint64)]


class Completion(ctypes.Structure):
    _fields_ = [("tag", ctypes.c_uint64), ("status", ctypes.c_int), ("batch_size", ctypes.c_uint32),
                ("count", ctypes.c_uint64), ("hash", ctypes.c_uint64), ("valid_roots", ctypes.c_uint64),
                ("pn", ctypes.c_uint32), ("slot", ctypes.c_uint32), ("ms_queue", ctypes.c_double),
                ("ms_service", ctypes.c_double), ("ms_latency", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("rejected", ctypes.c_uint64),
                ("launches", ctypes.c_uint64), ("device_bytes", ctypes.c_uint64), ("peak_device_bytes", ctypes.c_uint64),
                ("max_concurrent", ctypes.c_uint32), ("max_batch_seen", ctypes.c_uint32)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


# The benchmark workloads (seeded synthetic stand-ins for the reference's inputs).
WORKLOADS = {
    # Chung-Lu n=2,000, mean degree 10, exponent 2.5, 20 planted groups of 16 at density 0.9; k=2 q=8
    "small": dict(spec=dict(seed=1, n=2000, base_edges=10000, exponent=2.5, max_degree=0, groups=20,
                            group_min=16, group_max=16, density_min=0.9, density_max=0.9), k=2, q=8, thres=0.25, truss=0),
    # epinions-shaped: n=75,879, 405,740 edges, exponent 2.1, cap 3,044, 200 groups U[40,80] at 0.9; k=4 q=30
    "epinions": dict(spec=dict(seed=2, n=75879, base_edges=405740, exponent=2.1, max_degree=3044, groups=200,
                               group_min=40, group_max=80, density_min=0.9, density_max=0.9), k=4, q=30, thres=0.25, truss=0),
    # email-euall-shaped: n=265,214, 364,481 edges, exponent 1.8, cap 7,636, 50 groups U[15,25] at 0.85; k=3 q=12, truss
    "email": dict(spec=dict(seed=3, n=265214, base_edges=364481, exponent=1.8, max_degree=7636, groups=50,
                            group_min=15, group_max=25, density_min=0.85, density_max=0.85), k=3, q=12, thres=0.25, truss=1),
}

_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise KplexError(ERR_NO_DEVICE, f"{LIB_PATH} is not built (run make in {HERE})")
        L = ctypes.CDLL(LIB_PATH)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        L.kplex_enumerate_csr.argtypes = [u32p, u32p, ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER(Params), ctypes.POINTER(Result)]
        L.kplex_enumerate_file.argtypes = [ctypes.c_char_p, ctypes.POINTER(Params), ctypes.POINTER(Result)]
        L.kplex_prepare.argtypes = [u32p, u32p, ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER(Params),
                                    ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(Result)]
        L.kplex_search.argtypes = [ctypes.c_void_p, ctypes.POINTER(Result)]
        L.kplex_release.argtypes = [ctypes.c_void_p]
        L.kplex_release.restype = None
        L.kplex_load_bin.argtypes = [ctypes.c_char_p, ctypes.POINTER(Graph)]
        L.kplex_save_bin.argtypes = [ctypes.c_char_p, ctypes.POINTER(Graph)]
        L.kplex_free_graph.argtypes = [ctypes.POINTER(Graph)]
        L.kplex_free_graph.restype = None
        L.kplex_generate.argtypes = [ctypes.POINTER(GenSpec), ctypes.POINTER(Graph)]
        L.kplex_status_string.restype = ctypes.c_char_p
        L.kplex_last_error.restype = ctypes.c_char_p
        L.kplex_device_ok.argtypes = [ctypes.c_int]
        i32p = ctypes.POINTER(ctypes.c_int32)
        L.kplex_preprocess_csr.argtypes = [u32p, u32p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_uint32, u32p, u32p, i32p, i32p, u32p,
                                           ctypes.POINTER(ctypes.c_uint64)]
        L.kplex_preprocess_csr.restype = ctypes.c_longlong
        L.kplex_partition_roots.argtypes = [u32p, u32p, i32p, i32p, ctypes.c_uint32, ctypes.c_int, ctypes.c_uint32,
                                            ctypes.POINTER(ctypes.c_uint8)]
        L.kplex_partition_roots.restype = ctypes.c_longlong
        L.kplex_enumerate_batch.argtypes = [ctypes.POINTER(Job), ctypes.c_uint32, ctypes.POINTER(Params),
                                            ctypes.POINTER(Result), ctypes.POINTER(Result)]
        L.kplex_prepare_batch.argtypes = [ctypes.POINTER(Job), ctypes.c_uint32, ctypes.POINTER(Params),
                                          ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(Result)]
        L.kplex_search_batch.argtypes = [ctypes.c_void_p, ctypes.POINTER(Result), ctypes.POINTER(Result)]
        L.kplex_autotune_batch.argtypes = [ctypes.POINTER(Job), ctypes.c_uint32, ctypes.POINTER(Params), ctypes.c_uint32,
                                           ctypes.POINTER(Params), ctypes.POINTER(ctypes.c_double)]
        L.kplex_server_create.argtypes = [ctypes.POINTER(ServerConfig), ctypes.POINTER(ctypes.c_void_p)]
        L.kplex_server_submit.argtypes = [ctypes.c_void_p, ctypes.POINTER(Job), ctypes.c_uint64]
        L.kplex_server_poll.argtypes = [ctypes.c_void_p, ctypes.POINTER(Completion), ctypes.c_uint32, ctypes.c_int]
        L.kplex_server_drain.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.kplex_server_stats_get.argtypes = [ctypes.c_void_p, ctypes.POINTER(ServerStats)]
        L.kplex_server_destroy.argtypes = [ctypes.c_void_p]
        L.kplex_server_destroy.restype = None
        _lib = L
    return _lib


def _err(status: int) -> KplexError:
    L = lib()
    return KplexError(status, f"{L.kplex_status_string(status).decode()}: {L.kplex_last_error().decode()}")


def _u32p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def _graph_to_numpy(g: Graph):
    off = np.ctypeslib.as_array(g.offsets, shape=(g.n + 1,)).copy()
    adj = np.ctypeslib.as_array(g.neighbors, shape=(max(g.m_directed, 1),))[: g.m_directed].copy()
    return off, adj


def load_bin(path: str):
    """Read a reference .bin graph; returns (offsets u32[n+1], neighbors u32[m])."""
    g = Graph()
    rc = lib().kplex_load_bin(path.encode(), ctypes.byref(g))
    if rc:
        raise _err(rc)
    try:
        return _graph_to_numpy(g)
    finally:
        lib().kplex_free_graph(ctypes.byref(g))


def save_bin(path: str, off: np.ndarray, adj: np.ndarray) -> None:
    off = np.ascontiguousarray(off, dtype=np.uint32)
    adj = np.ascontiguousarray(adj, dtype=np.uint32)
    g = Graph(len(off) - 1, len(adj), _u32p(off), _u32p(adj))
    rc = lib().kplex_save_bin(path.encode(), ctypes.byref(g))
    if rc:
        raise _err(rc)


def generate(spec: dict):
    """Seeded synthetic graph (see WORKLOADS); returns (offsets, neighbors)."""
    s = GenSpec(**spec)
    g = Graph()
    rc = lib().kplex_generate(ctypes.byref(s), ctypes.byref(g))
    if rc:
        raise _err(rc)
    try:
        return _graph_to_numpy(g)
    finally:
        lib().kplex_free_graph(ctypes.byref(g))


def workload_graph(name: str):
    return generate(WORKLOADS[name]["spec"])


def make_params(k: int, q: int, thres: float = 0.25, truss: int = 0, flags: int = FLAG_QUIET, device: int = 0,
                pool_slots: int = 0, omp_threads: int = 0, shard_index: int = 0, shard_count: int = 0,
                blocks_per_sm: int = 0, stage_after: int = 0, root_begin: int = 0, root_end: int = 0) -> Params:
    return Params(k, q, thres, truss, flags, device, pool_slots, omp_threads, shard_index, shard_count,
                  blocks_per_sm, stage_after, root_begin, root_end)


def enumerate_csr(off: np.ndarray, adj: np.ndarray, k: int, q: int, thres: float = 0.25, truss: int = 0,
                  flags: int = FLAG_QUIET, device: int = 0, pool_slots: int = 0, check: bool = True,
                  shard_index: int = 0, shard_count: int = 0, root_begin: int = 0, root_end: int = 0,
                  blocks_per_sm: int = 0, stage_after: int = 0) -> dict:
    """Count and hash of the maximal k-plexes with >= q vertices (kplex_enumerate_csr).
    root_begin/root_end (end 0 = all) and shard_index/shard_count restrict the
    search to a stated subset of roots by degeneracy rank."""
    off = np.ascontiguousarray(off, dtype=np.uint32)
    adj = np.ascontiguousarray(adj, dtype=np.uint32)
    p = make_params(k, q, thres, truss, flags, device, pool_slots, 0, shard_index, shard_count,
                    blocks_per_sm=blocks_per_sm, stage_after=stage_after, root_begin=root_begin, root_end=root_end)
    r = Result()
    rc = lib().kplex_enumerate_csr(_u32p(off), _u32p(adj), len(off) - 1, len(adj), ctypes.byref(p), ctypes.byref(r))
    if rc and check:
        raise _err(rc)
    return r.as_dict()


def enumerate_file(path: str, k: int, q: int, thres: float = 0.25, truss: int = 0, flags: int = FLAG_QUIET,
                   device: int = 0) -> dict:
    p = make_params(k, q, thres, truss, flags, device)
    r = Result()
    rc = lib().kplex_enumerate_file(path.encode(), ctypes.byref(p), ctypes.byref(r))
    if rc:
        raise _err(rc)
    return r.as_dict()


@dataclass
class Prepared:
    """Preprocessed graph resident on the device; search() reruns the device stage."""
    handle: ctypes.c_void_p
    pre: dict

    def search(self) -> dict:
        r = Result()
        rc = lib().kplex_search(self.handle, ctypes.byref(r))
        if rc:
            raise _err(rc)
        return r.as_dict()

    def release(self) -> None:
        if self.handle:
            lib().kplex_release(self.handle)
            self.handle = None


def prepare(off: np.ndarray, adj: np.ndarray, k: int, q: int, thres: float = 0.25, truss: int = 0,
            flags: int = FLAG_QUIET, device: int = 0, pool_slots: int = 0, shard_index: int = 0,
            shard_count: int = 0, root_begin: int = 0, root_end: int = 0, blocks_per_sm: int = 0,
            stage_after: int = 0) -> Prepared:
    off = np.ascontiguousarray(off, dtype=np.uint32)
    adj = np.ascontiguousarray(adj, dtype=np.uint32)
    p = make_params(k, q, thres, truss, flags, device, pool_slots, 0, shard_index, shard_count,
                    blocks_per_sm=blocks_per_sm, stage_after=stage_after, root_begin=root_begin, root_end=root_end)
    h = ctypes.c_void_p()
    r = Result()
    rc = lib().kplex_prepare(_u32p(off), _u32p(adj), len(off) - 1, len(adj), ctypes.byref(p), ctypes.byref(h), ctypes.byref(r))
    if rc:
        raise _err(rc)
    return Prepared(h, r.as_dict())


def preprocess(off: np.ndarray, adj: np.ndarray, k: int, q: int, truss: int = 0, omp_threads: int = 0) -> dict:
    """Host preprocessing only: pruned CSR, degeneracy order, pruned->input id map."""
    off = np.ascontiguousarray(off, dtype=np.uint32)
    adj = np.ascontiguousarray(adj, dtype=np.uint32)
    n = len(off) - 1
    o_off = np.zeros(n + 1, dtype=np.uint32)
    o_adj = np.zeros(max(len(adj), 1), dtype=np.uint32)
    o_dpos = np.zeros(max(n, 1), dtype=np.int32)
    o_dseq = np.zeros(max(n, 1), dtype=np.int32)
    o_orig = np.zeros(max(n, 1), dtype=np.uint32)
    m = ctypes.c_uint64()
    i32 = ctypes.POINTER(ctypes.c_int32)
    pn = lib().kplex_preprocess_csr(_u32p(off), _u32p(adj), n, len(adj), k, q, truss, omp_threads, _u32p(o_off),
                                    _u32p(o_adj), o_dpos.ctypes.data_as(i32), o_dseq.ctypes.data_as(i32),
                                    _u32p(o_orig), ctypes.byref(m))
    if pn < 0:
        raise _err(int(-pn))
    return {"pn": int(pn), "off": o_off[: pn + 1], "adj": o_adj[: m.value], "dpos": o_dpos[:pn], "dseq": o_dseq[:pn],
            "orig": o_orig[:pn]}


def partition_roots(pre: dict, q: int, shards: int) -> np.ndarray:
    """Cost-weighted shard of every root (kplex_partition_roots) for a preprocess() result."""
    i32 = ctypes.POINTER(ctypes.c_int32)
    nroots = max(0, pre["pn"] - q + 2)
    owner = np.zeros(max(nroots, 1), dtype=np.uint8)
    off = np.ascontiguousarray(pre["off"], dtype=np.uint32)
    adj = np.ascontiguousarray(pre["adj"] if len(pre["adj"]) else np.zeros(1, np.uint32), dtype=np.uint32)
    dpos = np.ascontiguousarray(pre["dpos"], dtype=np.int32)
    dseq = np.ascontiguousarray(pre["dseq"], dtype=np.int32)
    rc = lib().kplex_partition_roots(_u32p(off), _u32p(adj), dpos.ctypes.data_as(i32), dseq.ctypes.data_as(i32),
                                     pre["pn"], q, shards, owner.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
    if rc < 0:
        raise _err(int(-rc))
    return owner[:nroots]


def _batch_draws(count: int, seed: int, q_per_k: int = 0):
    rng = np.random.default_rng(seed)
    for i in range(count):
        n = int(round(float(np.exp(rng.uniform(np.log(64), np.log(2048))))))
        deg = float(rng.uniform(8, 24))
        groups = min(int(rng.integers(1, 9)), max(1, n // 30))   # groups never exceed the graph
        gmax = int(min(30, n // groups))
        spec = dict(seed=int(seed) * 1_000_003 + i, n=n, base_edges=int(round(n * deg / 2)), exponent=2.3,
                    max_degree=0, groups=groups, group_min=min(10, gmax), group_max=gmax,
                    density_min=0.85, density_max=0.95)
        k = int(rng.integers(2, 5))
        q = int(rng.integers(8, 21))
        if q_per_k:
            q = max(q, q_per_k * k)
        yield spec, k, q


def batch_graph(index: int, seed: int = 4, q_per_k: int = 0):
    """Graph `index` of batch_workload(seed=seed) alone: (offsets, neighbors, k, q)."""
    for i, (spec, k, q) in enumerate(_batch_draws(index + 1, seed, q_per_k)):
        if i == index:
            off, adj = generate(spec)
            return off, adj, k, q


def batch_workload(count: int = 4096, seed: int = 4, q_per_k: int = 0):
    """The batched workload: `count` independent seeded graphs.  Per graph: n log-uniform
    in [64, 2048], Chung-Lu mean degree U[8, 24] with exponent 2.3, 1-8 planted groups
    of 10-30 vertices at density U[0.85, 0.95], k uniform in {2, 3, 4}, q uniform in [8, 20].
    q_per_k > 0 raises q to at least q_per_k * k (the same graphs and draws
    otherwise): with small q the dense planted groups hold hundreds of millions
    of maximal plexes per graph when k = 4 (one holds 586 M at q = 8).  Returns a list of (offsets, neighbors, k, q)."""
    out = []
    for spec, k, q in _batch_draws(count, seed, q_per_k):
        off, adj = generate(spec)
        out.append((off, adj, k, q))
    return out


class PreparedBatch:
    """A batch of graphs resident on the device; search() reruns the device stage."""

    def __init__(self, handle, n, total):
        self.handle, self.n, self.pre = handle, n, total

    def search(self):
        per = (Result * self.n)()
        tot = Result()
        rc = lib().kplex_search_batch(self.handle, per, ctypes.byref(tot))
        if rc:
            raise _err(rc)
        return [r.as_dict() for r in per], tot.as_dict()

    def release(self):
        if self.handle:
            lib().kplex_release(self.handle)
            self.handle = None


def _jobs(graphs, truss=0):
    keep = []
    jobs = (Job * len(graphs))()
    for i, (off, adj, k, q) in enumerate(graphs):
        off = np.ascontiguousarray(off, dtype=np.uint32)
        adj = np.ascontiguousarray(adj if len(adj) else np.zeros(1, np.uint32), dtype=np.uint32)
        keep.append((off, adj))
        jobs[i] = Job(_u32p(off), _u32p(adj), len(off) - 1, int(off[-1]), k, q, truss)
    return jobs, keep


def enumerate_batch(graphs, thres: float = 0.25, truss: int = 0, flags: int = FLAG_QUIET, device: int = 0,
                    pool_slots: int = 0, blocks_per_sm: int = 0, stage_after: int = 0):
    """graphs: list of (offsets, neighbors, k, q).  Returns (per-graph results, totals)."""
    jobs, keep = _jobs(graphs, truss)
    p = make_params(2, 3, thres, 0, flags, device, pool_slots, blocks_per_sm=blocks_per_sm, stage_after=stage_after)
    per = (Result * len(graphs))()
    tot = Result()
    rc = lib().kplex_enumerate_batch(jobs, len(graphs), ctypes.byref(p), per, ctypes.byref(tot))
    if rc:
        raise _err(rc)
    return [r.as_dict() for r in per], tot.as_dict()


def prepare_batch(graphs, thres: float = 0.25, truss: int = 0, flags: int = FLAG_QUIET, device: int = 0,
                  pool_slots: int = 0, blocks_per_sm: int = 0, stage_after: int = 0) -> PreparedBatch:
    jobs, keep = _jobs(graphs, truss)
    p = make_params(2, 3, thres, 0, flags, device, pool_slots, blocks_per_sm=blocks_per_sm, stage_after=stage_after)
    h = ctypes.c_void_p()
    tot = Result()
    rc = lib().kplex_prepare_batch(jobs, len(graphs), ctypes.byref(p), ctypes.byref(h), ctypes.byref(tot))
    if rc:
        raise _err(rc)
    return PreparedBatch(h, len(graphs), tot.as_dict())


def autotune_batch(graphs, sample: int = 256, thres: float = 0.25, truss: int = 0, flags: int = FLAG_QUIET,
                   device: int = 0) -> tuple[dict, float]:
    """Schedule chosen by kplex_autotune_batch on a sample of the batch: returns
    (tuned params as a dict for enumerate_batch/prepare_batch, sample device ms)."""
    jobs, keep = _jobs(graphs, truss)
    p = make_params(2, 3, thres, 0, flags, device)
    best = Params()
    ms = ctypes.c_double()
    rc = lib().kplex_autotune_batch(jobs, len(graphs), ctypes.byref(p), sample, ctypes.byref(best), ctypes.byref(ms))
    if rc:
        raise _err(rc)
    return {"thres": best.thres, "pool_slots": best.pool_slots, "blocks_per_sm": best.blocks_per_sm,
            "stage_after": best.stage_after}, ms.value


def device_ok(device: int = 0) -> bool:
    return bool(lib().kplex_device_ok(device))


class Server:
    """Continuous-batching request server (kplex_server_* in include/kplex.h).

    submit() copies the graph and returns at once; completions arrive through
    poll() as dicts with the request's tag, count, hash and its queue, service
    and end-to-end latencies in ms."""

    def __init__(self, device: int = 0, slots: int = 2, max_batch: int = 1024, mem_budget: int = 16 << 30,
                 split_grid: bool = False, thres: float = 0.25, flags: int = FLAG_QUIET, pool_slots: int = 0,
                 large_bytes: int = 0):
        cfg = ServerConfig(device, slots, max_batch, mem_budget, 1 if split_grid else 0, thres, flags, pool_slots,
                           large_bytes)
        h = ctypes.c_void_p()
        rc = lib().kplex_server_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc:
            raise _err(rc)
        self.handle = h

    def submit(self, off: np.ndarray, adj: np.ndarray, k: int, q: int, truss: int = 0, tag: int = 0) -> None:
        off = np.ascontiguousarray(off, dtype=np.uint32)
        adj = np.ascontiguousarray(adj, dtype=np.uint32) if len(adj) else np.zeros(1, np.uint32)
        m = int(off[-1])
        job = Job(_u32p(off), _u32p(adj), len(off) - 1, m, k, q, truss)
        rc = lib().kplex_server_submit(self.handle, ctypes.byref(job), tag)
        if rc:
            raise _err(rc)

    def poll(self, max_items: int = 256, timeout_ms: int = 0) -> list[dict]:
        buf = (Completion * max_items)()
        n = lib().kplex_server_poll(self.handle, buf, max_items, timeout_ms)
        if n < 0:
            raise _err(-n)
        return [buf[i].as_dict() for i in range(n)]

    def drain(self, timeout_ms: int = -1) -> None:
        rc = lib().kplex_server_drain(self.handle, timeout_ms)
        if rc:
            raise _err(rc)

    def stats(self) -> dict:
        st = ServerStats()
        lib().kplex_server_stats_get(self.handle, ctypes.byref(st))
        return st.as_dict()

    def close(self) -> None:
        if self.handle:
            lib().kplex_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
