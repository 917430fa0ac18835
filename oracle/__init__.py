"""CPU ORACLE — test infrastructure only.

ctypes view of oracle/liboracle.so: the C++ restatement of the reference
algorithm (oracle.cpp, which cites the reference file:line it follows) and an
independent brute-force enumerator (brute.cpp).  Only tests/, the smoke check
in __graft_entry__.py and bench.py's CPU baseline / reference arm import this
package; the product (libkplex.so and its Python view) never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


class OracleResult(ctypes.Structure):
    _fields_ = [("count", ctypes.c_uint64), ("hash", ctypes.c_uint64), ("tasks", ctypes.c_uint64),
                ("valid_roots", ctypes.c_uint64), ("truncated_roots", ctypes.c_uint64),
                ("depth_capped_roots", ctypes.c_uint64), ("oversized_roots", ctypes.c_uint64),
                ("pn", ctypes.c_uint32), ("pm", ctypes.c_uint32), ("max_n", ctypes.c_uint32), ("max_left", ctypes.c_uint32),
                ("ms_preprocess", ctypes.c_double), ("ms_search", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
        L = ctypes.CDLL(LIB_PATH)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        L.oracle_enumerate_csr.argtypes = [u32p, u32p, ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(OracleResult)]
        L.oracle_bruteforce_csr.argtypes = [u32p, u32p, ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
        L.oracle_preprocess.argtypes = [u32p, u32p, ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        u32p, u32p, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32), u32p,
                                        ctypes.POINTER(ctypes.c_uint64)]
        L.oracle_preprocess.restype = ctypes.c_longlong
        L.oracle_enumerate_sequential.argtypes = [u32p, u32p, ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_int, ctypes.POINTER(OracleResult)]
        L.oracle_enumerate_shard.argtypes = [u32p, u32p, ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(OracleResult)]
        L.oracle_enumerate_owned.argtypes = [u32p, u32p, ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, ctypes.POINTER(ctypes.c_uint8), ctypes.c_uint64,
                                             ctypes.c_uint32, ctypes.POINTER(OracleResult)]
        _lib = L
    return _lib


def _u32(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def enumerate_csr(off, adj, k: int, q: int, truss: int = 0, threads: int = 0,
                  root_begin: int = 0, root_end: int = 2**64 - 1) -> dict:
    """Count and hash of the maximal k-plexes with >= q vertices, as the reference computes them.

    root_begin/root_end restrict the run to a range of degeneracy ranks (a
    bounded sample for timing)."""
    off, po = _u32(off)
    adj, pa = _u32(adj)
    r = OracleResult()
    rc = lib().oracle_enumerate_csr(po, pa, len(off) - 1, k, q, truss, threads, root_begin, root_end, ctypes.byref(r))
    if rc:
        raise RuntimeError(f"oracle failed with {rc}")
    return r.as_dict()


def enumerate_sequential(off, adj, k: int, q: int, truss: int = 0, threads: int = 0) -> dict:
    """As enumerate_csr but with the reference's single sequential k-search per root."""
    off, po = _u32(off)
    adj, pa = _u32(adj)
    r = OracleResult()
    rc = lib().oracle_enumerate_sequential(po, pa, len(off) - 1, k, q, truss, threads, ctypes.byref(r))
    if rc:
        raise RuntimeError(f"oracle failed with {rc}")
    return r.as_dict()


def enumerate_shard(off, adj, k: int, q: int, truss: int, shard_index: int, shard_count: int, threads: int = 0) -> dict:
    """The roots whose degeneracy rank r has r % shard_count == shard_index (the multi-GPU partition)."""
    off, po = _u32(off)
    adj, pa = _u32(adj)
    r = OracleResult()
    rc = lib().oracle_enumerate_shard(po, pa, len(off) - 1, k, q, truss, threads, shard_index, shard_count, ctypes.byref(r))
    if rc:
        raise RuntimeError(f"oracle failed with {rc}")
    return r.as_dict()


def enumerate_owned(off, adj, k: int, q: int, truss: int, owner, me: int, threads: int = 0) -> dict:
    """The roots r with owner[r] == me (an explicit partition of the degeneracy ranks)."""
    off, po = _u32(off)
    adj, pa = _u32(adj)
    owner = np.ascontiguousarray(owner, dtype=np.uint8)
    r = OracleResult()
    rc = lib().oracle_enumerate_owned(po, pa, len(off) - 1, k, q, truss, threads,
                                      owner.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), len(owner), me, ctypes.byref(r))
    if rc:
        raise RuntimeError(f"oracle failed with {rc}")
    return r.as_dict()


def bruteforce_csr(off, adj, k: int, q: int, threads: int = 0) -> dict:
    """Exhaustive enumeration with no reference pruning rule (valid for q >= 2k-1)."""
    off, po = _u32(off)
    adj, pa = _u32(adj)
    c = ctypes.c_uint64()
    h = ctypes.c_uint64()
    rc = lib().oracle_bruteforce_csr(po, pa, len(off) - 1, k, q, threads, ctypes.byref(c), ctypes.byref(h))
    if rc:
        raise RuntimeError(f"brute force failed with {rc}")
    return {"count": c.value, "hash": h.value}


def preprocess(off, adj, k: int, q: int, truss: int = 0) -> dict:
    """Pruned CSR, degeneracy order and peeled->input id map, as host:16-122/761-851 compute them."""
    off, po = _u32(off)
    adj, pa = _u32(adj)
    n = len(off) - 1
    o_off = np.zeros(n + 1, dtype=np.uint32)
    o_adj = np.zeros(max(len(adj), 1), dtype=np.uint32)
    o_dpos = np.zeros(max(n, 1), dtype=np.int32)
    o_dseq = np.zeros(max(n, 1), dtype=np.int32)
    o_orig = np.zeros(max(n, 1), dtype=np.uint32)
    m = ctypes.c_uint64()
    pn = lib().oracle_preprocess(po, pa, n, k, q, truss, o_off.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                 o_adj.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                 o_dpos.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                 o_dseq.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                 o_orig.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), ctypes.byref(m))
    return {"pn": int(pn), "off": o_off[: pn + 1], "adj": o_adj[: m.value], "dpos": o_dpos[:pn], "dseq": o_dseq[:pn],
            "orig": o_orig[:pn]}


def random_graph(n: int, p: float, seed: int, planted: list[tuple[int, float]] | None = None):
    """Small seeded G(n,p) plus optional planted dense groups, as a symmetric sorted CSR (numpy)."""
    rng = np.random.default_rng(seed)
    A = rng.random((n, n)) < p
    A = np.triu(A, 1)
    if planted:
        perm = rng.permutation(n)
        pos = 0
        for size, dens in planted:
            size = min(size, n - pos)
            mem = perm[pos: pos + size]
            pos += size
            for i in range(size):
                for j in range(i + 1, size):
                    a, b = sorted((mem[i], mem[j]))
                    A[a, b] = rng.random() < dens
    A = A | A.T
    deg = A.sum(1)
    off = np.zeros(n + 1, dtype=np.uint32)
    off[1:] = np.cumsum(deg)
    adj = np.concatenate([np.nonzero(A[i])[0] for i in range(n)]).astype(np.uint32) if off[-1] else np.zeros(0, np.uint32)
    return off, adj
