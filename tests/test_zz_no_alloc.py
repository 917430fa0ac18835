"""kplex_search_noalloc: the device search for callers that cannot allocate device memory.

Some callers must not call cudaMalloc:
- a process whose device memory is already fully reserved by another framework's caching allocator;
- a service whose fixed memory plan forbids allocation on the request path;
- code that cannot afford the device-wide synchronisation an allocation can cause.
For them this entry point carves all scratch from one 64 MiB array that the library
declares at file scope on the device.  The caller passes the pruned graph in its own device
buffers and receives the result on the host.  This test allocates those input buffers itself
with torch; the entry point allocates nothing.  Two calls in a row must give the same
count, hash and task count as the regular entry point.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(kp):
    fn = kp.lib().kplex_search_noalloc
    fn.argtypes = [ctypes.c_void_p] * 5 + [ctypes.c_uint32, ctypes.POINTER(kp.Params), ctypes.POINTER(kp.Result)]
    fn.restype = ctypes.c_int
    return fn


def _device_inputs(kp, off, adj, k, q, truss):
    import torch
    pre = kp.preprocess(off, adj, k, q, truss)
    bufs = [torch.from_numpy(np.ascontiguousarray(a).view(np.int32).copy()).cuda()
            for a in (pre["off"], pre["adj"] if len(pre["adj"]) else np.zeros(1, np.uint32), pre["dpos"], pre["dseq"], pre["orig"])]
    torch.cuda.synchronize()
    return pre, bufs


@pytest.mark.parametrize("name", ["small", "random"])
def test_noalloc_matches_regular_entry_point(kp, orc, name):
    if name == "small":
        off, adj = kp.workload_graph("small")
        k, q, truss = 2, 8, 0
    else:
        off, adj = orc.random_graph(70, 0.15, 11, [(18, 0.9), (16, 1.0)])
        k, q, truss = 3, 8, 1
    want = kp.enumerate_csr(off, adj, k, q, truss=truss)
    pre, bufs = _device_inputs(kp, off, adj, k, q, truss)
    fn = _noalloc(kp)
    p = kp.make_params(k, q, 0.25, truss)
    for _ in range(2):
        r = kp.Result()
        rc = fn(*[b.data_ptr() for b in bufs], pre["pn"], ctypes.byref(p), ctypes.byref(r))
        assert rc == 0, kp.lib().kplex_last_error()
        assert (r.count, r.hash, r.tasks, r.valid_roots) == (want["count"], want["hash"], want["tasks"], want["valid_roots"])
        assert r.gpu_launches >= 3


def test_noalloc_rejects_oversized_graph(kp):
    off, adj = kp.workload_graph("small")
    pre, bufs = _device_inputs(kp, off, adj, 2, 8, 0)
    fn = _noalloc(kp)
    p = kp.make_params(2, 8)
    r = kp.Result()
    rc = fn(*[b.data_ptr() for b in bufs], 50_000_000, ctypes.byref(p), ctypes.byref(r))
    assert rc == kp.ERR_NOMEM
    assert b"64 MiB" in kp.lib().kplex_last_error()


def test_noalloc_reports_leftover_work_as_timeout(kp, orc):
    """With the test hook that makes every bounded device wait give up (one pool slot
    is claimed and never published), the call must end with KPLEX_ERR_TIMEOUT, not
    with a short count, and the next call on the same array must be exact."""
    off, adj = orc.random_graph(80, 0.15, 3, [(20, 0.9), (18, 0.95), (16, 1.0)])
    want = kp.enumerate_csr(off, adj, 3, 8)
    pre, bufs = _device_inputs(kp, off, adj, 3, 8, 0)
    fn = _noalloc(kp)
    p = kp.make_params(3, 8, 0.25, 0, flags=kp.FLAG_QUIET | kp.FLAG_TEST_NO_WAIT)
    r = kp.Result()
    rc = fn(*[b.data_ptr() for b in bufs], pre["pn"], ctypes.byref(p), ctypes.byref(r))
    assert rc == kp.ERR_TIMEOUT and r.status == kp.ERR_TIMEOUT
    p = kp.make_params(3, 8)
    r = kp.Result()
    rc = fn(*[b.data_ptr() for b in bufs], pre["pn"], ctypes.byref(p), ctypes.byref(r))
    assert rc == 0 and (r.count, r.hash, r.tasks) == (want["count"], want["hash"], want["tasks"])
