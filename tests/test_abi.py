"""The C-ABI library loads and exports every entry point that include/kplex.h declares."""
import os
import re
import subprocess

from conftest import PKG, ROOT


def declared():
    with open(os.path.join(ROOT, "include", "kplex.h")) as f:
        src = f.read()
    return sorted(set(re.findall(r"\b(kplex_[a-z_0-9]+)\s*\(", src)))


def test_every_declared_symbol_exported(kp):
    lib = kp.lib()
    names = declared()
    assert "kplex_enumerate_csr" in names and "kplex_load_bin" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", os.path.join(PKG, "libkplex.so")], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (kplex_\w+)", out))
    assert set(names) <= exported, set(names) - exported


def test_status_strings(kp):
    lib = kp.lib()
    for code in range(10):
        assert lib.kplex_status_string(code)
    assert lib.kplex_version() >= 1


def test_bad_params_rejected_before_device(kp):
    off, adj = kp.workload_graph("small")
    for k, q in [(1, 8), (4, 6), (40, 90)]:
        r = kp.enumerate_csr(off, adj, k, q, check=False)
        assert r["status"] == kp.ERR_PARAM, (k, q, r["status"])
    r = kp.enumerate_csr(off, adj, 2, 8, thres=0.0, check=False)
    assert r["status"] == kp.ERR_PARAM


def test_no_silent_cpu_path_without_a_device(kp):
    """Without a usable sm_100 device every device entry point fails with a status;
    nothing falls back to a CPU computation."""
    import pytest
    if kp.device_ok():
        pytest.skip("a CUDA device is present")
    off, adj = kp.workload_graph("small")
    r = kp.enumerate_csr(off, adj, 2, 8, check=False)
    assert r["status"] == kp.ERR_NO_DEVICE and r["count"] == 0
    graphs = kp.batch_workload(count=3, seed=4)
    with pytest.raises(kp.KplexError) as e:
        kp.enumerate_batch(graphs)
    assert e.value.status == kp.ERR_NO_DEVICE
    with pytest.raises(kp.KplexError) as e:
        kp.autotune_batch(graphs, sample=2)
    assert e.value.status == kp.ERR_NO_DEVICE
    with pytest.raises(kp.KplexError) as e:
        kp.Server(slots=1)
    assert e.value.status == kp.ERR_NO_DEVICE


def test_struct_layouts_match_header(kp, tmp_path):
    """The ctypes mirrors in kplex_b200.py have the sizes and field offsets the C
    compiler gives the structs of include/kplex.h (a field added on one side only
    would shift every later field)."""
    import ctypes
    structs = {"kplex_params": kp.Params, "kplex_result": kp.Result, "kplex_graph": kp.Graph, "kplex_job": kp.Job,
               "kplex_gen_spec": kp.GenSpec, "kplex_server_config": kp.ServerConfig,
               "kplex_completion": kp.Completion, "kplex_server_stats": kp.ServerStats}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "kplex.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("  return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        cname, key, val = line.split()
        got[(cname, key)] = int(val)
    for cname, py in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)
