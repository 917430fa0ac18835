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
