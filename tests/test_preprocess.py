"""Host preprocessing (core, truss, degeneracy) is identical to the reference's.

Compared against the oracle restatement always, and against the reference's own
compiled host code (oracle/_ref/ref_preprocess, built from the reference sources
by `make -C oracle ref`) when that binary is present."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, dataset

REF = os.path.join(ROOT, "oracle", "_ref", "ref_preprocess")
KEYS = ("off", "adj", "dpos", "dseq")


def ref_preprocess(path, k, q, tr, tmp):
    out = os.path.join(tmp, "pre.bin")
    subprocess.run([REF, path, str(k), str(q), str(tr), out], check=True, capture_output=True)
    d = np.fromfile(out, dtype=np.uint32)
    pn, m = int(d[0]), int(d[1])
    o = 2
    res = {"pn": pn, "off": d[o:o + pn + 1]}
    o += pn + 1
    res["adj"] = d[o:o + m]
    o += m
    res["dpos"] = d[o:o + pn].view(np.int32)
    o += pn
    res["dseq"] = d[o:o + pn].view(np.int32)
    return res


CASES = [("small", 2, 8, 0), ("small", 2, 8, 1), ("small", 3, 9, 1), ("small", 4, 12, 1), ("small", 3, 14, 0)]


@pytest.mark.parametrize("wl,k,q,tr", CASES)
def test_matches_oracle(kp, orc, wl, k, q, tr):
    off, adj = kp.workload_graph(wl)
    a = kp.preprocess(off, adj, k, q, tr)
    b = orc.preprocess(off, adj, k, q, tr)
    assert a["pn"] == b["pn"]
    for key in KEYS + ("orig",):
        assert np.array_equal(a[key], b[key]), key


@pytest.mark.parametrize("wl,k,q,tr", CASES)
def test_matches_reference_binary(kp, tmp_path, wl, k, q, tr):
    if not os.path.exists(REF):
        pytest.skip("reference harness not built (make -C oracle ref)")
    off, adj = kp.workload_graph(wl)
    p = str(tmp_path / "g.bin")
    kp.save_bin(p, off, adj)
    a = kp.preprocess(off, adj, k, q, tr)
    b = ref_preprocess(p, k, q, tr, str(tmp_path))
    assert a["pn"] == b["pn"]
    for key in KEYS:
        assert np.array_equal(a[key], b[key]), key


@pytest.mark.parametrize("name,k,q", [("email-euall.bin", 3, 12), ("soc-epinions.bin", 4, 30)])
@pytest.mark.parametrize("tr", [0, 1])
def test_datasets_match_reference_binary(kp, tmp_path, name, k, q, tr):
    p = dataset(name)
    if not p or not os.path.exists(REF):
        pytest.skip("dataset or reference harness missing")
    off, adj = kp.load_bin(p)
    a = kp.preprocess(off, adj, k, q, tr)
    b = ref_preprocess(p, k, q, tr, str(tmp_path))
    assert a["pn"] == b["pn"]
    for key in KEYS:
        assert np.array_equal(a[key], b[key]), key


def test_degenerate_inputs(kp, orc):
    # empty graph, graph smaller than q, a single clique
    off = np.zeros(1, np.uint32)
    adj = np.zeros(0, np.uint32)
    assert kp.preprocess(off, adj, 2, 8)["pn"] == 0
    n = 12
    rows = [[j for j in range(n) if j != i] for i in range(n)]
    off = np.zeros(n + 1, np.uint32)
    off[1:] = np.cumsum([len(r) for r in rows])
    adj = np.concatenate(rows).astype(np.uint32)
    a = kp.preprocess(off, adj, 2, 8)
    b = orc.preprocess(off, adj, 2, 8)
    assert a["pn"] == b["pn"] == n
    assert np.array_equal(a["dseq"], b["dseq"])
