"""The .bin reader/writer (inc/graph.h:45-62 layout) and its error reporting."""
import os
import struct

import numpy as np
import pytest

from conftest import dataset


def test_round_trip(kp, tmp_path):
    off, adj = kp.workload_graph("small")
    p = str(tmp_path / "g.bin")
    kp.save_bin(p, off, adj)
    off2, adj2 = kp.load_bin(p)
    assert np.array_equal(off, off2) and np.array_equal(adj, adj2)
    raw = np.fromfile(p, dtype=np.uint32)
    n = len(off) - 1
    assert raw[0] == n and raw[1] == len(adj)
    assert np.array_equal(raw[2:2 + n], np.diff(off))
    assert np.array_equal(raw[2 + n:], adj)


def _write(p, words):
    with open(p, "wb") as f:
        f.write(struct.pack(f"<{len(words)}I", *words))


def test_malformed_files(kp, tmp_path):
    bad = {
        "truncated": [3, 4, 1, 2, 1, 1, 0],          # header says 4 entries, file has 2
        "degree_sum": [2, 2, 1, 2, 1, 0],            # degrees sum to 3 != m = 2... with file size matching m=2? no
        "id_range": [2, 2, 1, 1, 5, 0],              # neighbour 5 >= n
        "unsorted": [3, 4, 2, 1, 1, 2, 1, 0, 0],     # vertex 0 list (2, 1) descending
        "self_loop": [2, 2, 1, 1, 0, 0],             # vertex 0 adjacent to itself
    }
    for name, words in bad.items():
        p = str(tmp_path / f"{name}.bin")
        _write(p, words)
        with pytest.raises(kp.KplexError) as e:
            kp.load_bin(p)
        assert e.value.status == kp.ERR_FORMAT, name
    with pytest.raises(kp.KplexError) as e:
        kp.load_bin(str(tmp_path / "does_not_exist.bin"))
    assert e.value.status == kp.ERR_IO


def test_empty_graph(kp, tmp_path):
    p = str(tmp_path / "empty.bin")
    _write(p, [0, 0])
    off, adj = kp.load_bin(p)
    assert len(off) == 1 and len(adj) == 0


@pytest.mark.parametrize("name,n,m", [("soc-epinions.bin", 75879, 811480), ("email-euall.bin", 265009, 728962)])
def test_shipped_datasets(kp, name, n, m):
    p = dataset(name)
    if not p:
        pytest.skip("dataset not copied (tests/golden/fetch_datasets.sh)")
    off, adj = kp.load_bin(p)
    assert len(off) - 1 == n and len(adj) == m
