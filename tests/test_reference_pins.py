"""The committed golden values against what the reference itself printed.

`reference_runs` in golden.json holds the lines of the reference CudaPlex
(rebuilt for sm_100a) and of its hashed checker copy, run on a B200
(tests/golden/reference_runs.md, built by oracle/Makefile `ref`).  The oracle's
fixtures for the same inputs must agree on the count, the valid roots and the
project hash, so the hash is pinned by the reference and not only by this
project's own oracle."""
import json
import os

import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.json")


def _golden():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.mark.parametrize("key", ["soc-epinions.bin:4:30:0", "email-euall.bin:3:12:0", "email-euall.bin:3:12:1"])
def test_fixture_equals_reference_output(key):
    g = _golden()
    ref, ours = g["reference_runs"][key], g["datasets"][key]
    assert ours["count"] == ref["count"]
    assert ours["valid_roots"] == ref["valid_roots"]
    assert ours["hash"] == ref["hash"], (hex(ours["hash"]), hex(ref["hash"]))


def test_readme_counts():
    # README.md:142 and :144 of the reference
    g = _golden()["reference_runs"]
    assert g["soc-epinions.bin:4:30:0"]["count"] == 13172906
    assert g["email-euall.bin:3:12:0"]["count"] == 32639016
