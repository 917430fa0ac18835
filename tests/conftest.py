"""Shared fixtures.  GPU tests carry @pytest.mark.gpu and call through the C ABI."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "maximal-kplex-enumeration_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

DATASETS = os.path.join(ROOT, "datasets")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) device")
    config.addinivalue_line("markers", "slow: minutes of CPU time; run with KPLEX_SLOW=1")


def pytest_collection_modifyitems(config, items):
    if os.environ.get("KPLEX_SLOW") == "1":
        return
    skip = pytest.mark.skip(reason="slow oracle pin; set KPLEX_SLOW=1")
    for it in items:
        if "slow" in it.keywords:
            it.add_marker(skip)


def _ensure_built():
    lib = os.path.join(PKG, "libkplex.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", PKG, "-j8"], check=True)
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "-j4"], check=True)


@pytest.fixture(scope="session")
def kp():
    _ensure_built()
    import kplex_b200
    return kplex_b200


@pytest.fixture(scope="session")
def orc():
    _ensure_built()
    import oracle
    return oracle


def dataset(name):
    p = os.path.join(DATASETS, name)
    return p if os.path.exists(p) else None
