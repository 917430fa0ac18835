"""The drop-in CLI keeps the reference's usage text, argument handling and exit codes (main.cu:11-55)."""
import os
import subprocess

import pytest

from conftest import PKG

CLI = os.path.join(PKG, "bin", "kplex_main")


def run(*args):
    return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=120)


@pytest.fixture(scope="module", autouse=True)
def built(kp):
    if not os.path.exists(CLI):
        subprocess.run(["make", "-s", "-C", PKG, "bin/kplex_main"], check=True)


def test_usage_and_exit_codes():
    usage = "usage : ./PlexEnum <dataset> -k <k> -q <q> -t <thres> -tr <truss>"
    r = run("g.bin", "-k", "2")
    assert r.returncode == 1 and usage in r.stderr and r.stdout == ""
    r = run("g.bin", "-k", "2", "-q", "8", "-x", "1")
    assert r.returncode == 1 and usage in r.stderr
    assert r.stdout.startswith("file: g.bin\n")
    r = run("g.bin", "-k", "2", "-q", "8", "-t")
    assert r.returncode == 1


def test_header_lines_and_missing_file(tmp_path):
    r = run(str(tmp_path / "nope.bin"), "-k", "2", "-q", "8", "-t", "0.25", "-tr", "0")
    lines = r.stdout.splitlines()
    assert lines[0] == f"file: {tmp_path / 'nope.bin'}"
    assert lines[1] == "k=2,q=8,thres=0.250000, truss: 0"
    assert r.returncode == 2   # KPLEX_ERR_IO


@pytest.mark.gpu
def test_cli_output_lines(kp, tmp_path):
    off, adj = kp.workload_graph("small")
    p = str(tmp_path / "small.bin")
    kp.save_bin(p, off, adj)
    r = run(p, "-k", "2", "-q", "8", "-t", "0.25", "-tr", "0")
    assert r.returncode == 0, r.stderr
    out = r.stdout
    for key in ("n=2000, m=", "pn = 1100", "Start copying graph to GPU....", "Total Time Elapsed:",
                "Total Valid Blocks: 212, Maximal k-Plexes: 871", "Total tasks generated: 2585",
                "Kernel Launch Successfully", "Maximal k-Plexes (64-bit): 871"):
        assert key in out, key
