#!/usr/bin/env python
"""Regenerates tests/golden/golden.json (the committed parity fixtures).

Sources of truth, in order:
  * README.md:142 and README.md:144 of the reference: the published counts for
    the two shipped datasets (soc-epinions k=4 q=30 -> 13,172,906;
    email-euall k=3 q=12 -> 32,639,016); the hash comes from the oracle.
  * oracle.bruteforce_csr: exhaustive enumeration without the reference's
    pruning rules, for the small random graphs.
  * oracle.enumerate_csr: the restatement of the reference algorithm, for every
    case (count, hash and the number of generated tasks, which the device path
    must reproduce because it builds the same search tree).
Usage: python tests/golden/make_golden.py [--datasets DIR] [--synthetic] [--subsets]

--subsets pins stated root ranges of the two full-size synthetic workloads,
which hold too many maximal k-plexes for the oracle to enumerate whole: the
roots of degeneracy rank r in [root_begin, root_end) (SUBSETS below).
"""
import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "maximal-kplex-enumeration_b200")]
import numpy as np  # noqa: E402

import kplex_b200 as kp  # noqa: E402
import oracle  # noqa: E402

README = {("soc-epinions.bin", 4, 30): 13172906, ("email-euall.bin", 3, 12): 32639016}

# name -> (workload, root_begin, root_end): stated root ranges of the full-size
# synthetic workloads that the oracle finishes in minutes
SUBSETS = {
    # email-shaped (k=3, q=12, truss on): 118 valid roots, two of them with more than
    # 1024 local vertices (1028 and 1137)
    "email:2560:2688": ("email", 2560, 2688),
    # epinions-shaped (k=4, q=30): two roots inside planted density-0.9 groups (local
    # subgraphs of 56 and 50 vertices; 7.4 M and 0.44 M maximal 4-plexes)
    "epinions:13158:13159": ("epinions", 13158, 13159),
    "epinions:13590:13591": ("epinions", 13590, 13591),
}


def random_cases():
    cases = []
    for seed in range(24):
        rng = np.random.default_rng(1000 + seed)
        n = int(rng.integers(24, 64))
        p = round(float(rng.uniform(0.05, 0.25)), 3)
        planted = [(int(rng.integers(8, 16)), round(float(rng.uniform(0.8, 1.0)), 3)) for _ in range(int(rng.integers(1, 4)))]
        k = int(rng.integers(2, 5))
        q = int(2 * k - 1 + rng.integers(0, 4))
        tr = int(rng.integers(0, 2))
        cases.append(dict(seed=1000 + seed, n=n, p=p, planted=planted, k=k, q=q, truss=tr))
    return cases


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--datasets", default=os.path.join(ROOT, "datasets"))
    ap.add_argument("--synthetic", action="store_true", help="also run the full-size synthetic workloads (long)")
    ap.add_argument("--subsets", action="store_true", help="pin the stated root ranges of the full-size workloads")
    ap.add_argument("--batch", action="store_true",
                    help="pin the batched workload's original draws: the first 512 graphs of seed 4 without "
                         "the k=4, q<12 ones (those hold up to hundreds of millions of plexes each)")
    args = ap.parse_args()
    dst = os.path.join(HERE, "golden.json")
    if args.batch:
        with open(dst) as f:
            gold = json.load(f)
        rows = []
        for i, (off, adj, k, q) in enumerate(kp.batch_workload(512, 4)):
            if k == 4 and q < 12:
                continue
            o = oracle.enumerate_csr(off, adj, k, q, 0)
            rows.append([i, k, q, o["count"], o["hash"]])
        gold["batch_original"] = {"seed": 4, "first": 512, "excluded": "k == 4 and q < 12", "graphs": rows}
        with open(dst, "w") as f:
            json.dump(gold, f, indent=1, sort_keys=True)
        print("batch_original:", len(rows), "graphs,", sum(r[3] for r in rows), "plexes")
        return
    if args.subsets:   # add (or refresh) the subset fixtures only
        with open(dst) as f:
            gold = json.load(f)
        gold.setdefault("subsets", {})
        for name, (wname, rb, re_) in SUBSETS.items():
            w = kp.WORKLOADS[wname]
            off, adj = kp.workload_graph(wname)
            o = oracle.enumerate_csr(off, adj, w["k"], w["q"], w["truss"], root_begin=rb, root_end=re_)
            gold["subsets"][name] = {"workload": wname, "root_begin": rb, "root_end": re_,
                                     **{k: o[k] for k in ("count", "hash", "tasks", "valid_roots", "max_n", "max_left")}}
            print(name, gold["subsets"][name], flush=True)
        with open(dst, "w") as f:
            json.dump(gold, f, indent=1, sort_keys=True)
        return
    out = {"random": [], "workloads": {}, "datasets": {}, "subsets": {}}
    for c in random_cases():
        off, adj = oracle.random_graph(c["n"], c["p"], c["seed"], [tuple(x) for x in c["planted"]])
        o = oracle.enumerate_csr(off, adj, c["k"], c["q"], c["truss"], threads=1)
        b = oracle.bruteforce_csr(off, adj, c["k"], c["q"], threads=1)
        assert (o["count"], o["hash"]) == (b["count"], b["hash"]), (c, o, b)
        out["random"].append({**c, "count": o["count"], "hash": o["hash"], "tasks": o["tasks"]})
    names = ["small"] + (["epinions", "email"] if args.synthetic else [])
    for name in names:
        w = kp.WORKLOADS[name]
        off, adj = kp.workload_graph(name)
        o = oracle.enumerate_csr(off, adj, w["k"], w["q"], w["truss"])
        rec = {k: o[k] for k in ("count", "hash", "tasks", "valid_roots", "pn", "max_n", "max_left", "truncated_roots")}
        if name == "small":
            b = oracle.bruteforce_csr(off, adj, w["k"], w["q"])
            assert (b["count"], b["hash"]) == (o["count"], o["hash"])
            rec["bruteforce"] = True
        out["workloads"][name] = rec
    for (fname, k, q), cnt in README.items():
        path = os.path.join(args.datasets, fname)
        if not os.path.exists(path):
            continue
        off, adj = kp.load_bin(path)
        for tr in (0, 1):
            o = oracle.enumerate_csr(off, adj, k, q, tr)
            assert o["count"] == cnt, (fname, tr, o["count"], cnt)
            out["datasets"][f"{fname}:{k}:{q}:{tr}"] = {k2: o[k2] for k2 in ("count", "hash", "tasks", "valid_roots", "pn")}
    old = {}
    if os.path.exists(dst):
        with open(dst) as f:
            old = json.load(f)
    for key in ("workloads", "datasets", "subsets", "reference_runs"):
        for name, rec in old.get(key, {}).items():
            out.setdefault(key, {}).setdefault(name, rec)
    with open(dst, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", dst)


if __name__ == "__main__":
    main()
