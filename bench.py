#!/usr/bin/env python
"""Benchmark: maximal k-plexes per second on B200 (one JSON line on rank 0).

One step = one full enumeration of the workload graph on the device
(decomposition + k-search + branch-and-bound), with the pruned graph already
resident in HBM (`value`), and the same enumeration through the public C ABI
from host CSR arrays (`e2e`: host preprocessing, upload, search, result read).
Under torchrun each rank searches the roots whose degeneracy rank r satisfies
r % world == rank (strong scaling over one graph); the only collective is a
final all-reduce of (count, hash, device time).

--impl reference times the reference algorithm's CPU restatement (the oracle,
OpenMP over all host cores) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "maximal-kplex-enumeration_b200")
sys.path.insert(0, PKG)

import numpy as np  # noqa: E402

import kplex_b200 as kp  # noqa: E402

METRIC = "maximal k-plexes/sec"
# The reference's headline graph (its README's soc-Epinions1 run, k=4, q=30).
# The epinions-shaped synthetic graph of the same size holds too many plexes
# to enumerate in a bench step, so it is a named workload only.
DEFAULT_WORKLOAD = os.path.join(ROOT, "datasets", "soc-epinions.bin") + ":4:30:0"
UNIT = "plexes/s"


def read_bin(path: str):
    """The reference's .bin layout (inc/graph.h:45-62): u32 n, u32 m, u32 degree[n],
    then the neighbour lists.  Read with numpy so that the reference arm loads no
    library of this repository."""
    raw = np.fromfile(path, dtype=np.uint32)
    n, m = int(raw[0]), int(raw[1])
    if raw.size != 2 + n + m:
        raise ValueError(f"{path}: size does not match its header")
    off = np.zeros(n + 1, np.uint32)
    off[1:] = np.cumsum(raw[2:2 + n], dtype=np.uint64).astype(np.uint32)
    return off, raw[2 + n:].copy()


def load_workload(name: str, numpy_reader: bool = False):
    if name in kp.WORKLOADS:
        w = kp.WORKLOADS[name]
        off, adj = kp.workload_graph(name)
        return off, adj, dict(workload=f"{name}-shaped synthetic" if name != "small" else "small synthetic",
                              seed=w["spec"]["seed"], n=int(len(off) - 1), m_directed=int(len(adj)),
                              k=w["k"], q=w["q"], t=w["thres"], truss=w["truss"])
    if name.startswith("batch:"):   # graph i of the batched workload, alone
        i = int(name.split(":")[1])
        off, adj, k, q = kp.batch_graph(i, 4)
        return off, adj, dict(workload=f"batched-workload graph {i} (seed 4)", n=int(len(off) - 1),
                              m_directed=int(len(adj)), k=k, q=q, t=0.25, truss=0)
    # a real .bin graph: name = path:k:q:truss
    path, k, q, tr = name.split(":")
    off, adj = read_bin(path) if numpy_reader else kp.load_bin(path)
    return off, adj, dict(workload=os.path.basename(path) + f" k={k} q={q} truss={tr}", n=int(len(off) - 1),
                          m_directed=int(len(adj)),
                          k=int(k), q=int(q), t=0.25, truss=int(tr), input=os.path.relpath(path, ROOT))


def data_kind(cfg) -> str:
    if "synthetic" in cfg["workload"]:
        return "synthetic (seeded Chung-Lu + planted dense groups)"
    return "real graph file (.bin)"


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict | None:
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def allreduce_results(dist, count: int, hsum: int, ms: float, device) -> tuple[int, int, float]:
    """Whole-graph (count, hash) = sums over root shards (hash mod 2^64); time = max over ranks."""
    import torch
    mx = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    signed = hsum - (1 << 64) if hsum >= (1 << 63) else hsum
    tot = torch.tensor([count, signed], dtype=torch.int64, device=device)
    dist.all_reduce(tot)
    return int(tot[0].item()), int(tot[1].item()) & ((1 << 64) - 1), float(mx.item())


def cpu_sample(off, adj, cfg, budget_s: float = 20.0, stride: int | None = None):
    """Oracle (OpenMP, all host cores) on a stratified root sample of the workload:
    the roots whose degeneracy rank r has r % stride == 0, spread over the whole
    order so that the sample's plexes per second stand for the whole graph's.  The
    stride starts near nroots / 8 and halves (doubling the sample) until one run
    takes budget_s / 4, or is `stride` when given.  Returns the baseline dict and
    the stride used."""
    sys.path.insert(0, ROOT)
    import oracle  # CPU baseline only

    pre = oracle.preprocess(off, adj, cfg["k"], cfg["q"], cfg["truss"])
    nroots = max(1, pre["pn"] - cfg["q"] + 2)
    fixed = stride is not None
    if not fixed:
        stride = 1
        while stride * 16 <= nroots:
            stride *= 2
    while True:
        t0 = time.perf_counter()
        r = oracle.enumerate_shard(off, adj, cfg["k"], cfg["q"], cfg["truss"], 0, stride, threads=0)
        el = time.perf_counter() - t0
        if fixed or el >= budget_s / 4 or stride == 1:
            break
        stride //= 2
    nsample = (nroots + stride - 1) // stride
    return {"value": r["count"] / el if el > 0 else 0.0, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": f"roots of degeneracy rank r % {stride} == 0 ({nsample} of {nroots}, spread over the whole "
                      f"order): {r['count']} plexes in {el:.2f} s (oracle restatement, preprocessing included, "
                      f"all {os.cpu_count()} host threads)"}, stride


def cudaplex_run(cfg, timeout_s: float = 300.0):
    """The reference CudaPlex, unmodified and rebuilt for sm_100a (oracle/_ref/cudaplex,
    compile.sh:5 with -arch changed), run once on this GPU on the same graph and
    parameters, outside the timed steps.  Returns its own "Total Time Elapsed"
    (preprocessing + search, inc/host_funcs.h:747-858, 1021-1149), its count and the
    process wall time, or None when the binary or the .bin input is absent."""
    exe = os.path.join(ROOT, "oracle", "_ref", "cudaplex")
    path = os.path.join(ROOT, cfg["input"]) if cfg.get("input") else None
    if not path or not os.path.exists(exe) or not os.path.exists(path):
        return None
    cmd = [exe, path, "-k", str(cfg["k"]), "-q", str(cfg["q"]), "-t", str(cfg["t"]), "-tr", str(cfg["truss"])]
    t0 = time.perf_counter()
    try:
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout_s).stdout
    except (subprocess.TimeoutExpired, OSError) as e:
        return {"error": str(e)[:200]}
    wall = (time.perf_counter() - t0) * 1e3
    rec = {"command": " ".join(["oracle/_ref/cudaplex", os.path.relpath(path, ROOT)] + cmd[2:]), "wall_ms": wall}
    for line in out.splitlines():
        if line.startswith("Total Time Elapsed:"):
            rec["ms_ref_region"] = float(line.split(":")[1].split()[0])
        elif "Maximal k-Plexes:" in line:
            rec["count"] = int(line.rsplit(":", 1)[1])
            rec["valid_blocks"] = int(line.split("Total Valid Blocks:")[1].split(",")[0])
    return rec


def run_reference(args, cfg, off, adj):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    steps = []
    stride = None   # sized on the first (warm-up) step, then fixed
    for i in range(args.warmup + args.steps):
        cb, stride = cpu_sample(off, adj, cfg, budget_s=args.cpu_budget, stride=stride)
        if i >= args.warmup:
            steps.append(cb)
    v = statistics.median([s["value"] for s in steps])
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u32",
            "data": data_kind(cfg),
            "config": cfg, "cpu_baseline": {**steps[-1], "value": v},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_subsets(device: int, steps: int = 3):
    """Stated root ranges of the full-size synthetic workloads (the epinions-shaped and
    email-shaped graphs hold too many maximal k-plexes to enumerate whole in a bench
    step): device throughput on each, checked against the oracle's committed fixture
    (tests/golden/golden.json "subsets")."""
    import torch
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        subsets = json.load(f).get("subsets", {})
    out = {}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{device}")
    for key, s in sorted(subsets.items()):
        w = kp.WORKLOADS[s["workload"]]
        off, adj = kp.workload_graph(s["workload"])
        prep = kp.prepare(off, adj, w["k"], w["q"], w["thres"], w["truss"], device=device,
                          root_begin=s["root_begin"], root_end=s["root_end"])
        prep.search()
        res = []
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            res.append(prep.search())
        prep.release()
        dev_ms = sum(r["ms_device"] for r in res)
        t0 = time.perf_counter()
        e = kp.enumerate_csr(off, adj, w["k"], w["q"], w["thres"], w["truss"], device=device,
                             root_begin=s["root_begin"], root_end=s["root_end"])
        e2e_ms = (time.perf_counter() - t0) * 1e3
        r = res[-1]
        out[key] = {"workload": f"{s['workload']}-shaped synthetic, roots of rank [{s['root_begin']}, {s['root_end']})",
                    "value": r["count"] * steps / (dev_ms / 1e3), "unit": UNIT, "ms_per_step": dev_ms / steps,
                    "count": r["count"], "hash": f"{r['hash']:#018x}",
                    "exact_vs_oracle_fixture": (r["count"], r["hash"], r["tasks"]) == (s["count"], s["hash"], s["tasks"]),
                    "max_local_n": r["max_local_n"], "nodes": r["nodes"],
                    "e2e": {"value": e["count"] / (e2e_ms / 1e3), "unit": UNIT, "ms": e2e_ms},
                    "bnb_bytes_per_ms": r["bnb_bytes"] / r["ms_bnb"] if r["ms_bnb"] else None}
    return out


def run_sharding(args, off, adj, cfg, device: int = 0):
    """Load balance of the multi-GPU root partition, measured on one GPU: every
    shard of S in {2, 4, 8} searched in turn (each with the whole device, as it
    would have on its own GPU), for the r % S rule and for the cost-weighted
    partition.  The slowest shard bounds an S-GPU run: balance = mean / max."""
    out = {}
    for mode in ("modulo", "weighted"):
        flags = kp.FLAG_QUIET | (kp.FLAG_SHARD_WEIGHTED if mode == "weighted" else 0)
        for S in (2, 4, 8):
            ms, cnt = [], 0
            for s in range(S):
                prep = kp.prepare(off, adj, cfg["k"], cfg["q"], cfg["t"], cfg["truss"], flags=flags, device=device,
                                  shard_index=s, shard_count=S)
                prep.search()
                r = prep.search()
                prep.release()
                ms.append(r["ms_device"])
                cnt += r["count"]
            out[f"{mode}_{S}"] = {"shard_ms": ms, "max_ms": max(ms), "balance": (sum(ms) / S) / max(ms),
                                  "count": cnt}
    return out


def _pct(xs, p):
    xs = sorted(xs)
    if not xs:
        return 0.0
    i = min(len(xs) - 1, max(0, int(round(p / 100.0 * (len(xs) - 1)))))
    return xs[i]


def run_batched(args):
    """4,096 seeded graphs (n log-uniform in [64, 2048], mixed k and q) in one launch,
    on the autotuned schedule, against one plain launch per graph."""
    import torch
    torch.cuda.set_device(0)
    graphs = kp.batch_workload(args.batch_count, 4, q_per_k=0 if args.batch_full else 4)
    tuned, tune_ms = kp.autotune_batch(graphs, sample=min(args.tune_sample, len(graphs)))
    prep = kp.prepare_batch(graphs, **tuned)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda:0")
    for _ in range(args.warmup):
        prep.search()
        flush.zero_()
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    res = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        res.append(prep.search())
    clocks = sampler.stop()
    prep.release()
    per, tot = res[-1]
    dev_ms = sum(t["ms_device"] for _, t in res)
    # end to end: host preprocessing of every graph, upload, search, per-graph results
    t0 = time.perf_counter()
    per_e2e, tot_e2e = kp.enumerate_batch(graphs, **tuned)
    e2e_ms = (time.perf_counter() - t0) * 1e3
    # one plain launch per graph, back to back (each timed, for the tail analysis)
    seq, seq_each = [], []
    t0 = time.perf_counter()
    for (o, a, k, q) in graphs:
        t1 = time.perf_counter()
        seq.append(kp.enumerate_csr(o, a, k, q))
        seq_each.append((time.perf_counter() - t1) * 1e3)
    seq_ms = (time.perf_counter() - t0) * 1e3
    exact = all((per[i]["count"], per[i]["hash"]) == (seq[i]["count"], seq[i]["hash"]) ==
                (per_e2e[i]["count"], per_e2e[i]["hash"]) for i in range(len(graphs)))
    # where the time goes: a batched launch cannot end before its largest graph does
    order = sorted(range(len(graphs)), key=lambda i: -seq[i]["ms_device"])
    tail = {"largest_graph": {"index": order[0], "count": seq[order[0]]["count"],
                              "plain_device_ms": seq[order[0]]["ms_device"]},
            "top10_share_of_plain_device_ms": sum(seq[i]["ms_device"] for i in order[:10]) /
                                              max(1e-9, sum(r["ms_device"] for r in seq)),
            "plain_device_ms_total": sum(r["ms_device"] for r in seq),
            "plain_host_ms_total": seq_ms - sum(r["ms_device"] for r in seq),
            "batched_device_ms": dev_ms / args.steps,
            "batched_warp_share": {x: tot[x + "_warp_ms"] / (tot["search_warps"] * tot["ms_bnb"])
                                   if tot["search_warps"] and tot["ms_bnb"] else None for x in ("bnb", "ks", "idle")}}
    orig = batch_original_subset(tuned)
    count = tot["count"]
    h2d = sum(4 * (len(o) + len(a)) for (o, a, _, _) in graphs)
    line = {"metric": METRIC + " (batched)", "value": count * args.steps / (dev_ms / 1e3), "unit": UNIT,
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded Chung-Lu + planted dense groups)",
            "config": {"workload": f"{len(graphs)} graphs, seed 4, n log-uniform [64, 2048], k in {{2,3,4}}, q in [8, 20]"
                                   + ("" if args.batch_full else ", q raised to >= 4k"),
                       "schedule": tuned, "autotune_sample_ms": tune_ms, "l2": "256 MiB flush between steps"},
            "count": count, "exact_vs_plain": exact,
            "e2e": {"value": count / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": 20 * len(graphs), "ms_per_step": e2e_ms},
            "sequential_plain": {"value": count / (seq_ms / 1e3), "unit": UNIT, "ms": seq_ms,
                                 "launches": len(graphs)},
            "batched_e2e_over_sequential": seq_ms / e2e_ms,
            "tail": tail, "original_draws_subset": orig,
            "gpu_launches": sum(t["gpu_launches"] for _, t in res), "clocks": clocks}
    return line


def batch_original_subset(tuned):
    """The batched workload as drawn (q not raised), on the stated subset the oracle
    pins (tests/golden/golden.json "batch_original": the first 512 graphs of seed 4
    without the k=4, q<12 ones): one batched call against one plain call per graph,
    both end to end, and every graph's count and hash against the fixture."""
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        fix = json.load(f).get("batch_original")
    if fix is None:
        return None
    allg = kp.batch_workload(fix["first"], fix["seed"])
    graphs = [allg[i] for i, *_ in fix["graphs"]]
    kp.enumerate_batch(graphs, **tuned)   # warm the workspace for this shape
    t0 = time.perf_counter()
    per, tot = kp.enumerate_batch(graphs, **tuned)
    b_ms = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    seq = [kp.enumerate_csr(o, a, k, q) for (o, a, k, q) in graphs]
    s_ms = (time.perf_counter() - t0) * 1e3
    exact = all((p["count"], p["hash"]) == (s["count"], s["hash"]) == (c, h)
                for p, s, (_, _, _, c, h) in zip(per, seq, fix["graphs"]))
    return {"workload": f"{len(graphs)} graphs: the first {fix['first']} of seed {fix['seed']} "
                        f"without {fix['excluded']}, q as drawn", "count": tot["count"],
            "batched_e2e_ms": b_ms, "sequential_plain_ms": s_ms, "batched_over_sequential": s_ms / b_ms,
            "batched_device_ms": tot["ms_device"], "exact_vs_oracle_fixture": exact}


def served_requests(rate: float, duration: float, seed: int = 5):
    """Open-loop Poisson arrivals: 95% graphs drawn as in the batched workload, 5% the
    epinions graph (the shipped soc-Epinions1 when datasets/ holds it, else the small
    synthetic graph) at q=30 with k in {2, 3, 4}."""
    rng = np.random.default_rng(seed)
    times = []
    t = 0.0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= duration:
            break
        times.append(t)
    small = kp.batch_workload(len(times), seed, q_per_k=4)
    epi = DEFAULT_WORKLOAD.split(":")[0]
    big = kp.load_bin(epi) if os.path.exists(epi) else kp.workload_graph("small")
    big_name = "soc-epinions.bin" if os.path.exists(epi) else "small synthetic"
    reqs = []
    for i, at in enumerate(times):
        if rng.random() < 0.05:
            k = int(rng.integers(2, 5))
            reqs.append((at, big[0], big[1], k, 30 if big_name == "soc-epinions.bin" else 2 * k + 4, "large"))
        else:
            o, a, k, q = small[i]
            reqs.append((at, o, a, k, q, "small"))
    return reqs, big_name


def run_served(args):
    """Continuous batching server under an open-loop Poisson stream, against one
    request at a time through plain launches (FIFO queueing from the measured
    service times on the same arrival schedule)."""
    import torch
    torch.cuda.set_device(0)
    reqs, big_name = served_requests(args.rate, args.duration)
    # warm the library and both paths
    kp.enumerate_csr(reqs[0][1], reqs[0][2], reqs[0][3], reqs[0][4])
    done = {}
    sampler = ClockSampler(0)
    with kp.Server(slots=args.slots, max_batch=args.max_batch, split_grid=args.split_grid,
                   mem_budget=args.mem_budget << 30) as srv:
        sampler.start()
        t0 = time.perf_counter()
        for i, (at, o, a, k, q, _) in enumerate(reqs):
            now = time.perf_counter() - t0
            if at > now:
                time.sleep(at - now)
            srv.submit(o, a, k, q, tag=i)
            for c in srv.poll(256, 0):
                done[c["tag"]] = c
        while len(done) < len(reqs):
            for c in srv.poll(256, 1000):
                done[c["tag"]] = c
        makespan = time.perf_counter() - t0
        clocks = sampler.stop()
        st = srv.stats()
    lat = [done[i]["ms_latency"] for i in range(len(reqs))]
    total = sum(done[i]["count"] for i in range(len(reqs)))
    # plain launches, one request at a time
    svc = []
    plain = []
    for (_, o, a, k, q, _) in reqs:
        t1 = time.perf_counter()
        r = kp.enumerate_csr(o, a, k, q)
        svc.append(time.perf_counter() - t1)
        plain.append((r["count"], r["hash"]))
    free_at = 0.0
    lat_seq = []
    for (at, *_), d in zip(reqs, svc):
        start = max(at, free_at)
        free_at = start + d
        lat_seq.append((free_at - at) * 1e3)
    seq_makespan = free_at - reqs[0][0] if reqs else 0.0
    exact = all((done[i]["count"], done[i]["hash"]) == plain[i] for i in range(len(reqs)))
    line = {"metric": METRIC + " (served)", "value": total / makespan, "unit": UNIT, "n_gpus": 1,
            "steps": 1, "warmup": 1, "ms_per_step": makespan * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic stream (seeded) + " + big_name,
            "config": {"workload": f"Poisson {args.rate}/s for {args.duration}s, seed 5, 95% batched-workload graphs, "
                                   f"5% {big_name} q=30 k in {{2,3,4}}", "requests": len(reqs),
                       "slots": args.slots, "max_batch": args.max_batch, "split_grid": args.split_grid,
                       "mem_budget_gib": args.mem_budget},
            "latency_ms": {"p50": _pct(lat, 50), "p99": _pct(lat, 99), "max": max(lat) if lat else 0},
            "latency_ms_small": {"p50": _pct([l for l, r in zip(lat, reqs) if r[5] == "small"], 50),
                                 "p99": _pct([l for l, r in zip(lat, reqs) if r[5] == "small"], 99)},
            "exact_vs_plain": exact, "count": total, "server": st,
            "one_at_a_time": {"value": total / seq_makespan if seq_makespan else 0.0, "unit": UNIT,
                              "latency_ms": {"p50": _pct(lat_seq, 50), "p99": _pct(lat_seq, 99)},
                              "busy_s": sum(svc)},
            "e2e": {"value": total / makespan, "unit": UNIT,
                    "h2d_bytes_per_step": sum(4 * (len(r[1]) + len(r[2])) for r in reqs),
                    "d2h_bytes_per_step": 88 * len(reqs)},
            "clocks": clocks}
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=None,
                    help="a named synthetic workload (small, epinions, email) or path:k:q:truss; default: "
                         "the soc-Epinions1 graph at k=4, q=30 when datasets/ holds it, else small")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-subsets", action="store_true",
                    help="skip the pinned root ranges of the full-size synthetic workloads")
    ap.add_argument("--no-cudaplex", action="store_true",
                    help="skip the one run of the reference CudaPlex (oracle/_ref/cudaplex) on the same graph")
    ap.add_argument("--mode", default="plain", choices=["plain", "batched", "served"],
                    help="plain: one graph per step (the headline); batched: many graphs per launch; "
                         "served: an open-loop request stream through the server")
    ap.add_argument("--batch-count", type=int, default=4096)
    ap.add_argument("--batch-full", action="store_true",
                    help="batched: keep q < 4k (about 12 billion plexes, hours of GPU time)")
    ap.add_argument("--rate", type=float, default=80.0,
                    help="served: requests per second (one request at a time was busy 35.5 s of 60 s at 40/s, so "
                         "80/s asks for more than it can deliver)")
    ap.add_argument("--tune-sample", type=int, default=128, help="batched: graphs the autotuner times")
    ap.add_argument("--no-modes", action="store_true",
                    help="plain: skip the batched and served records that the default run adds to its line")
    ap.add_argument("--duration", type=float, default=60.0, help="served: seconds of arrivals")
    ap.add_argument("--slots", type=int, default=2)
    ap.add_argument("--max-batch", type=int, default=256)
    ap.add_argument("--no-split-grid", dest="split_grid", action="store_false",
                    help="served: give each launch the whole device instead of 1/slots of the SMs")
    ap.add_argument("--mem-budget", type=int, default=32, help="served: GiB")
    ap.add_argument("--shard-mode", default="weighted", choices=["weighted", "modulo"],
                    help="multi-GPU root partition: cost-weighted (kplex_partition_roots) or r % world")
    ap.add_argument("--blocks-per-sm", type=int, default=0,
                    help="plain: 9-warp blocks per SM of the search kernel (2 or 3; 0 = the library default)")
    ap.add_argument("--stage-after", type=int, default=0,
                    help="plain: branch nodes on one root before its adjacency matrix is staged in shared memory")
    ap.add_argument("--shards", type=int, default=1,
                    help="plain, one GPU: search only the roots of rank r % shards == 0 (a small case for profiling)")
    args = ap.parse_args()
    if args.mode == "batched" and args.impl == "ours":
        print(json.dumps(run_batched(args)), flush=True)
        return
    if args.mode == "served" and args.impl == "ours":
        print(json.dumps(run_served(args)), flush=True)
        return
    if args.workload is None:
        args.workload = DEFAULT_WORKLOAD if os.path.exists(DEFAULT_WORKLOAD.split(":")[0]) else "small"

    off, adj, cfg = load_workload(args.workload, numpy_reader=args.impl == "reference")
    if args.impl == "reference":
        run_reference(args, cfg, off, adj)
        return

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    cfg.update(parallelism=f"root-shard x{world}" if world > 1 else "single GPU",
               l2="256 MiB flush between steps")
    shard_index, shard_count = (rank, world) if world > 1 else (0, args.shards if args.shards > 1 else 0)
    if shard_count and world == 1:
        cfg["shard"] = f"roots r % {shard_count} == 0 only"
    sched = dict(blocks_per_sm=args.blocks_per_sm, stage_after=args.stage_after)
    if args.blocks_per_sm or args.stage_after:
        cfg["schedule"] = {k: v for k, v in sched.items() if v}
    shard_flags = kp.FLAG_QUIET | (kp.FLAG_SHARD_WEIGHTED if world > 1 and args.shard_mode == "weighted" else 0)
    if world > 1:
        cfg["shard_mode"] = args.shard_mode
    prep = kp.prepare(off, adj, cfg["k"], cfg["q"], cfg["t"], cfg["truss"], flags=shard_flags, device=local,
                      shard_index=shard_index, shard_count=shard_count, **sched)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    for _ in range(args.warmup):
        prep.search()
        flush.zero_()
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    res = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        res.append(prep.search())
    barrier()
    clocks = sampler.stop()

    dev_ms = sum(r["ms_device"] for r in res)
    bnb_ms = sum(r["ms_bnb"] for r in res)
    bnb_bytes = sum(r["bnb_bytes"] for r in res)
    bnb_launches = sum(1 + r["pauses"] for r in res)
    launches = sum(r["gpu_launches"] for r in res)
    count = res[-1]["count"]
    hsum = res[-1]["hash"]
    consistent = all(r["count"] == count and r["hash"] == hsum for r in res)
    if world > 1:
        total_count, total_hash, dev_ms_max = allreduce_results(dist, count, hsum, dev_ms, f"cuda:{local}")
    else:
        dev_ms_max, total_count, total_hash = dev_ms, count, hsum

    # end to end through the public C ABI from host CSR arrays (rank's shard)
    e2e_ms = []
    e2e_ref = []
    e2e_count = 0
    e2e_parts = {}
    for _ in range(args.e2e_steps):
        r = kp.enumerate_csr(off, adj, cfg["k"], cfg["q"], cfg["t"], cfg["truss"], flags=shard_flags, device=local,
                             shard_index=shard_index, shard_count=shard_count, **sched)
        e2e_ms.append(r["ms_total"])
        e2e_ref.append(r["ms_ref_region"])
        e2e_count = r["count"]
        e2e_parts = {"ms_preprocess": r["ms_preprocess"], "ms_device": r["ms_device"],
                     "ms_ref_region": r["ms_ref_region"], "ms_total": r["ms_total"]}
    if world > 1:
        e = torch.tensor([max(e2e_ms)], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(e, op=dist.ReduceOp.MAX)
        e2e_max = float(e.item())
        c = torch.tensor([e2e_count], dtype=torch.int64, device=f"cuda:{local}")
        dist.all_reduce(c)
        e2e_total = int(c.item())
    else:
        e2e_max, e2e_total = (statistics.median(e2e_ms), e2e_count) if e2e_ms else (0.0, 0)
    pr = prep.pre
    h2d = 4 * ((pr["pn"] + 1) + pr["pm"] + 3 * pr["pn"])

    peak, peak_kind = measured_peak()
    achieved = (bnb_bytes / (bnb_ms / 1e3)) / 1e9 if bnb_ms > 0 else 0.0
    traffic = None
    # DRAM bytes per launch of the search kernel from an ncu capture ("key: value" lines)
    prof = os.path.join(ROOT, "profiles", "search_kernel_traffic.txt")
    if os.path.exists(prof):
        with open(prof) as f:
            pj = dict(line.split(":", 1) for line in f if ":" in line and not line.startswith("#"))
        pj = {k.strip(): v.strip() for k, v in pj.items()}
        if pj.get("workload") == cfg["workload"] and "dram_bytes_per_launch" in pj:
            traffic = float(pj["dram_bytes_per_launch"])

    # instruction issue, the resource this latency-bound search actually uses: warp
    # instructions per branch node from an ncu capture of the same kernel on a root
    # shard (profiles/search_kernel_issue.txt), times this launch's nodes, against
    # SMs x 4 schedulers x one instruction per cycle at the sampled SM clock
    issue = None
    iprof = os.path.join(ROOT, "profiles", "search_kernel_issue.txt")
    if os.path.exists(iprof) and clocks and bnb_ms > 0:
        with open(iprof) as f:
            ij = dict(line.split(":", 1) for line in f if ":" in line and not line.startswith("#"))
        ij = {k.strip(): v.strip() for k, v in ij.items()}
        if ij.get("workload") == cfg["workload"] and "inst_per_node" in ij:
            sms = torch.cuda.get_device_properties(local).multi_processor_count
            inst = float(ij["inst_per_node"]) * res[-1]["nodes"]
            cyc = (bnb_ms / max(bnb_launches, 1)) * 1e-3 * clocks["sm_mhz"] * 1e6
            issue = {"inst_per_node": float(ij["inst_per_node"]), "inst_per_launch": inst,
                     "issue_slots_per_launch": sms * 4 * cyc, "frac": inst / (sms * 4 * cyc),
                     "source": "profiles/search_kernel_issue.txt (" + ij.get("capture", "") + ")"}

    line = {
        "metric": METRIC,
        "value": total_count * args.steps / (dev_ms_max / 1e3) if dev_ms_max > 0 else 0.0,
        "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "u32",
        "data": data_kind(cfg),
        "config": cfg,
        "count": total_count, "hash": f"{total_hash:#018x}", "results_consistent": consistent,
        "roofline": {"bound": "hbm", "kernel": "search_kernel", "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak if peak else 0.0,
                     "traffic": traffic, "bytes_per_launch": bnb_bytes / max(bnb_launches, 1),
                     "ms_per_launch": bnb_ms / max(bnb_launches, 1),
                     # the search runs from L1, shared memory and L2 (traffic is about 1/30,000 of the
                     # algorithmic bytes): the limiter is instruction issue, not HBM
                     "limiter": "issue", "issue": issue},
        "e2e": {"value": e2e_total / (e2e_max / 1e3) if e2e_max > 0 else 0.0, "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 512, "ms_per_step": e2e_max, "parts": e2e_parts},
        "gpu_launches": launches,
        "device_counters": {x: res[-1][x] for x in ("tasks", "ks_tasks", "nodes", "valid_roots", "max_local_n",
                                                    "max_left", "pauses", "stage_copies", "roots_bytes", "search_warps")},
        # share of warp time in branch-and-bound nodes, in k-search, and idle (per warp-second of the launch)
        "warp_time_share": {x: (res[-1][x + "_warp_ms"] / (res[-1]["search_warps"] * res[-1]["ms_bnb"])
                                if res[-1]["search_warps"] and res[-1]["ms_bnb"] > 0 else None)
                            for x in ("bnb", "ks", "idle")},
        "phases_ms_per_step": {"decompose": sum(r["ms_decompose"] for r in res) / args.steps,
                               "ksearch": sum(r["ms_ksearch"] for r in res) / args.steps,
                               "bnb": bnb_ms / args.steps},
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_sample(off, adj, cfg, budget_s=args.cpu_budget)[0]
    if rank == 0 and world == 1 and not args.no_subsets and shard_count == 0:
        line["subsets"] = run_subsets(local)
    if rank == 0 and world == 1 and not args.no_cudaplex and shard_count == 0:
        ref = cudaplex_run(cfg)
        if ref is not None:
            line["cudaplex_sm100a"] = ref
            if "ms_ref_region" in ref and e2e_ref:
                ours_ref = statistics.median(e2e_ref)
                # the same boundary on both sides: preprocessing + device search
                line["vs_cudaplex"] = {"ref_region": ref["ms_ref_region"] / ours_ref,
                                       "wall": ref["wall_ms"] / e2e_max if e2e_max > 0 else None,
                                       "ours_ms_ref_region": ours_ref,
                                       "count_equal": ref.get("count") == (total_count & 0xffffffff)}
    prep.release()
    if rank == 0 and world == 1 and not args.no_modes and shard_count == 0:
        try:
            line["sharding"] = run_sharding(args, off, adj, cfg, local)
        except Exception as exc:
            line["sharding"] = {"error": f"{type(exc).__name__}: {exc}"[:300]}
    if rank == 0 and world == 1 and not args.no_modes and shard_count == 0:
        # the batched and served targets, measured in the same run (outside the timed steps)
        import argparse as _ap
        for key, fn, extra in (("batched", run_batched, dict(steps=2, warmup=1, tune_sample=64)),
                               ("served", run_served, {})):
            sub = _ap.Namespace(**{**vars(args), **extra})
            try:
                line[key] = fn(sub)
            except Exception as exc:   # a failing sub-record must not cost the headline line
                line[key] = {"error": f"{type(exc).__name__}: {exc}"[:300]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
