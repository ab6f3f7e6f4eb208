#!/usr/bin/env python3
"""Benchmark: soft-gradient global affine batch GCUPS on one B200 (and N GPUs as replicas),
against the plain GPU fill, plus p50/p99 serving latency.

Workload (the soft-gradient batch configuration, seeded synthetic stand-in for the
reference's protein fixtures): 100,000 homologous protein pairs over a 20-letter alphabet,
A of length U[100, 500], B = A with 30 % substitutions and indels at rate 0.05 per position
(geometric lengths, mean 3), plus 100,000 decoys (B shuffled); a symmetric integer matrix
(off-diagonal U{-4..3}, diagonal U{4..11}), gap_open 11, gap_extend 1 on both sides.  One
step = pos.score_and_grad() + neg.score_and_grad() + the contrastive margin gradient
pos.compute_grad() - neg.compute_grad(), float32 DP.  GCUPS = sum of len(a) * len(b) over
both batches / step time (the reference's cell definition, tools/fleetbench/arm.py:317).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

The headline arm runs the autotuned geometries (``SeqPairBatch.autotune``); the plain arm
runs the same steps with the plain fill (one fixed geometry, 32 lanes x 4 rows, one launch
per size bucket).  The serving arm streams requests (lengths log-uniform 20-5000, batch sizes
log-uniform 1-4096, B a mutated copy of A) through the continuous-batching server and, for
comparison, through plain-fill batches one request at a time, first as a burst (throughput)
then as Poisson arrivals at 70 % of the server's burst capacity (p50/p99 latency).

Prints one JSON line (rank 0).  Under torchrun every rank aligns its own copy of the
workload (weak scaling) and the margin gradients are summed over ranks (NCCL all-reduce).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

AA = "ACDEFGHIKLMNPQRSTVWY"
OPS_PER_CELL_SOFT = 32.0          # soft affine: ~10 forward + ~22 backward/gradient FP32 ops
OPS_PER_CELL_HARD = 22.0          # hard affine: 13 FP32 + 9 compare/select
FP32_LANE_OPS_PEAK = 148 * 128 * 1.965e9   # ops/s at the maximum SM clock
SOFT_DRAM_BYTES_PER_CELL = 30.2            # ncu, soft kernel 32x4 on 800+800 pairs of this workload


def measured_hbm_gbs():
    """The pool's measured copy bandwidth, when the measured peaks file is present."""
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    except (OSError, ValueError, KeyError):
        return 6650.0


# ── workload ─────────────────────────────────────────────────────────────────
def c2_matrix(rng):
    m = rng.integers(-4, 4, size=(20, 20)).astype(np.float64)
    m = np.triu(m) + np.triu(m, 1).T
    m[np.diag_indices(20)] = rng.integers(4, 12, size=20)
    return m


def _mutate_codes(rng, a, freqs, sub=0.30, indel=0.05):
    """B from A: substitutions at rate `sub`, indels at rate `indel` per position (half
    insertions, half deletions), lengths geometric with mean 3."""
    L = a.size
    b = a.copy()
    s = rng.random(L) < sub
    b[s] = rng.choice(20, size=int(s.sum()), p=freqs)
    ev = np.nonzero(rng.random(L) < indel)[0]
    if ev.size == 0:
        return b
    parts = []
    prev = 0
    for pos in ev:
        if pos < prev:
            continue
        k = int(rng.geometric(1.0 / 3.0))
        if rng.random() < 0.5:   # insertion after pos
            parts.append(b[prev:pos + 1])
            parts.append(rng.choice(20, size=k, p=freqs).astype(np.uint8))
            prev = pos + 1
        else:                    # deletion of k residues from pos
            parts.append(b[prev:pos])
            prev = min(L, pos + k)
    parts.append(b[prev:])
    return np.concatenate(parts).astype(np.uint8)


def c2_workload(n_pairs, seed=1, lmax=500):
    """(mat, codes_a, off_a, codes_b_pos, off_b_pos, codes_b_neg, off_b_neg); lmax < 500 caps A's
    length (profiling cases of the same distribution that still fill the device)."""
    cache = os.path.join("/tmp", f"nwgrad_b200_c2_{n_pairs}_{seed}_{lmax}.npz")
    if os.path.exists(cache):
        z = np.load(cache)
        return tuple(z[k] for k in ("mat", "a", "oa", "bp", "obp", "bn", "obn"))
    rng = np.random.default_rng(seed)
    freqs = rng.dirichlet(np.full(20, 5.0))
    mat = c2_matrix(rng)
    la = rng.integers(100, lmax + 1, size=n_pairs)
    oa = np.zeros(n_pairs + 1, np.int64)
    oa[1:] = np.cumsum(la)
    a = rng.choice(20, size=int(oa[-1]), p=freqs).astype(np.uint8)
    bs = [_mutate_codes(rng, a[oa[p]:oa[p + 1]], freqs) for p in range(n_pairs)]
    obp = np.zeros(n_pairs + 1, np.int64)
    obp[1:] = np.cumsum([x.size for x in bs])
    bp = np.concatenate(bs)
    bn = np.concatenate([rng.permutation(x) for x in bs])
    obn = obp.copy()
    try:
        np.savez(cache, mat=mat, a=a, oa=oa, bp=bp, obp=obp, bn=bn, obn=obn)
    except OSError:
        pass
    return mat, a, oa, bp, obp, bn, obn


def c1_workload(n_pairs=10000, seed=0):
    """Plain global affine hard batch: A and B independent, lengths U[50, 300]."""
    rng = np.random.default_rng(seed)
    freqs = rng.dirichlet(np.full(20, 5.0))
    mat = c2_matrix(rng)
    la = rng.integers(50, 301, size=n_pairs)
    lb = rng.integers(50, 301, size=n_pairs)
    oa = np.zeros(n_pairs + 1, np.int64); oa[1:] = np.cumsum(la)
    ob = np.zeros(n_pairs + 1, np.int64); ob[1:] = np.cumsum(lb)
    a = rng.choice(20, size=int(oa[-1]), p=freqs).astype(np.uint8)
    b = rng.choice(20, size=int(ob[-1]), p=freqs).astype(np.uint8)
    return mat, a, oa, b, ob


def c5_requests(n_req, seed=5, max_batch=4096, lmin=20, lmax=5000):
    """Serving requests: batch size log-uniform 1..max_batch, A lengths log-uniform lmin-lmax,
    B = A with 30 % substitutions and single-residue insertions / deletions at 2.5 % each."""
    rng = np.random.default_rng(seed)
    freqs = rng.dirichlet(np.full(20, 5.0))
    out = []
    for _ in range(n_req):
        k = min(max_batch, int(np.exp(rng.uniform(0.0, np.log(max_batch + 1)))))
        la = np.exp(rng.uniform(np.log(lmin), np.log(lmax), size=k)).astype(np.int64)
        oa = np.zeros(k + 1, np.int64)
        np.cumsum(la, out=oa[1:])
        a = rng.choice(20, size=int(oa[-1]), p=freqs).astype(np.uint8)
        b = a.copy()
        s = rng.random(b.size) < 0.30
        b[s] = rng.choice(20, size=int(s.sum()), p=freqs)
        keep = (rng.random(b.size) >= 0.025).astype(np.int64)
        ins = rng.random(b.size) < 0.025
        cnt = keep + ins
        cnt[oa[1:] - 1] = np.maximum(cnt[oa[1:] - 1], 1)     # no pair's B comes out empty
        bb = b[np.repeat(np.arange(b.size), cnt)]
        last = np.cumsum(cnt) - 1
        bb[last[ins]] = rng.choice(20, size=int(ins.sum()), p=freqs)
        ob = np.zeros(k + 1, np.int64)
        np.cumsum(np.add.reduceat(cnt, oa[:-1]), out=ob[1:])
        out.append((a, oa, bb.astype(np.uint8), ob))
    return out


def cells_of(oa, ob):
    return float(np.sum(np.diff(oa).astype(np.float64) * np.diff(ob).astype(np.float64)))


# ── clocks ───────────────────────────────────────────────────────────────────
class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, max, throttle reasons)."""

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[3 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ── the reference's CPU path ─────────────────────────────────────────────────
def cpu_reference(mat, a, oa, bp, obp, bn, obn, sample_pairs, steps, warmup):
    """Time the reference's own batch path (SeqPairBatchT<float>, soft, its default fill and
    SIMD kernels, all physical host cores) on the first `sample_pairs` pairs of each batch,
    in its own process (oracle/_ref/nwref_bench)."""
    import oracle
    if not oracle.ref_bench_available():
        return None
    k = sample_pairs
    cells = cells_of(oa[:k + 1], obp[:k + 1]) + cells_of(oa[:k + 1], obn[:k + 1])
    gaps = np.array([[11.0, 1.0, 11.0, 1.0]])
    tp, _, threads, isa = oracle.ref_time_codes(32, 1, 0, 2, AA, mat[None], gaps, a, oa[:k + 1], bp, obp[:k + 1],
                                                warmup=warmup, reps=steps)
    tn, _, _, _ = oracle.ref_time_codes(32, 1, 0, 2, AA, mat[None], gaps, a, oa[:k + 1], bn, obn[:k + 1],
                                        warmup=warmup, reps=steps)
    per_step = tp + tn
    return {"cells": cells, "seconds": per_step.tolist(), "threads": threads, "isa": isa,
            "value": cells / float(np.min(per_step)) / 1e9}


def parity_sample(batches, a, oa, mat, per_bin=250, seed=11):
    """Checker of the timed workload's own results: a stratified sample of pairs of each batch
    (per_bin pairs with A in each of 100-199, 200-299, 300-399, 400-500) recomputed by the CPU
    oracle (double, log space, several host threads), against the per-pair scores and expected
    counts the GPU left in the batches.  Returns the largest relative errors: scores against
    max(|log Z|, 1), counts against each pair's largest count (the parity tests' convention)."""
    import concurrent.futures as cf
    import oracle
    rng = np.random.default_rng(seed)
    la = np.diff(oa)
    gaps = np.array([[11.0, 1.0, 11.0, 1.0]])
    err_s = err_g = 0.0
    n_checked = refused = 0
    for b, bcodes, ob in batches:
        idx = []
        for lo, hi in ((100, 200), (200, 300), (300, 400), (400, 501)):
            cand = np.nonzero((la >= lo) & (la < hi))[0]
            idx.extend(rng.choice(cand, size=min(per_bin, cand.size), replace=False).tolist())
        idx = np.sort(np.asarray(idx, np.int64))
        s_gpu = b.scores()[idx]
        gm, gg = b.grads()
        g_gpu = np.concatenate([gm[idx].reshape(idx.size, -1), gg[idx].reshape(idx.size, -1)], axis=1)
        refused += int(np.count_nonzero(b.soft_status()[idx] & 0xff))
        A = [a[oa[i]:oa[i + 1]].tolist() for i in idx]
        B = [bcodes[ob[i]:ob[i + 1]].tolist() for i in idx]

        def run(lo):
            enc = oracle.Encoded(A[lo:lo + 25], B[lo:lo + 25])
            return oracle.soft(1, 0, mat[None], gaps, enc)
        with cf.ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
            parts = list(ex.map(run, range(0, idx.size, 25)))
        so = np.concatenate([p[0] for p in parts])
        go = np.concatenate([p[1] for p in parts])
        err_s = max(err_s, float(np.max(np.abs(s_gpu - so) / np.maximum(np.abs(so), 1.0))))
        scale = np.maximum(np.abs(go).max(axis=1, keepdims=True), 1.0)
        err_g = max(err_g, float(np.max(np.abs(g_gpu - go) / scale)))
        n_checked += idx.size
    return {"pairs": n_checked, "max_rel_err_scores": err_s, "max_rel_err_counts": err_g, "tol": 1e-4,
            "ok": bool(err_s <= 1e-4 and err_g <= 1e-4), "float32_refused_to_double": refused,
            "oracle": "CPU oracle, double log-space forward-backward",
            "sample": f"{per_bin} pairs per A-length bin (100-199 .. 400-500) of each batch, seeded"}


def _tune_mod():
    from nwgrad_b200 import tune
    return tune


def cpu_model():
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ── serving ──────────────────────────────────────────────────────────────────
def _quantiles(lat):
    v = np.sort(np.asarray(lat, np.float64))
    q = lambda f: float(v[min(v.size, max(1, int(np.ceil(f * v.size)))) - 1]) if v.size else None  # noqa: E731
    return q(0.50), q(0.99)


def serve_server(params, reqs, arrivals, device, workers=3):
    """Requests through the continuous-batching server; arrivals in seconds from the start
    (all zero: a burst).  Returns (p50 ms, p99 ms, GCUPS over the makespan, batches)."""
    import queue
    from nwgrad_b200.serve import Server
    q = queue.Queue()
    lat = []
    cells = sum(cells_of(oa, ob) for _, oa, _, ob in reqs)

    def waiter(srv):
        while True:
            item = q.get()
            if item is None:
                return
            t, k = item
            lat.append(srv.wait(t, k)[2])

    with Server(params, grad_mode="soft", workers=workers, hbm_budget_gb=96.0, max_batch_pairs=16384,
                device=device) as srv:
        th = threading.Thread(target=waiter, args=(srv,), daemon=True)
        th.start()
        t0 = time.perf_counter()
        for (a, oa, b, ob), at in zip(reqs, arrivals):
            d = at - (time.perf_counter() - t0)
            if d > 0:
                time.sleep(d)
            q.put((srv.submit_codes(a, oa, b, ob), len(oa) - 1))
        q.put(None)
        th.join()
        span = time.perf_counter() - t0
        st = srv.stats()
    p50, p99 = _quantiles(lat)
    return {"p50_ms": p50, "p99_ms": p99, "gcups": cells / span / 1e9, "seconds": span,
            "batches": int(st["batches"]), "requests": len(reqs),
            "device_overlap": st["device_overlap"], "device_busy_ms": st["device_busy_ms"],
            "device_sum_ms": st["device_sum_ms"]}


def serve_plain(params, reqs, arrivals, device):
    """The same requests through plain-fill batches, one request at a time in arrival order
    (upload, align, read back): latency = done - arrival."""
    import nwgrad_b200 as nw
    lat = []
    cells = sum(cells_of(oa, ob) for _, oa, _, ob in reqs)
    t0 = time.perf_counter()
    for (a, oa, b, ob), at in zip(reqs, arrivals):
        d = at - (time.perf_counter() - t0)
        if d > 0:
            time.sleep(d)
        bt = nw.SeqPairBatch.from_codes(a, oa, b, ob, params, grad_mode="soft", device=device)
        bt.use_plain_fill()
        bt.score_and_grad()
        bt.scores()
        bt.compute_grad()
        lat.append((time.perf_counter() - t0 - at) * 1e3)
        del bt
    span = time.perf_counter() - t0
    p50, p99 = _quantiles(lat)
    return {"p50_ms": p50, "p99_ms": p99, "gcups": cells / span / 1e9, "seconds": span, "requests": len(reqs)}


def serve_bench(params, n_req, device, seed=5, n_lat=10000):
    reqs = c5_requests(n_req, seed=seed)
    cells = sum(cells_of(oa, ob) for _, oa, _, ob in reqs)
    burst = [0.0] * len(reqs)
    # warm both paths (library, pools, plans) on a few requests
    serve_server(params, reqs[:8], burst[:8], device)
    serve_plain(params, reqs[:8], burst[:8], device)
    srv_burst = serve_server(params, reqs, burst, device)
    plain_burst = serve_plain(params, reqs, burst, device)
    # Poisson arrivals at 70 % of the server's own capacity (its burst throughput); the plain
    # one-at-a-time arm gets the same arrivals, which it cannot keep up with
    rate = 0.7 * len(reqs) / srv_burst["seconds"]
    rng = np.random.default_rng(seed + 1000)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(reqs))).tolist()
    srv_poisson = serve_server(params, reqs, arrivals, device)
    plain_poisson = serve_plain(params, reqs, arrivals, device)
    return {"requests": len(reqs), "pairs": int(sum(len(oa) - 1 for _, oa, _, _ in reqs)), "cells": cells,
            "workload": "lengths log-uniform 20-5000, batch sizes log-uniform 1-4096, B = A mutated "
                        "(30% subs, 2.5% ins, 2.5% del), soft global affine f32",
            "offered_rate_per_s": rate,
            "server": {"burst": srv_burst, "poisson": srv_poisson, "workers": 3},
            "plain_fill_one_at_a_time": {"burst": plain_burst, "poisson": plain_poisson},
            "latency": serve_latency(params, n_lat, device, seed=seed + 7)}


def serve_latency(params, n_req, device, seed=12, load=0.8, n_plain=2000):
    """Latency arm at the small end of the serving distribution (lengths log-uniform 20-300,
    batch sizes log-uniform 1-64): the server's capacity from a burst of all n_req requests,
    then Poisson arrivals at `load` of that capacity through the server (p50 / p99 over n_req
    requests) and, for comparison, the first n_plain of the same arrivals through plain-fill
    batches one request at a time."""
    reqs = c5_requests(n_req, seed=seed, max_batch=64, lmin=20, lmax=300)
    burst = [0.0] * len(reqs)
    serve_server(params, reqs[:64], burst[:64], device)
    serve_plain(params, reqs[:16], burst[:16], device)
    cap = serve_server(params, reqs, burst, device)
    rate = load * len(reqs) / cap["seconds"]
    rng = np.random.default_rng(seed + 1000)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(reqs))).tolist()
    srv = serve_server(params, reqs, arrivals, device)
    plain = serve_plain(params, reqs[:n_plain], arrivals[:n_plain], device)
    return {"requests": len(reqs), "workload": "lengths log-uniform 20-300, batch sizes log-uniform 1-64, "
                                               "B = A mutated, soft global affine f32",
            "capacity_req_per_s": len(reqs) / cap["seconds"], "offered_rate_per_s": rate, "load": load,
            "server_burst": cap, "server_poisson": srv,
            "plain_fill_one_at_a_time_poisson": dict(plain, note=f"first {n_plain} arrivals")}


# ── main ─────────────────────────────────────────────────────────────────────
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--pairs", type=int, default=100000, help="pairs per batch (positives; as many decoys)")
    ap.add_argument("--cpu-sample", type=int, default=4000, help="pairs per batch in the CPU-baseline sample")
    ap.add_argument("--lmax", type=int, default=500, help="longest A (profiling cases; the workload is 100-500)")
    ap.add_argument("--scratch-gb", type=float, default=-1,
                    help="soft scratch budget per batch in GiB (default: the library's, from free memory)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-fill arm")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving arm")
    ap.add_argument("--serve-requests", type=int, default=200)
    ap.add_argument("--no-tune", action="store_true", help="the planner's geometries instead of the autotuner's")
    ap.add_argument("--checkpoint-mb", type=float, default=-1,
                    help="soft: per-pair forward tables above this many MiB are checkpointed (-1: default)")
    ap.add_argument("--geometry", default=None, help="LANESxROWS for every pair (no tuning), e.g. 32x4")
    ap.add_argument("--workload", default="c2-soft",
                    choices=["c2-soft", "c1-hard", "c4-long", "c3-short", "c5-serve-train", "c6-glocal"],
                    help="c2-soft (default): the soft-gradient batch; side measurements: c1-hard (plain hard "
                         "batch), c4-long (64 long pairs: Pointers, Hirschberg, soft, banded), c3-short "
                         "(many short local linear tracked pairs, hard and soft), c5-serve-train (the "
                         "server under a Poisson stream while an autograd loop trains the parameters), "
                         "c6-glocal (miRNA-like A within longer B, glocal ends, hard and soft)")
    ap.add_argument("--glocal-pairs", type=int, default=200_000)
    ap.add_argument("--long-pairs", type=int, default=64)
    ap.add_argument("--short-pairs", type=int, default=10_000_000)
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the other configurations' measurements (hard batch, short pairs, long pairs, "
                         "serve + train) in the default run")
    ap.add_argument("--train-pairs", type=int, default=2000, help="c5-serve-train: homolog pairs (as many decoys)")
    ap.add_argument("--train-steps", type=int, default=200)
    args = ap.parse_args()
    side = {"c1-hard": bench_c1, "c4-long": bench_c4, "c3-short": bench_c3, "c5-serve-train": bench_c5,
            "c6-glocal": bench_c6}
    if args.workload in side:
        print(json.dumps(side[args.workload](args)))
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    mat, a, oa, bp, obp, bn, obn = c2_workload(args.pairs, seed=1, lmax=args.lmax)
    cells = cells_of(oa, obp) + cells_of(oa, obn)
    config = {"workload": "soft-gradient global affine batch, float32 DP: 100k homologous protein pairs "
                          "(L 100-500, 30% subs, indels 0.05) + 100k shuffled decoys, margin gradient",
              "pairs": 2 * args.pairs, "cells_per_step": cells, "alphabet": 20, "gap_open": 11,
              "gap_extend": 1, "l2": "inputs+scratch > L2 and a 256 MiB L2 flush between timed steps",
              "parallelism": f"replicas x{world}"}

    if args.impl == "reference":
        if rank != 0:
            return
        r = cpu_reference(mat, a, oa, bp, obp, bn, obn, args.cpu_sample, max(args.steps, 1),
                          max(args.warmup, 1))
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libnwref.so is not built"}))
            return
        v = r["value"]
        best = float(np.min(r["seconds"]))
        print(json.dumps({
            "impl": "reference", "metric": "soft-grad batch GCUPS", "value": v, "unit": "GCUPS",
            "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "ms_per_step": best * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)", "config": dict(config, cpu_sample_pairs=2 * args.cpu_sample),
            "cpu_baseline": {"value": v, "unit": "GCUPS", "cores": r["threads"], "kind": "reference",
                             "sample": f"{2 * args.cpu_sample} pairs ({r['cells']:.3g} cells) of the workload, "
                                       f"best of {len(r['seconds'])}, {cpu_model()}, isa {r['isa']}"},
            "e2e": {"value": v, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    import torch
    import nwgrad_b200 as nw

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    params = nw.AlignParams.from_arrays(mat[None], [[11.0, 1.0, 11.0, 1.0]], alphabet=nw.AA20)
    pos = nw.SeqPairBatch.from_codes(a, oa, bp, obp, params, grad_mode="soft", device=local)
    neg = nw.SeqPairBatch.from_codes(a, oa, bn, obn, params, grad_mode="soft", device=local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    if args.checkpoint_mb >= 0:
        for b in (pos, neg):
            b.set_memory(checkpoint_bytes=int(args.checkpoint_mb * (1 << 20)))
    if args.scratch_gb > 0:
        for b in (pos, neg):
            b.set_memory(scratch_budget_bytes=int(args.scratch_gb * (1 << 30)))
    tune_table = {}
    if args.geometry:
        geo = tuple(int(x) for x in args.geometry.lower().split("x"))
        pos._tune = neg._tune = geo
        args.no_tune = True
        tune_table = {"all": geo}
    elif not args.no_tune:
        tune_table = pos.autotune()
        neg.autotune()

    def step():
        pos.score_and_grad()
        neg.score_and_grad()
        g = pos.compute_grad() - neg.compute_grad()
        return g

    def allreduce(g):
        if dist is None:
            return g
        from nwgrad_b200.replicas import allreduce_grad
        return allreduce_grad(g, device=torch.device("cuda", local))

    def timed(sample_clocks):
        for _ in range(max(args.warmup, 3)):
            allreduce(step())
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
        kernel_ms = 0.0
        launches = 0
        cap0 = pos.graph_stats()[0] + neg.graph_stats()[0]
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        clk = ClockSampler(local) if sample_clocks else None
        if clk:
            clk.__enter__()
        try:
            for k in range(args.steps):
                flush.zero_()                        # L2 flush, outside the timed events
                torch.cuda.synchronize()
                ev[k][0].record()
                allreduce(step())
                ev[k][1].record()
                for b in (pos, neg):
                    ms_b, l_b = b.last_timing()
                    kernel_ms += ms_b
                    launches += l_b
                launches += 4                        # two reductions per compute_grad
            torch.cuda.synchronize()
        finally:
            if clk:
                clk.__exit__()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        step_ms = [e[0].elapsed_time(e[1]) for e in ev]
        if clk:
            clk.captures = pos.graph_stats()[0] + neg.graph_stats()[0] - cap0   # graphs captured while timed
        total_ms = float(np.sum(step_ms))
        if dist is not None:
            t = torch.tensor([total_ms], dtype=torch.float64, device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            total_ms = float(t.item())
        return total_ms, step_ms, kernel_ms, launches, clk

    total_ms, step_ms, kernel_ms, launches, clk = timed(True)
    value = world * cells * args.steps / (total_ms / 1e3) / 1e9
    plain = None
    if not args.no_plain:
        # plain and tuned interleaved, three runs of K steps each (the headline is the first
        # tuned run above): the tuner's gain against run-to-run spread
        saved = pos._tune
        gc = lambda ms: world * cells * args.steps / (ms / 1e3) / 1e9   # noqa: E731
        runs = {"plain": [], "tuned": [value]}
        p_kms = 0.0
        for rep in range(3):
            pos._tune = neg._tune = (0, 0)
            pos.use_plain_fill()
            neg.use_plain_fill()
            p_total, _, p_kms_r, _, _ = timed(False)
            runs["plain"].append(gc(p_total))
            p_kms += p_kms_r
            pos._tune = neg._tune = saved
            if not args.no_tune:
                pos.autotune()
                neg.autotune()
            if rep < 2:
                runs["tuned"].append(gc(timed(False)[0]))
        med = {k: float(np.median(v)) for k, v in runs.items()}
        plain = {"value": med["plain"], "unit": "GCUPS", "kernel_ms_per_step": p_kms / (3 * args.steps),
                 "geometry": "32 lanes x 4 rows for every pair, one launch per size bucket",
                 "runs": runs, "median": med,
                 "range": {k: [float(min(v)), float(max(v))] for k, v in runs.items()},
                 "tuned_over_plain": med["tuned"] / med["plain"]}

    # end to end through the public API: host codes uploaded, aligned, gradient read back
    e2e = None
    if not args.no_e2e:
        h2d = int(a.nbytes + bp.nbytes + bn.nbytes + 3 * oa.nbytes)
        gs = params.num_sets * (20 * 20 + 4)
        d2h = int(2 * gs * 8 + 8)
        # the step's inputs in pinned host memory (a loader's staging buffers): the library
        # copies them to HBM inside the timed region at DMA speed
        keep = []

        def pinned(x):
            t = torch.empty(x.shape, dtype=torch.from_numpy(x[:0]).dtype, pin_memory=True)
            v = t.numpy()
            v[...] = x
            keep.append(t)
            return v
        ha, hoa, hbp, hobp, hbn, hobn = (pinned(x) for x in (a, oa, bp, obp, bn, obn))
        e2e_ms = []
        for k in range(max(1, min(args.steps, 3))):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            p_ = nw.SeqPairBatch.from_codes(ha, hoa, hbp, hobp, params, grad_mode="soft", device=local)
            n_ = nw.SeqPairBatch.from_codes(ha, hoa, hbn, hobn, params, grad_mode="soft", device=local)
            if args.geometry:
                p_._tune = n_._tune = pos._tune
            elif not args.no_tune:
                p_.autotune()
                n_.autotune()
            s = p_.score_and_grad() - n_.score_and_grad()
            g = p_.compute_grad() - n_.compute_grad()
            allreduce(g)
            torch.cuda.synchronize()
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
            del p_, n_
        em = float(np.min(e2e_ms))
        if dist is not None:
            t = torch.tensor([em], dtype=torch.float64, device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            em = float(t.item())
        e2e = {"value": world * cells / (em / 1e3) / 1e9, "unit": "GCUPS", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": em,
               "path": "SeqPairBatch.from_codes (pinned host codes -> HBM) + autotune (cached table) + "
                       "score_and_grad + compute_grad"}

    clocks = clk.summary()
    # roofline of the soft kernel: algorithmic FP32 ops per cell over the kernels' device time
    kernel_s = kernel_ms / 1e3
    ach = cells * args.steps * OPS_PER_CELL_SOFT / kernel_s / 1e12 if kernel_s > 0 else None
    # DRAM traffic of one launch (one batch): bytes per cell from an ncu capture of the same
    # kernel on a small case (dram__bytes_read.sum + dram__bytes_write.sum over its cells),
    # scaled by this launch's cells (the forward table is per cell)
    traffic = SOFT_DRAM_BYTES_PER_CELL * cells / 2.0
    kernel_launch_s = kernel_s / (2 * args.steps) if kernel_s > 0 else None
    hbm_peak = measured_hbm_gbs()
    hbm = {"achieved": traffic / kernel_launch_s / 1e9 if kernel_launch_s else None, "peak": hbm_peak,
           "unit": "GB/s", "frac": (traffic / kernel_launch_s / 1e9 / hbm_peak) if kernel_launch_s and hbm_peak else None,
           "peak_note": "measured copy bandwidth (of measured)"}
    roofline = {"bound": "alu", "achieved": ach, "peak": FP32_LANE_OPS_PEAK / 1e12, "unit": "TOP/s",
                "frac": (ach / (FP32_LANE_OPS_PEAK / 1e12)) if ach else None, "traffic": traffic, "hbm": hbm,
                "peak_note": "FP32 lane-op peak 148 SM x 128 lanes x 1.965 GHz (the recurrence is max-plus / "
                             "sum-product: no tensor-core contraction)",
                "ops_per_cell": OPS_PER_CELL_SOFT, "kernel_ms_per_step": kernel_ms / args.steps}
    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the CPU leg: the oracle checks the timed batches' own results on a stratified sample,
        # then the reference's CPU path is timed on a sample of the same workload
        pos.score_and_grad()          # the tuned geometries' results (the plain arm ran last)
        neg.score_and_grad()
        parity = parity_sample([(pos, bp, obp), (neg, bn, obn)], a, oa, mat)
        r = cpu_reference(mat, a, oa, bp, obp, bn, obn, args.cpu_sample, 2, 1)
        if r is not None:
            cpu = {"value": r["value"], "unit": "GCUPS", "cores": r["threads"], "kind": "reference",
                   "sample": f"{2 * args.cpu_sample} pairs ({r['cells']:.3g} cells) of the workload, best of "
                             f"{len(r['seconds'])}, {cpu_model()}, isa {r['isa']}"}
    serve = None
    if rank == 0 and world == 1 and not args.no_serve and args.serve_requests > 0:
        serve = serve_bench(params, args.serve_requests, local)
    extras = None
    if rank == 0 and world == 1 and not args.no_extras:
        # the other configurations, each measured on its own inputs after the headline's
        import copy
        extras = {}
        for name, fn, over in (("c1_hard_batch", bench_c1, {}), ("c3_short_pairs", bench_c3, {}),
                               ("c4_long_pairs", bench_c4, {}), ("c5_serve_train", bench_c5, {"serve_requests": 60})):
            a2 = copy.copy(args)
            for k, v in over.items():
                setattr(a2, k, v)
            t0 = time.perf_counter()
            extras[name] = fn(a2)
            extras[name]["wall_s"] = time.perf_counter() - t0
    if rank == 0:
        print(json.dumps({
            "metric": "soft-grad batch GCUPS", "value": value, "unit": "GCUPS", "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)", "config": config, "e2e": e2e, "roofline": roofline,
            "cpu_baseline": cpu, "parity": parity, "clocks": clocks, "gpu_launches": launches, "extras": extras,
            "plain_fill": plain, "serve": serve,
            "autotune": {str(k): _tune_mod().describe(v) for k, v in tune_table.items()},
            "step_ms": step_ms, "graph_captures_timed": getattr(clk, "captures", None)}))
    if dist is not None:
        dist.destroy_process_group()


def _small_step(p, g, size=0.05):
    """A gradient step whose largest move is `size` (scores in nats).  The summed gradient of
    64 long pairs runs to tens of thousands per entry, so a fixed learning rate on it would move
    the scores by tens of nats: weights near e^60, far outside a training step."""
    big = max(float(np.abs(g.matrices).max()), float(np.abs(g.gaps).max()), 1e-30)
    return p + g * (size / big)


def c4_workload(n_pairs=64, seed=4):
    """Long pairs: A of length log-uniform 5,000-36,000, B = A with 20 % substitutions and
    single-residue indels (2.5 % each)."""
    rng = np.random.default_rng(seed)
    freqs = rng.dirichlet(np.full(20, 5.0))
    mat = c2_matrix(rng)
    la = np.exp(rng.uniform(np.log(5000), np.log(36000), size=n_pairs)).astype(np.int64)
    oa = np.zeros(n_pairs + 1, np.int64); np.cumsum(la, out=oa[1:])
    a = rng.choice(20, size=int(oa[-1]), p=freqs).astype(np.uint8)
    b = a.copy()
    s = rng.random(b.size) < 0.20
    b[s] = rng.choice(20, size=int(s.sum()), p=freqs)
    keep = (rng.random(b.size) >= 0.025).astype(np.int64)
    ins = rng.random(b.size) < 0.025
    cnt = keep + ins
    cnt[oa[1:] - 1] = np.maximum(cnt[oa[1:] - 1], 1)
    bb = b[np.repeat(np.arange(b.size), cnt)]
    bb[(np.cumsum(cnt) - 1)[ins]] = rng.choice(20, size=int(ins.sum()), p=freqs)
    ob = np.zeros(n_pairs + 1, np.int64); np.cumsum(np.add.reduceat(cnt, oa[:-1]), out=ob[1:])
    return mat, a, oa, bb.astype(np.uint8), ob


def _timed_run(fn, reps=1):
    import torch
    best = None
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    return best


def bench_c4(args):
    """Side measurement: long pairs (log-uniform 5k-36k).  Hard gradient by Pointers (tiles of
    256 x 256 cells, a launch per anti-diagonal of tiles), by the grid traceback (the same tiles
    score-only, then a walk that refills the tiles its path crosses) and by Hirschberg (float32
    prefix-max carry and float64 exact carry; the large half-sweeps as tiles), each hard run
    then re-aligned banded (bandwidth 64) after a 1e-3 parameter step; soft gradient (tiles:
    forward and backward a launch per anti-diagonal), then soft banded re-alignment after a
    step.  GCUPS per stage from wall time around each call (after a warm call)."""
    import nwgrad_b200 as nw
    mat, a, oa, b, ob = c4_workload(args.long_pairs)
    cells = cells_of(oa, ob)
    p = nw.AlignParams.from_arrays(mat[None], [[11.0, 1.0, 11.0, 1.0]], alphabet=nw.AA20)
    out = {"metric": "long-pair GCUPS per stage", "unit": "GCUPS", "n_gpus": 1,
           "config": {"workload": f"{args.long_pairs} pairs, A log-uniform 5k-36k, B = A 20% mutated",
                      "cells": cells, "max_len": int(np.diff(oa).max())}, "stages": {}}
    for name, cls, tb in (("hard_pointers_f32", nw.SeqPairBatch, "pointers"),
                          ("hard_grid_f32", nw.SeqPairBatch, "grid"),
                          ("hard_hirschberg_pmax_f32", nw.SeqPairBatch, "hirschberg_pmax"),
                          ("hard_hirschberg_f64", nw.SeqPairBatchDouble, "hirschberg")):
        bt = cls.from_codes(a, oa, b, ob, p, grad_mode="hard", traceback=tb)
        bt.score_and_grad()                                     # warm
        t = _timed_run(lambda: (bt.score_and_grad(), bt.compute_grad()))
        out["stages"][name] = {"seconds": t, "gcups": cells / t / 1e9}
        if name == "hard_hirschberg_pmax_f32":
            bt.set_params(_small_step(p, bt.compute_grad()))
            bt.banded_grad(64)                                  # warm: the band plan and its graph
            t = _timed_run(lambda: (bt.banded_grad(64), bt.compute_grad()))
            band_cells = float(np.sum(np.diff(oa) * 129))
            out["stages"]["banded64_after_step_f32"] = {"seconds": t, "gcups_full_equivalent": cells / t / 1e9,
                                                         "band_cells": band_cells}
        del bt
    bt = nw.SeqPairBatch.from_codes(a, oa, b, ob, p, grad_mode="soft")
    bt.score_and_grad()
    t = _timed_run(lambda: (bt.score_and_grad(), bt.compute_grad()))
    out["stages"]["soft_f32"] = {"seconds": t, "gcups": cells / t / 1e9}
    # soft banded re-alignment (bandwidth 64) around the Viterbi guides after a parameter step,
    # in float32 (the batch's precision)
    bt.set_params(_small_step(p, bt.compute_grad()))
    bt.banded_grad(64)                                      # warm: the band plan
    t = _timed_run(lambda: (bt.banded_grad(64), bt.compute_grad()))
    band_cells = float(np.sum(np.diff(oa) * 129))
    out["stages"]["soft_banded64_after_step_f32"] = {"seconds": t, "gcups_full_equivalent": cells / t / 1e9,
                                                     "band_cells": band_cells,
                                                     "refused_to_double": int(np.count_nonzero(bt.soft_status() & 0xFF))}
    return out


def c3_workload(n_pairs, seed=3):
    """Many short pairs: A a 22-nt RNA (ACGU), B 30-50 nt DNA (ACGT) with the reverse complement
    of A[1:8] (6-8 nt) at a random offset; alphabet ACGTU; track of A: 0 seed (A[1:8]), 1 the
    3' region (A[13:]), 2 the rest."""
    rng = np.random.default_rng(seed)
    A = np.array([0, 1, 2, 4], np.uint8)           # A C G U in "ACGTU"
    comp = {0: 4, 1: 2, 2: 1, 4: 0}                # RNA -> complementary DNA base (U pairs with A)
    a = A[rng.integers(0, 4, size=(n_pairs, 22))]
    lb = rng.integers(30, 51, size=n_pairs)
    ob = np.zeros(n_pairs + 1, np.int64); np.cumsum(lb, out=ob[1:])
    b = rng.integers(0, 4, size=int(ob[-1])).astype(np.uint8)   # A C G T
    seed_len = rng.integers(6, 9, size=n_pairs)
    lut = np.array([3, 2, 1, 0, 0], np.uint8)      # complement of A C G T U as DNA: T G C A A
    for p in range(0, n_pairs):
        k = int(seed_len[p]); off = int(rng.integers(0, lb[p] - k + 1))
        site = lut[a[p, 1:1 + k][::-1]]
        b[ob[p] + off: ob[p] + off + k] = site
    oa = np.arange(n_pairs + 1, dtype=np.int64) * 22
    tr = np.full((n_pairs, 22), 2, np.uint16); tr[:, 1:8] = 0; tr[:, 13:] = 1
    mat = np.full((3, 5, 5), -4.0)
    for k in range(3):
        for x, y in ((0, 3), (1, 2), (2, 1), (3, 0), (4, 0), (2, 4)):   # A-T, C-G, G-C, T-A, U-A, G-U wobble
            mat[k, x, y] = 5.0
    gaps = np.tile([6.0, 6.0, 6.0, 6.0], (3, 1))
    return mat, gaps, a.reshape(-1), oa, b, ob, tr.reshape(-1)


def c6_workload(n_pairs, seed=6):
    """miRNA-like A (22 nt RNA, ACGU) against B of 200-1000 nt (ACGT) holding the reverse
    complement of A[1:8] at a random offset: the "A within B" problem of glocal ends."""
    rng = np.random.default_rng(seed)
    A = np.array([0, 1, 2, 4], np.uint8)
    a = A[rng.integers(0, 4, size=(n_pairs, 22))]
    lb = rng.integers(200, 1001, size=n_pairs)
    ob = np.zeros(n_pairs + 1, np.int64); np.cumsum(lb, out=ob[1:])
    b = rng.integers(0, 4, size=int(ob[-1])).astype(np.uint8)
    lut = np.array([3, 2, 1, 0, 0], np.uint8)
    for p in range(n_pairs):
        off = int(rng.integers(0, lb[p] - 8))
        b[ob[p] + off: ob[p] + off + 7] = lut[a[p, 1:8][::-1]]
    oa = np.arange(n_pairs + 1, dtype=np.int64) * 22
    mat = np.full((1, 5, 5), -4.0)
    for x, y in ((0, 3), (1, 2), (2, 1), (3, 0), (4, 0), (2, 4)):
        mat[0, x, y] = 5.0
    gaps = np.array([[5.0, 2.0, 5.0, 2.0]])
    return mat, gaps, a.reshape(-1), oa, b, ob


def bench_c6(args):
    """Side measurement: glocal ends (A within B), affine, hard and soft, autotuned; the same
    batch with Global ends beside it, and the reference's CPU path on a bounded sample."""
    import nwgrad_b200 as nw
    import oracle
    mat, gaps, a, oa, b, ob = c6_workload(args.glocal_pairs)
    cells = cells_of(oa, ob)
    p = nw.AlignParams.from_arrays(mat, gaps, alphabet="ACGTU")
    out = {"metric": "glocal GCUPS", "unit": "GCUPS", "n_gpus": 1,
           "config": {"workload": f"{args.glocal_pairs} pairs, A 22 nt RNA, B 200-1000 nt DNA with a seed site, "
                                  f"affine (5, 2), glocal ends", "cells": cells}, "modes": {}}
    for grad in ("hard", "soft"):
        res = {}
        for mode in ("glocal", "global"):
            bt = nw.SeqPairBatch.from_codes(a, oa, b, ob, p, grad_mode=grad, mode=mode)
            table = bt.autotune()
            bt.score_and_grad()
            t = _timed_run(lambda: (bt.score_and_grad(), bt.compute_grad()), reps=3)
            ms, launches = bt.last_timing()
            res[mode] = {"gcups": cells / t / 1e9, "seconds": t, "device_ms": ms, "launches": launches,
                         "autotune": {str(k): _tune_mod().describe(v) for k, v in table.items()}}
            del bt
        if oracle.ref_bench_available() and not args.no_cpu_baseline:
            k = min(args.glocal_pairs, 20000)
            secs, _, threads, isa = oracle.ref_time_codes(32, 1, 2, 2 if grad == "soft" else 1, "ACGTU", mat, gaps,
                                                          a, oa[:k + 1], b, ob[:k + 1], warmup=1, reps=2,
                                                          free_ends=12)
            ck = cells_of(oa[:k + 1], ob[:k + 1])
            res["cpu_reference"] = {"gcups": ck / float(np.min(secs)) / 1e9, "pairs": k, "cores": threads,
                                    "isa": isa, "sample": f"first {k} pairs, best of {len(secs)}"}
        out["modes"][grad] = res
    return out


def bench_c3(args):
    """Side measurement: many short pairs, local linear, K = 3 parameter sets by a per-residue
    track of A; hard and soft; one launch per geometry bucket, autotuned."""
    import nwgrad_b200 as nw
    mat, gaps, a, oa, b, ob, tr = c3_workload(args.short_pairs)
    cells = cells_of(oa, ob)
    p = nw.AlignParams.from_arrays(mat, gaps, alphabet="ACGTU")
    out = {"metric": "short-pair GCUPS", "unit": "GCUPS", "n_gpus": 1,
           "config": {"workload": f"{args.short_pairs} pairs, A 22 nt, B 30-50 nt, local linear, K=3 tracked",
                      "cells": cells}, "modes": {}}
    for mode in ("hard", "soft"):
        bt = nw.SeqPairBatch.from_codes(a, oa, b, ob, p, grad_mode=mode, gap_model="linear", mode="local",
                                        tracks=tr)
        table = bt.autotune()
        bt.score_and_grad()
        t = _timed_run(lambda: (bt.score_and_grad(), bt.compute_grad()), reps=3)
        ms, launches = bt.last_timing()
        bt.use_plain_fill()
        bt.score_and_grad()
        tp = _timed_run(lambda: (bt.score_and_grad(), bt.compute_grad()), reps=3)
        out["modes"][mode] = {"gcups": cells / t / 1e9, "seconds": t, "device_ms": ms, "launches": launches,
                              "plain_fill_gcups": cells / tp / 1e9,
                              "autotune": {str(k): _tune_mod().describe(v) for k, v in table.items()}}
        del bt
    return out


def bench_c1(args):
    """Side measurement: the plain global affine hard batch (10k pairs L 50-300), GCUPS of
    score_and_grad() + compute_grad() with the codes resident."""
    import torch
    import nwgrad_b200 as nw
    mat, a, oa, b, ob = c1_workload()
    cells = cells_of(oa, ob)
    params = nw.AlignParams.from_arrays(mat[None], [[11.0, 1.0, 11.0, 1.0]], alphabet=nw.AA20)
    bt = nw.SeqPairBatch.from_codes(a, oa, b, ob, params, grad_mode="hard")
    table = {} if args.no_tune else bt.autotune()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(max(args.warmup, 3)):
        bt.score_and_grad(); bt.compute_grad()
    ms = []
    kms = 0.0
    for _ in range(args.steps):
        flush.zero_(); torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(); bt.score_and_grad(); bt.compute_grad(); e1.record(); torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1)); kms += bt.last_timing()[0]
    tot = float(np.sum(ms))
    return ({"metric": "hard-grad batch GCUPS", "value": cells * args.steps / (tot / 1e3) / 1e9,
                      "unit": "GCUPS", "n_gpus": 1, "steps": args.steps, "ms_per_step": tot / args.steps,
                      "kernel_ms_per_step": kms / args.steps, "config": {"workload": "c1 hard global affine float32, "
                      "10k pairs L 50-300", "cells_per_step": cells},
                      "autotune": {str(k): _tune_mod().describe(v) for k, v in table.items()}, "step_ms": ms})


def _trainer(pos, neg, mat, gaps0, steps, srv=None):
    """Adam (lr 1e-3) on the matrix and the four gap costs, maximising the mean homolog - decoy
    soft-score margin; with a server, it takes the parameters after every step."""
    import torch
    import nwgrad_b200 as nw
    from nwgrad_b200.autograd import align_scores
    M = torch.tensor(mat[None], dtype=torch.float64, requires_grad=True)
    G = torch.tensor(gaps0, dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([M, G], lr=1e-3)
    margins = []
    t0 = time.perf_counter()
    for _ in range(steps):
        opt.zero_grad()
        margin = (align_scores(pos, M, G) - align_scores(neg, M, G)).mean()
        (-margin).backward()
        opt.step()
        margins.append(float(margin))
        if srv is not None:
            srv.set_params(nw.AlignParams.from_arrays(M.detach().numpy().copy(), G.detach().numpy().copy(),
                                                      alphabet=nw.AA20))
    return time.perf_counter() - t0, margins


def bench_c5(args):
    """Side measurement: serving plus an autograd training loop.  A Poisson stream of requests
    (A lengths log-uniform 20-5000, batch sizes log-uniform 1-4096, B a mutated copy) goes
    through the continuous-batching server while 200 Adam steps (lr 1e-3) train the 20x20
    matrix and four gap costs on the soft-gradient batch's pair distribution; after every
    step the server takes the new parameters.  Each half is also run alone."""
    import queue
    import nwgrad_b200 as nw
    from nwgrad_b200.serve import Server
    mat, a, oa, bp, obp, bn, obn = c2_workload(args.train_pairs, seed=1)
    gaps0 = np.array([[11.0, 1.0, 11.0, 1.0]])
    p0 = nw.AlignParams.from_arrays(mat[None], gaps0, alphabet=nw.AA20)
    pos = nw.SeqPairBatch.from_codes(a, oa, bp, obp, p0, grad_mode="soft")
    neg = nw.SeqPairBatch.from_codes(a, oa, bn, obn, p0, grad_mode="soft")
    train_cells = cells_of(oa, obp) + cells_of(oa, obn)
    reqs = c5_requests(args.serve_requests)
    req_cells = sum(cells_of(o1, o2) for _, o1, _, o2 in reqs)
    steps = args.train_steps
    _trainer(pos, neg, mat, gaps0, 3)                       # warm: plans, graphs, pools
    serve_server(p0, reqs[:8], [0.0] * 8, 0)
    train_alone, margins = _trainer(pos, neg, mat, gaps0, steps)
    burst = serve_server(p0, reqs, [0.0] * len(reqs), 0)
    rate = 0.7 * len(reqs) / burst["seconds"]
    rng = np.random.default_rng(1005)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(reqs))).tolist()
    serve_alone = serve_server(p0, reqs, arrivals, 0)
    # both at once
    lat = []
    q = queue.Queue()
    out = {}
    with Server(p0, grad_mode="soft", workers=3, hbm_budget_gb=96.0, max_batch_pairs=16384, device=0) as srv:
        def waiter():
            while True:
                item = q.get()
                if item is None:
                    return
                lat.append(srv.wait(item[0], item[1])[2])

        def train():
            out["train"] = _trainer(pos, neg, mat, gaps0, steps, srv)

        wt = threading.Thread(target=waiter, daemon=True)
        tt = threading.Thread(target=train, daemon=True)
        wt.start()
        t0 = time.perf_counter()
        tt.start()
        for (ca, o1, cb, o2), at in zip(reqs, arrivals):
            d = at - (time.perf_counter() - t0)
            if d > 0:
                time.sleep(d)
            q.put((srv.submit_codes(ca, o1, cb, o2), len(o1) - 1))
        q.put(None)
        wt.join()
        serve_span = time.perf_counter() - t0
        tt.join()
    p50, p99 = _quantiles(lat)
    train_mixed, margins_mixed = out["train"]
    return ({
        "metric": "serve p50/p99 latency and training GCUPS, both at once", "n_gpus": 1,
        "config": {"workload": "Poisson request stream (lengths log-uniform 20-5000, batch sizes log-uniform "
                               "1-4096, B mutated) through the server, offered at 70% of its burst capacity, "
                               f"while {steps} Adam steps (lr 1e-3) train the matrix and gaps on "
                               f"{args.train_pairs} homolog + {args.train_pairs} decoy pairs (L 100-500); "
                               "set_params into the server after every step",
                   "requests": len(reqs), "request_cells": req_cells, "train_cells_per_step": train_cells,
                   "offered_rate_per_s": rate},
        "serve_alone": {"p50_ms": serve_alone["p50_ms"], "p99_ms": serve_alone["p99_ms"],
                        "gcups": serve_alone["gcups"]},
        "train_alone": {"seconds": train_alone, "steps_per_s": steps / train_alone,
                        "gcups": train_cells * steps / train_alone / 1e9,
                        "margin_first": margins[0], "margin_last": margins[-1]},
        "mixed": {"serve_p50_ms": p50, "serve_p99_ms": p99, "serve_gcups": req_cells / serve_span / 1e9,
                  "train_seconds": train_mixed, "train_gcups": train_cells * steps / train_mixed / 1e9,
                  "margin_last": margins_mixed[-1]},
    })


if __name__ == "__main__":
    main()
