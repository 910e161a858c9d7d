#!/usr/bin/env python
"""Benchmark of the continuous Frechet distance engine on B200.

One step is one full solve (endpoint bound, DFD, VE-FD, learned bracket, epsilon search to
2^-33 relative, i.e. within 1e-9 of the FP64 result) of the long-pair workload: two
200,000-point 3D robot-like paths (Catmull-Rom through 2,000 waypoints U[-100,100]^3, the
second path under a 20-knot monotone time warp plus N(0, 0.1^2) noise, seed 1), 4.0e10
free-space cells per decision.  Inputs are synthetic and seeded (the reference ships no data).

  value : FD solves/s with both curves resident in HBM (rfd_distance on device pointers, the
          shipped bracket network)
  e2e   : the same through the C ABI with host buffers (H2D copy, solve, D2H result)
  plain : the plain method (bisection of [VE-FD, DFD], no bracket) on the same pair
  batch : the 4096-pair uneven batch (lognormal lengths, seed 2): learned and plain batched
          calls, and single-pair plain calls on a sample of it
  mixed_precision : large 3D pairs with coordinates ~1e4, FP32 filter against FP64
          (fraction of decision cells computed in FP64, error against the FP64 path)
  oversize : two 1,000,000-point 3D spline paths (10^12 cells), whose one-row-per-strip
          boundary (250 GB) does not fit: the VE-FD and decision strips run in launch windows
          over an O(n+m) ring; learned form with the coarse bound, host buffers
  roofline : the dominant phase kernel against the measured FP64 FMA peak
  cpu_baseline : the CPU oracle (dense FP64 restatement, OpenMP) on a bounded sample,
                 extrapolated to the plain method's probes on the full pair

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--no-batch]
Under torchrun every rank solves the same pair (the path does not shard: replicas only).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FD solves/s and free-space cells/s at <=1e-9 rel err vs FP64 plain GPU form"
WORKLOAD = ("long pair: 2 x 200,000-point 3D spline paths (2,000 waypoints U[-100,100]^3, "
            "20-knot time warp, noise 0.1, seed 1); FD to 2^-33 relative")
# algorithmic FP64 flops per cell (fma = 2, sqrt/div = 1), from the reference expressions:
# DFD .cu:615-626, VE-FD .cu:373-419, decision .cu:1173-1244
# ncu dram__bytes_read.sum + dram__bytes_write.sum on the 20,000-point case: one decision
# round, both halves of the split pair (mirror 3.584768 MB + forward 4.161792 MB); one VE-FD
# launch of the unsplit pair (two launches averaged; the split VE-FD was not captured)
DEC_DRAM_BYTES_20K = 3.584768e6 + 4.161792e6
VEFD_DRAM_BYTES_20K = 4.31e6
COARSE_UB = 6  # the learned form's upper bound: inflated DFD of every 6th point (rfd.h coarse_ub)
ARITY = 4  # batched forms: radii per round for the longest-chain pairs (rfd.h search_arity)
DFD_DRAM_BYTES_200K = 31.5e6 + 68.4e6  # ncu, the exact DFD launch of the long pair (32-row ring)
KERNEL_OF_PHASE = {"dfd": f"dfd_kernel<{'1, INFL' if COARSE_UB else '8'}>",
                   "vefd": "team_kernel<K_VEFD> (forward and mirror halves)",
                   "search": "team_kernel<K_DEC> (forward and mirror halves)"}
FLOPS_PER_CELL = {"dfd": lambda d: 3 * d + 3 + (4 if COARSE_UB else 0),  # + sqrt, 2 adds, square
                  "vefd": lambda d: 24 * d + 2,
                  "search": lambda d: 12 * d + 22}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-sample", type=int, default=60000,
                    help="points per curve of the CPU-baseline sample")
    ap.add_argument("--points", type=int, default=200000,
                    help="points per curve of the long pair (smaller values: profiling cases)")
    ap.add_argument("--no-batch", action="store_true", help="skip the 4096-pair batch leg")
    ap.add_argument("--mixed-pairs", type=int, default=2,
                    help="pairs of the mixed-precision workload to solve (0: skip that leg)")
    ap.add_argument("--plain-steps", type=int, default=2, help="timed plain-method solves")
    ap.add_argument("--oversize-points", type=int, default=1000000,
                    help="points per curve of the oversize pair (0: skip that leg)")
    ap.add_argument("--profile-batch", type=int, default=0, metavar="N",
                    help="profiling case: one batched call (one probe) on the first N pairs of "
                         "the uneven batch, then exit (no JSON line)")
    ap.add_argument("--profile-search", type=int, default=0, metavar="N",
                    help="profiling case: one batched call of the learned form (every probe, "
                         "k-ary rounds) on the first N pairs of the uneven batch, then exit (no "
                         "JSON line)")
    ap.add_argument("--profile-bounds", type=int, default=0, metavar="N",
                    help="profiling case: N calls of the exact bounds (DFD, then VE-FD pruned by "
                         "it) on the long pair of --points points, then exit (no JSON line)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for name, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        load = [v for v in sm if v > 0.5 * (mx or 1)] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload(points=200000, gen=None):
    """The long pair; other sizes keep its generator (waypoints = points / 100, seed 1).
    gen: the module whose seeded generator makes it (the CPU arm passes the oracle, which
    carries a copy of the same generator, so that it never loads librfd.so)."""
    if gen is None:
        import robotfd_b200 as gen
    if points == 200000:
        return gen.gen_config(1)[0]
    return gen.gen_pair(1, 3, points, points, 100.0, 0.1, 1, 0)


GOLDENS = os.path.join(ROOT, "tests", "golden", "config_goldens.json")


def workload_probes(P, Q, points):
    """Decisions of the plain method's solve of the workload at 2^-33, as the CPU oracle made
    them: the committed golden of the long pair, or (other sizes) an oracle solve."""
    import oracle
    if points == 200000 and os.path.exists(GOLDENS):
        with open(GOLDENS) as f:
            rec = json.load(f)["cases"].get("config1/0")
        if rec:
            return rec["probes"], "oracle golden of this pair (tests/golden/config_goldens.json)"
    r = oracle.distance(P, Q, stop_mode=1, quirks=False, threads=oracle.max_threads())
    return r["probes"], "oracle solve of this pair"


def config_dict(points, n1, n2, d, world):
    """The workload description both arms print (same keys and values)."""
    return {"workload": WORKLOAD if points == 200000 else
            f"long-pair generator at {points} points per curve", "n1": n1, "n2": n2,
            "dims": d, "stop": "ub-lb <= 2^-33 ub",
            "form": f"learned bracket (shipped network), coarse upper bound k={COARSE_UB}",
            "parallelism": f"replicas x{world}",
            "l2": "flushed before every step (256 MiB write outside the timed events)"}


def cpu_sample(P, Q, m, probes, probes_src="the plain method's decisions"):
    """Dense CPU oracle on the first m points of each curve: DFD, VE-FD and one decision,
    timed; the rates extrapolate to one solve of the full pair with `probes` decisions."""
    import oracle
    threads = oracle.max_threads()
    Ps, Qs = np.ascontiguousarray(P[:m]), np.ascontiguousarray(Q[:m])
    lb = oracle.endpoint(Ps, Qs)
    t0 = time.perf_counter()
    dsq = oracle.dfd_sq(Ps, Qs, threads)
    t1 = time.perf_counter()
    vsq = oracle.vefd_sq(Ps, Qs, lb, threads)
    t2 = time.perf_counter()
    oracle.decide(Ps, Qs, 0.5 * (np.sqrt(dsq) + np.sqrt(vsq)), threads)
    t3 = time.perf_counter()
    pts, cells = m * m, (m - 1) * (m - 1)
    r_dfd, r_ve, r_dec = pts / (t1 - t0), cells / (t2 - t1), cells / (t3 - t2)
    n1, n2 = len(P), len(Q)
    sec = n1 * n2 / r_dfd + (n1 - 1) * (n2 - 1) * (1 / r_ve + probes / r_dec)
    return {
        "value": 1.0 / sec, "unit": "solves/s", "cores": threads, "kind": "port",
        "sample": (f"oracle (dense FP64, OpenMP {threads} threads): DFD, VE-FD and one decision "
                   f"on the first {m} points of each curve ({t3 - t0:.1f} s), extrapolated to "
                   f"the full pair with {probes} decisions ({probes_src})"),
        "cells_per_s": {"dfd": r_dfd, "vefd": r_ve, "decision": r_dec},
    }


def cpu_batch_sample(every=64):
    """Measured, not extrapolated: the CPU oracle fully solves (plain method, 2^-33) every
    `every`-th pair of the uneven batch, one pair after another on all host threads."""
    import oracle
    threads = oracle.max_threads()
    dims, n1, n2, styles, scales, noises = oracle.gen_batch_spec(2, 4096, 2)
    idx = list(range(0, 4096, every))
    pairs = [oracle.gen_pair(int(styles[k]), int(dims[k]), int(n1[k]), int(n2[k]),
                             float(scales[k]), float(noises[k]), 2, k) for k in idx]
    t0 = time.perf_counter()
    res = [oracle.distance(p, q, stop_mode=1, quirks=False, threads=threads) for p, q in pairs]
    sec = time.perf_counter() - t0
    return {"value": len(idx) / sec, "unit": "solves/s", "cores": threads, "kind": "port",
            "sample": f"{len(idx)} pairs of the 4096-pair batch (every {every}th), each fully "
                      f"solved by the oracle (dense FP64, OpenMP), {sec:.1f} s",
            "mean_probes": statistics.mean(r["probes"] for r in res)}


def reference_arm(args):
    """CPU implementation of the path (the oracle port: the reference has no CPU path).
    Imports only the oracle (inputs from its copy of the generator): librfd.so stays
    unloaded in this arm."""
    import oracle
    rank, world, _ = dist_env()
    if rank != 0:
        return
    P, Q = workload(args.points, gen=oracle)
    probes, src = workload_probes(P, Q, args.points)
    vals = []
    for k in range(args.warmup + args.steps):
        r = cpu_sample(P, Q, args.cpu_sample, probes, src)
        if k >= args.warmup:
            vals.append(r["value"])
    v = statistics.median(vals)
    r["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": config_dict(args.points, len(P), len(Q), P.shape[1], world),
            "cpu_baseline": r,
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def batch_pairs(npairs=4096, seed=2):
    """The uneven batch (config 2 generator), generated on all host threads."""
    from concurrent.futures import ThreadPoolExecutor
    import robotfd_b200 as rfd
    dims, n1, n2, styles, scales, noises = rfd.gen_batch_spec(2, npairs, seed)

    def one(k):
        return rfd.gen_pair(int(styles[k]), int(dims[k]), int(n1[k]), int(n2[k]),
                            float(scales[k]), float(noises[k]), seed, k)
    with ThreadPoolExecutor(max(1, min(32, os.cpu_count() or 1))) as ex:
        return list(ex.map(one, range(npairs)))


def batch_leg(ctx, model, timed, sample=128, dist=None):
    """4096 uneven pairs: learned batched, plain batched, and plain single-pair calls on a
    fixed sample (every 32nd pair), each timed with CUDA events on the context stream.  Under
    torchrun the learned batch is sharded over the ranks (robotfd_b200.shard: a fixed 4096
    pairs, strong scaling), timed as the maximum over ranks."""
    pairs = batch_pairs()
    Ps, Qs = [p for p, _ in pairs], [q for _, q in pairs]
    n = len(Ps)
    if dist is not None:
        import torch
        from robotfd_b200 import shard
        shard.distance_batch_sharded(ctx, Ps[:256], Qs[:256], precise=True, model=model,
                                     search_arity=ARITY)  # warm
        t_s, res = timed(lambda: shard.distance_batch_sharded(ctx, Ps, Qs, precise=True,
                                                              model=model, search_arity=ARITY), 2)
        t = torch.tensor([statistics.median(t_s)], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return {
            "workload": "4096 uneven pairs (config 2 generator, seed 2), sharded over "
                        f"{dist.get_world_size()} ranks by cells; FD to 2^-33 relative",
            "solves_per_s": {"learned_sharded": n / (float(t.item()) * 1e-3)},
            "scaling": "strong (the 4096 pairs are split over the ranks)",
            "mean_probes": {"learned": statistics.mean(r["probes"] for r in res)},
        }
    import robotfd_b200 as rfd
    # the project's autotuners pick the DFD sweep's tile shape and the team strips' shape and
    # search split for this workload (the learned form, on a sample of the batch)
    tuned = ctx.autotune(Ps, Qs, reps=1)
    samp = list(range(0, n, 4))
    tuned_search = ctx.autotune_search([Ps[k] for k in samp], [Qs[k] for k in samp], reps=1,
                                       precise=True, model=model)
    ctx.distance_batch(Ps[:64], Qs[:64], precise=True, model=model)  # warm
    # the batched forms run as CUDA graphs: the first (untimed) call captures, the timed
    # calls with the same layout replay
    batched = dict(precise=True, model=model, graph=True, search_arity=ARITY)
    ctx.distance_batch(Ps, Qs, **batched)
    t_l, learned = timed(lambda: ctx.distance_batch(Ps, Qs, **batched), 2)
    # the same with plain bisection rounds (one radius per probe)
    bisect = dict(batched, search_arity=0)
    ctx.distance_batch(Ps, Qs, **bisect)
    t_b, learned_b = timed(lambda: ctx.distance_batch(Ps, Qs, **bisect), 2)
    # the north star's target form: batched, learned bracket, mixed precision (FP32 filter)
    mixed = dict(batched, precision=rfd.RFD_PREC_FP32_FILTER)
    ctx.distance_batch(Ps, Qs, **mixed)
    t_m, learned_mixed = timed(lambda: ctx.distance_batch(Ps, Qs, **mixed), 2)
    # untimed first call: the coarse pairs' arrays can grow the context's workspace once
    ctx.distance_batch(Ps, Qs, precise=True, model=model, coarse_ub=COARSE_UB,
                       search_arity=ARITY)
    t_c, _ = timed(lambda: ctx.distance_batch(Ps, Qs, precise=True, model=model,
                                              coarse_ub=COARSE_UB, search_arity=ARITY), 1)
    t_p, plain = timed(lambda: ctx.distance_batch(Ps, Qs, precise=True), 1)
    # the same search without the network: the threshold probe over VE-FD alone (a bracket at
    # the VE-FD bound), as a replayed graph like the learned form
    alone = dict(precise=True, graph=True, search_arity=ARITY,
                 brackets=[(r["vefd"] * (1 - 1e-15), r["vefd"]) for r in plain])
    ctx.distance_batch(Ps, Qs, **alone)
    t_a, thr = timed(lambda: ctx.distance_batch(Ps, Qs, **alone), 2)
    tail = [k for k, r in enumerate(thr) if r["probes"] > 1]
    idx = list(range(0, n, max(1, n // sample)))[:sample]
    t_s, single = timed(lambda: [ctx.distance(Ps[k], Qs[k], precise=True) for k in idx], 1)
    dev = max(abs(a["distance"] - b["distance"]) / a["distance"]
              for a, b in zip(plain, learned) if a["distance"] > 0)
    assert dev <= 1e-9, f"learned and plain batch results differ by {dev:.3g}"
    # the filter only classifies intervals that FP64 would compute identically
    mixed_err = max(abs(a["distance"] - b["distance"]) / a["distance"]
                    for a, b in zip(learned, learned_mixed) if a["distance"] > 0)
    fp64_frac = (sum(r["cells_fp64"] for r in learned_mixed) /
                 max(1, sum(r["cells_evaluated"] for r in learned_mixed)))
    for k, r in zip(idx, single):
        assert r["distance"] == plain[k]["distance"], "single and batched plain results differ"
    sps = {"learned_batched": n / (statistics.median(t_l) * 1e-3),
           "learned_batched_bisection": n / (statistics.median(t_b) * 1e-3),
           "learned_batched_mixed": n / (statistics.median(t_m) * 1e-3),
           "learned_batched_coarse_ub": n / (t_c[0] * 1e-3),
           "plain_batched": n / (statistics.median(t_p) * 1e-3),
           "threshold_only_batched": n / (statistics.median(t_a) * 1e-3),
           "plain_single_calls": len(idx) / (sum(t_s) * 1e-3)}
    return {
        "workload": "4096 uneven pairs (2D/3D 50/50, lognormal lengths median 2000, sigma 1, "
                    "clipped [100, 50000], walk/spline shapes, seed 2); FD to 2^-33 relative",
        "solves_per_s": sps,
        "learned_batched_vs_plain_single_calls": sps["learned_batched"] / sps["plain_single_calls"],
        # the north star's target: batched + learned bracket + mixed precision against the plain
        # FP64 form (one pair per call, bisection, FP64 intervals)
        "target_form_vs_plain_fp64": sps["learned_batched_mixed"] / sps["plain_single_calls"],
        "mixed": {"max_rel_error_vs_fp64": mixed_err, "decision_cells_fp64_fraction": fp64_frac},
        "autotune": {"dfd_rows_per_lane": tuned["rows"], "dfd_skewed": tuned["skew"],
                     "ms": {f"{r}x{'skew' if k else 'stack'}": round(v, 2)
                            for (r, k), v in tuned["ms"].items()},
                     "team_warps": tuned_search["warps"],
                     "search_switch": tuned_search["switch"],
                     "search_window": tuned_search["window"],
                     "search_sample": f"{len(samp)} pairs (every 4th), learned form",
                     "search_ms": {f"w{w}_s{['quarter', 'teams', 'queue'][si]}_win{win}":
                                   round(v, 2) for (w, si, win), v in tuned_search["ms"].items()}},
        "cuda_graph": "batched forms captured once and replayed (rfd_options.graph)",
        "search_arity": f"{ARITY} radii per round for the 32 longest-chain pairs once few pairs "
                        "remain (rfd_options.search_arity), in every learned and threshold-only "
                        "form; plain_batched and learned_batched_bisection bisect",
        "plain_single_sample": f"{len(idx)} pairs (every {n // len(idx)}th), one call each",
        "mean_probes": {"learned": statistics.mean(r["probes"] for r in learned),
                        "learned_bisection": statistics.mean(r["probes"] for r in learned_b),
                        "plain": statistics.mean(r["probes"] for r in plain),
                        "threshold_only": statistics.mean(r["probes"] for r in thr)},
        "tail_pairs": {"count": len(tail),
                       "mean_probes_learned": statistics.mean(learned[k]["probes"] for k in tail)
                       if tail else None,
                       "mean_probes_threshold_only": statistics.mean(thr[k]["probes"] for k in tail)
                       if tail else None},
        "bracket_network": network_timing(model, n),
        "probe_rounds": {"learned": max(r["probes"] for r in learned),
                         "plain": max(r["probes"] for r in plain)},
        "max_rel_dev_learned_vs_plain": dev,
        "cells": sum(len(p) * len(q) for p, q in pairs),
    }


def network_timing(model, n):
    """The bracket network's forward pass on n pairs (its hand-written mma.sync BF16 kernels)
    against the same layer shapes on cuBLAS through torch (BF16 matmuls, FP32 accumulate, GELU),
    CUDA events, median of 20 after 5 warm-up calls."""
    import torch
    x = torch.randn(n, 400, device="cuda")
    y = torch.empty(n, 2, device="cuda")
    w = [torch.randn(o, i, device="cuda", dtype=torch.bfloat16) * (1.0 / i ** 0.5)
         for o, i in ((256, 400), (256, 256), (256, 256), (2, 256))]
    xb = x.to(torch.bfloat16)

    def ours():
        model.forward(x.data_ptr(), n, y.data_ptr())

    def lib():
        h = xb
        for k, wk in enumerate(w):
            h = h @ wk.t()
            if k < 3:
                h = torch.nn.functional.gelu(h, approximate="tanh")
        return h

    def med(fn):
        s = torch.cuda.current_stream()
        for _ in range(5):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(20):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            fn()
            e1.record(s)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)
    torch.cuda.synchronize()
    return {"pairs": n, "ms_ours_mma_sync": med(ours), "ms_cublas_bf16_torch": med(lib),
            "note": "the network runs once per call on its own stream; both are launch-bound"}


def mixed_leg(ctx, model, timed, npairs):
    """The mixed-precision workload (config 4: large 3D spline pairs, coordinates ~1e4):
    the first npairs pairs in one batched call in the learned form (bracket network, coarse
    upper bound k = COARSE_UB), FP32 filter against FP64 intervals."""
    import robotfd_b200 as rfd
    pairs = rfd.gen_config(4, npairs=npairs)
    Ps, Qs = [p for p, _ in pairs], [q for _, q in pairs]
    kw = dict(precise=True, model=model, coarse_ub=COARSE_UB)
    # untimed first call: the context's workspace grows to these sizes once
    ctx.distance_batch(Ps, Qs, **kw)
    ctx.phase_times(enable=1)
    t64, r64 = timed(lambda: ctx.distance_batch(Ps, Qs, **kw), 1)
    ph64 = ctx.phase_times(enable=0)
    ctx.phase_times(enable=1)
    t32, r32 = timed(lambda: ctx.distance_batch(Ps, Qs, precision=rfd.RFD_PREC_FP32_FILTER,
                                                **kw), 1)
    ph = ctx.phase_times(enable=0)
    err = max(abs(a["distance"] - b["distance"]) / a["distance"] for a, b in zip(r64, r32))
    ev = sum(r["cells_evaluated"] for r in r32)
    return {
        "workload": f"first {npairs} of 512 3D spline pairs (100k-400k points, waypoints "
                    "U[-1e4,1e4]^3, seed 5), one batched call, bracket network, coarse upper "
                    f"bound k={COARSE_UB}",
        "points": [[len(p), len(q)] for p, q in pairs],
        "ms": {"fp64": sum(t64), "fp32_filter": sum(t32)},
        "phase_ms_fp64": {k: ph64[k + "_ms"] for k in ("dfd", "vefd", "search")},
        "phase_ms_fp32_filter": {k: ph[k + "_ms"] for k in ("dfd", "vefd", "search")},
        "probes": [r["probes"] for r in r32],
        "decision_cells_evaluated": ev,
        "decision_cells_fp64_fraction": sum(r["cells_fp64"] for r in r32) / max(ev, 1),
        "max_rel_error_vs_fp64": err,
        "decision_cells_per_s": {
            "nominal": sum(r["cells_nominal"] for r in r32) / max(ph["search_ms"] * 1e-3, 1e-9),
            "evaluated": ev / max(ph["search_ms"] * 1e-3, 1e-9)},
    }


def oversize_leg(model, timed, points):
    """Two 3D spline paths of `points` points each (seed 1, stream 7) in a fresh context: one
    boundary row per 32-row strip would take about points^2 / 4 bytes, so the VE-FD and
    decision strips run in launch windows over a ring of at most 4097 rows.  One untimed solve
    sizes the workspace (its growth is reported), then one timed solve with host buffers."""
    import torch
    import robotfd_b200 as rfd
    P, Q = rfd.gen_pair(1, 3, points, points, 100.0, 0.1, 1, 7)
    c = rfd.Context(torch.cuda.current_device())
    c.set_stream(torch.cuda.current_stream().cuda_stream)  # the stream `timed` records on
    try:
        free0 = torch.cuda.mem_get_info()[0]
        kw = dict(precise=True, model=model, coarse_ub=COARSE_UB)
        c.distance(P, Q, **kw)
        used = free0 - torch.cuda.mem_get_info()[0]
        c.phase_times(enable=1)
        t, r = timed(lambda: c.distance(P, Q, **kw), 1)
        ph = c.phase_times(enable=0)
    finally:
        c.close()
    rows = min(len(P), len(Q))
    return {
        "workload": f"2 x {points:,}-point 3D spline paths (waypoints U[-100,100]^3, seed 1, "
                    "stream 7); learned form, coarse bound k=6, FD to 2^-33; host buffers",
        "cells_per_decision": (len(P) - 1) * (len(Q) - 1),
        "one_row_per_strip_bytes": ((rows - 1 + 31) // 32 - 1) * 8 * (len(Q) + 31) // 32 * 32,
        "device_bytes_used": used,
        "ms_per_solve": t[0],
        "phase_ms": {k: ph[k + "_ms"] for k in ("dfd", "vefd", "search")},
        "probes": r["probes"],
        "flags": r["flags"],
        "bracket": [r["lb"], r["ub"]],
    }


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    import torch
    import robotfd_b200 as rfd
    if args.profile_batch:
        pairs = batch_pairs()[: args.profile_batch]
        ctx = rfd.Context(0)
        ctx.distance_batch([p for p, _ in pairs], [q for _, q in pairs], precise=True, max_probes=1)
        ctx.close()
        return
    if args.profile_bounds:
        P, Q = workload(args.points)
        ctx = rfd.Context(0)
        for _ in range(args.profile_bounds):
            ctx.bounds(P, Q, quirks=False)
        ctx.close()
        return
    if args.profile_search:
        pairs = batch_pairs()[: args.profile_search]
        ctx = rfd.Context(0)
        ctx.distance_batch([p for p, _ in pairs], [q for _, q in pairs], precise=True,
                           model=rfd.Model.pretrained(0), search_arity=ARITY)
        ctx.close()
        return

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    ctx = rfd.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    model = rfd.Model.pretrained(local)
    P, Q = workload(args.points)
    n1, n2, d = len(P), len(Q), P.shape[1]
    dP = torch.from_numpy(P).cuda()
    dQ = torch.from_numpy(Q).cuda()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    torch.cuda.synchronize()

    def step_dev():
        return ctx.distance_device(dP.data_ptr(), n1, dQ.data_ptr(), n2, d, precise=True,
                                   model=model, coarse_ub=COARSE_UB)

    def step_host():
        return ctx.distance(P, Q, precise=True, model=model, coarse_ub=COARSE_UB)

    def step_plain():
        return ctx.distance_device(dP.data_ptr(), n1, dQ.data_ptr(), n2, d, precise=True)

    def step_plain_kary():
        return ctx.distance_device(dP.data_ptr(), n1, dQ.data_ptr(), n2, d, precise=True,
                                   search_arity=ARITY)

    def timed(fn, k):
        times, res = [], None
        for _ in range(k):
            flush.fill_(1)  # L2 flush outside the event pair
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            res = fn()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        return times, res

    for _ in range(args.warmup):
        step_dev()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ctx.phase_times(enable=1)
    clocks = Clocks(local)
    clocks.start()
    torch.cuda.synchronize()
    times, res = timed(step_dev, args.steps)
    torch.cuda.synchronize()
    clk = clocks.stop()
    phases = ctx.phase_times(enable=0)
    total_ms = sum(times)
    if dist:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    ms_per_step = total_ms / args.steps
    value = world * args.steps / (total_ms / 1e3)

    # e2e: host buffers through the C ABI, copies inside the timed region (one untimed call
    # first: host inputs add the curves to the device workspace, which may then grow)
    step_host()
    ctx.phase_times(enable=1)
    etimes, eres = timed(step_host, args.steps)
    ephase = ctx.phase_times(enable=0)
    e_ms = sum(etimes)
    if dist:
        t = torch.tensor([e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e_ms = float(t.item())
    e2e_value = world * args.steps / (e_ms / 1e3)
    assert eres["distance"] == res["distance"], "host and device inputs disagree"

    # the plain method on the same pair (no bracket): the reference's probe sequence
    step_plain()
    ctx.phase_times(enable=1)
    ptimes, pres = timed(step_plain, args.plain_steps)
    pphase = ctx.phase_times(enable=0)
    rel = abs(pres["distance"] - res["distance"]) / pres["distance"]
    assert rel <= 1e-9, f"learned and plain results differ by {rel:.3g}"
    # the plain method with k-ary rounds: ARITY radii per launch round
    step_plain_kary()
    ktimes, kres = timed(step_plain_kary, args.plain_steps)
    krel = abs(kres["distance"] - pres["distance"]) / pres["distance"]
    assert krel <= 1e-9, f"k-ary and bisection results differ by {krel:.3g}"

    peak = ctx.fp64_peak()
    calls = max(phases["calls"], 1)
    ph_ms = {k: phases[k + "_ms"] / calls for k in ("dfd", "vefd", "search")}
    # the learned form's DFD phase sweeps the coarse pair: anchors every COARSE_UB-th point
    cn1, cn2 = ((n1 - 2) // COARSE_UB + 2, (n2 - 2) // COARSE_UB + 2) if COARSE_UB else (n1, n2)
    cells = {
        "dfd": cn1 * cn2,
        "vefd": res["cells_vefd"],
        "search": res["cells_evaluated"],
    }
    dom = max(ph_ms, key=ph_ms.get)
    flops = cells[dom] * FLOPS_PER_CELL[dom](d)
    achieved = flops / (ph_ms[dom] * 1e-3) / 1e12
    traffic = None
    if dom in ("search", "vefd"):
        # ncu dram__bytes_read.sum + dram__bytes_write.sum of one decision (VE-FD) launch on the
        # 20,000-point case (cold cache: every touched point record and boundary word once);
        # the touched data grows with the points, not the cells, so it scales by n1 + n2
        per20k = DEC_DRAM_BYTES_20K if dom == "search" else VEFD_DRAM_BYTES_20K
        traffic = per20k * (n1 + n2) / 40000
    elif dom == "dfd" and not COARSE_UB:
        # ncu dram__bytes_read.sum + dram__bytes_write.sum of the DFD launch on the full
        # 200,000-point pair (one pass): curves and the ring rows L2 evicts, scaled by points
        traffic = DFD_DRAM_BYTES_200K * (n1 + n2) / 400000
    sm_mhz = clk.get("sm_mhz") or 1965.0
    pcalls = max(pphase["calls"], 1)

    line = {
        "metric": METRIC,
        "value": value,
        "unit": "solves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": config_dict(args.points, n1, n2, d, world),
        "fd": res["distance"],
        "dfd": res["dfd"],
        "vefd": res["vefd"],
        "probes": res["probes"],
        "plain": {"solves_per_s": args.plain_steps / (sum(ptimes) * 1e-3),
                  "ms_per_solve": sum(ptimes) / args.plain_steps, "probes": pres["probes"],
                  "phase_ms": {k: pphase[k + "_ms"] / pcalls for k in ("dfd", "vefd", "search")},
                  "rel_dev_vs_learned": rel,
                  "kary": {"search_arity": ARITY,
                           "solves_per_s": args.plain_steps / (sum(ktimes) * 1e-3),
                           "ms_per_solve": sum(ktimes) / args.plain_steps,
                           "decisions": kres["probes"], "flags": kres["flags"],
                           "rel_dev_vs_bisection": krel}},
        "free_space_cells_per_s": {
            "nominal": res["cells_nominal"] / (ph_ms["search"] * 1e-3),
            "evaluated": res["cells_evaluated"] / (ph_ms["search"] * 1e-3),
            "evaluated_fraction": res["cells_evaluated"] / max(res["cells_nominal"], 1),
        },
        "bounds_cells_per_s": {"dfd": cells["dfd"] / (ph_ms["dfd"] * 1e-3),
                               "vefd_nominal": (n1 - 1) * (n2 - 1) / (ph_ms["vefd"] * 1e-3),
                               "vefd_evaluated": res["cells_vefd"] / (ph_ms["vefd"] * 1e-3)},
        "phase_ms": ph_ms,
        "roofline": {"bound": "fp64", "kernel": KERNEL_OF_PHASE[dom], "achieved": achieved,
                     "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": traffic,
                     "peak_source": "measured FP64 FMA throughput (rfd_fp64_peak), this GPU",
                     "flops_per_cell": FLOPS_PER_CELL[dom](d), "cells": cells[dom],
                     "traffic_note": ("bytes per launch, ncu capture of the full-size launch"
                                      if dom == "dfd" else
                                      "bytes per probe round (both halves of the split pair), "
                                      "ncu cold-cache capture at 20k points scaled by points"
                                      if dom == "search" else
                                      "bytes of one unsplit VE-FD launch, ncu cold-cache capture "
                                      "at 20k points scaled by points")},
        # the pruned sweeps are bound by their dependency chain, not by flops or bytes: the
        # wavefront has n1 + n2 anti-diagonals, so this is the latency each one adds
        "critical_path": {
            "antidiagonals": n1 + n2,
            "ms_per_probe": pphase["search_ms"] / pcalls / max(pres["probes"], 1),
            "cycles_per_antidiagonal": pphase["search_ms"] / pcalls / max(pres["probes"], 1)
                                       * 1e-3 * sm_mhz * 1e6 / (n1 + n2)},
        "e2e": {"value": e2e_value, "unit": "solves/s",
                "h2d_bytes_per_step": ephase["h2d_bytes"] / max(ephase["calls"], 1),
                "d2h_bytes_per_step": ephase["d2h_bytes"] / max(ephase["calls"], 1)},
        "gpu_launches": int(phases["launches"]),
        "clocks": clk,
    }
    if not args.no_batch:
        line["batch"] = batch_leg(ctx, model, timed, dist=dist)
    if args.mixed_pairs > 0 and world == 1:
        line["mixed_precision"] = mixed_leg(ctx, model, timed, args.mixed_pairs)
    if args.oversize_points > 0 and world == 1:
        line["oversize"] = oversize_leg(model, timed, args.oversize_points)
    if rank == 0:
        if world == 1:
            probes, src = workload_probes(P, Q, args.points)
            line["cpu_baseline"] = cpu_sample(P, Q, args.cpu_sample, probes, src)
            if "batch" in line:
                line["batch"]["cpu_measured"] = cpu_batch_sample()
                line["batch"]["learned_batched_vs_cpu_measured"] = (
                    line["batch"]["solves_per_s"]["learned_batched"] /
                    line["batch"]["cpu_measured"]["value"])
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    model.close()
    ctx.close()


if __name__ == "__main__":
    main()
