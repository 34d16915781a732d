#!/usr/bin/env python
"""EMC iteration throughput on B200: pattern x rotation evaluations per second.

One step = one full EMC iteration (expand -> maximize -> compress, emc.c:989-1084)
over every pattern and rotation of the workload, inputs resident in HBM.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Default workload: 128^3 model, 128x128 detector with a radius-6 beamstop
(16,272 active pixels), 86,520 rotations (600-cell n=12, halved), 50,000
seeded synthetic Poisson patterns (mean 500 photons, ~3% non-zero pixels,
lognormal scale sigma 0.5).  The headline is the dense mixed-precision
iteration (every pattern x rotation pair evaluated); beside it the line
reports the plain FP32 iteration, the learned orientation proposal (top
cells of a BF16 network's coarse posterior, the dense iteration as
fallback) with its captured responsibility mass and model error, the error
of the mixed path against the FP64 oracle on a sample, and the oracle's CPU
rate on that sample.
Multi-GPU (torchrun): patterns are sharded across ranks (each rank holds its
own N patterns of one seeded dataset: weak scaling) and every iteration sums
the model/weight insertion accumulators with one NCCL all-reduce before
normalisation -- the only exchange of an EMC iteration.  Time is the max over
ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "pattern×rotation evals/s"
UNIT = "evals/s"
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}
# DRAM bytes (read + write) per launch of the maximize contraction (the
# two-SM kernel the default workload selects) on the default workload (128^3,
# 86,520 rotations, 50,000 patterns), measured with ncu
# (dram__bytes_read.sum + dram__bytes_write.sum, one pass).
MAXIMIZE_TRAFFIC_BYTES = 671_161_542_400 + 17_579_778_304


def parse():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="large128")
    ap.add_argument("--patterns", type=int, default=None, help="override the pattern count")
    ap.add_argument("--rot-n", type=int, default=None,
                    help="override the 600-cell refinement of the rotation sampling")
    ap.add_argument("--likelihood", default="poisson", choices=["poisson", "gauss"])
    ap.add_argument("--interp", default="nearest", choices=["nearest", "trilinear"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp32"])
    ap.add_argument("--rotation-chunk", type=int, default=0,
                    help="rotations the log-likelihood buffer holds at a time (0: all)")
    ap.add_argument("--deterministic", action="store_true",
                    help="order-independent insertion sums (bitwise reproducible)")
    ap.add_argument("--fp32-steps", type=int, default=3, help="steps of the plain FP32 comparison")
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--batch-steps", type=int, default=5)
    ap.add_argument("--learned-steps", type=int, default=10)
    ap.add_argument("--train-iters", type=int, default=5,
                    help="dense iterations whose responsibilities train the proposal network")
    ap.add_argument("--train-epochs", type=int, default=12)
    ap.add_argument("--top-k", type=int, default=2048,
                    help="fine rotations per pattern covered by the cells of its previous posterior")
    ap.add_argument("--keep-tail", type=float, default=0.0,
                    help="also keep the cells holding all but this share of the previous posterior")
    ap.add_argument("--spec-top-k", type=int, default=512,
                    help="the smaller top-k reported beside the timed one (one step and 12 chained)")
    ap.add_argument("--oracle-patterns", type=int, default=16,
                    help="patterns whose proposed responsibilities are checked against the oracle")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--profile-case", choices=["proposed", "expand", "grouped"], default=None,
                    help="run one small fixed case for a profiler and exit (no JSON line): "
                         "proposed = two dense and three proposed iterations of the default "
                         "workload; expand = three dense iterations at 128^3 with 25,680 "
                         "rotations and 2,000 patterns; grouped = one dense and two proposed "
                         "iterations at 128^3 with 25,680 rotations and 20,000 patterns")
    return ap.parse_args()


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.isfile(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return FALLBACK_PEAKS, "fallback"


# ---------------------------------------------------------------- clocks --

class ClockSampler:
    """nvidia-smi clock / throttle-reason samples while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.out = None

    def __enter__(self):
        try:
            self.out = open(os.path.join("/tmp", f"emc_clocks_{os.getpid()}.csv"), "w+")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms",
                 "100", "-i", str(self.device)], stdout=self.out, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.out:
            return None
        self.out.seek(0)
        rows = [r.split(",") for r in self.out.read().strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[5 + i]
                          and "Not" not in r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# ------------------------------------------------------------ CPU baseline --

def sample_indices(d, max_rotations=2048):
    """An evenly strided subset of the rotations (every k-th): the CPU sample
    and the oracle parity sample of large workloads."""
    R = d["q"].shape[0]
    k = max(1, -(-R // max_rotations))
    return np.arange(0, R, k)


def cpu_oracle_rate(d, likelihood, interp, seconds, rot=None):
    """FP64 C++/OpenMP oracle (oracle/) on a bounded sample of the workload:
    the rotations `rot` (default: an evenly strided subset of at most 2048) and
    the first n patterns, n sized for about `seconds` of CPU work.  Returns
    (evals/s, sample text, oracle output (model, scaling, P, stats), n, rot)."""
    from oracle import oracle as O
    w = d["workload"]
    rot = sample_indices(d) if rot is None else rot
    r = len(rot)

    n_all = d["counts"].shape[0]

    def run(n):
        n = min(n, n_all)
        cfg = O.make_config(w.side, n, r, likelihood=O.LL_POISSON if likelihood == "poisson"
                            else O.LL_GAUSS, interp=O.NEAREST if interp == "nearest"
                            else O.TRILINEAR)
        t = time.perf_counter()
        out = O.iterate(cfg, d["counts"][:n], d["mask"], d["q"][rot], d["w"][rot], d["x"],
                        d["y"], d["z"], d["model0"], d["scaling0"][:n], want_resp=True)
        return time.perf_counter() - t, out

    n1, n2 = min(64, n_all), min(256, n_all)
    t8, _ = run(8)
    # per-pattern cost from two sizes (the fixed expand / insert cost cancels)
    if t8 < seconds / 8 and n1 > 8:
        t1, _ = run(n1)
        t2, _ = run(n2) if t1 < seconds / 4 and n2 > n1 else (None, None)
        if t2 is not None and t2 > t1:
            per = (t2 - t1) / (n2 - n1)
        else:
            per = max(t1 - t8, 1e-4) / (n1 - 8)
        base = t1
    else:
        per, base = t8 / 8, t8
    n = int(max(8, min(n_all, (seconds - base) / max(per, 1e-5))))
    n = min(n_all, max(8, (n // 8) * 8))
    t, out = run(n)
    R = d["q"].shape[0]
    return (n * r / t, f"1 FP64 iteration, {n} patterns x {r} rotations (every "
            f"{-(-R // r)}th of {R}; {t:.1f} s)", out, n, rot)


def sgemm_tflops(n=8192, reps=5):
    """cuBLAS FP32 GEMM on CUDA cores (TF32 off), best of `reps`: the FP32
    rate the plain path's contractions are measured against."""
    import torch
    prev = torch.get_float32_matmul_precision()
    torch.set_float32_matmul_precision("highest")
    x = torch.randn(n, n, device="cuda")
    y = torch.randn(n, n, device="cuda")
    torch.matmul(x, y)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(x, y)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    torch.set_float32_matmul_precision(prev)
    return 2.0 * n ** 3 / (best / 1e3) / 1e12


def compact(x):
    """Floats rounded to 4 significant digits, recursively (keeps the line short)."""
    if isinstance(x, float):
        return float(f"{x:.4g}") if math.isfinite(x) else None
    if isinstance(x, dict):
        return {k: compact(v) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [compact(v) for v in x]
    return x


def cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count()


def reference_arm(a):
    """--impl reference: the CPU implementation of the path (the FP64 oracle;
    the reference itself has no CPU iteration loop), all host threads."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from emc_b200 import workloads as W  # workload shapes only; the engine is not loaded
    from oracle import oracle as O
    O.build() if not os.path.isfile(O.LIB_PATH) else None
    w = workload_of(a)
    d = O.make_workload(w, wavelength=W.WAVELENGTH, distance=W.DISTANCE,
                        pixel_size=W.pixel_size(w.side))
    w = d["workload"]
    N, R = d["counts"].shape[0], d["q"].shape[0]
    for _ in range(max(0, min(a.warmup, 1))):
        cpu_oracle_rate(d, a.likelihood, a.interp, 2.0)
    rates, samples = [], []
    per = max(2.0, 90.0 / max(1, a.steps))
    for _ in range(a.steps):
        r, s, _, _, _ = cpu_oracle_rate(d, a.likelihood, a.interp, per)
        rates.append(r)
        samples.append(s)
    v = statistics.median(rates)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": N * R / v * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": config_desc(a, d),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores(), "kind": "port",
                         "sample": samples[-1] + "; extrapolated per evaluation to the full workload"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def workload_of(a):
    """The named workload with the --patterns / --rot-n overrides."""
    from emc_b200 import workloads as W
    w0 = W.WORKLOADS[a.workload]
    return W.Workload(w0.name, w0.side, a.rot_n or w0.rot_n, a.patterns or w0.n_patterns,
                      w0.mean_photons, w0.scale_sigma, w0.beamstop, w0.iterations, seed=w0.seed)


def config_desc(a, d):
    w = d["workload"]
    N, R = d["counts"].shape[0], d["q"].shape[0]
    npa = int((d["mask"] != 0).sum())
    return {"workload": f"{w.name}: {w.side}^3 model, {w.side}x{w.side} detector "
                        f"(beamstop r={w.beamstop:g}, {npa} active px), {R} rotations, {N} patterns, "
                        f"{a.likelihood} likelihood, {a.interp} interpolation",
            "precision": a.precision, "l2": "inputs larger than L2"} | (
        {"rotation_chunk": a.rotation_chunk} if getattr(a, "rotation_chunk", 0) else {}) | (
        {"insertion": "deterministic"} if getattr(a, "deterministic", False) else {})


# ------------------------------------------------------- learned proposal --

def oracle_columns(d, model, scaling, q, cols, likelihood, interp, chunk=6144):
    """The FP64 oracle's dense responsibilities [R][n] of patterns `cols`
    from (model, scaling): log-likelihoods against every rotation in chunks
    of rotations (bounded host memory), then the per-pattern softmax."""
    from oracle import oracle as O
    w = d["workload"]
    R, n = q.shape[0], len(cols)
    LL = np.empty((R, n), np.float64)
    counts, sc = d["counts"][cols], np.asarray(scaling, np.float64)[cols]
    for r0 in range(0, R, chunk):
        r1 = min(R, r0 + chunk)
        cfg = O.make_config(w.side, n, r1 - r0,
                            likelihood=O.LL_POISSON if likelihood == "poisson" else O.LL_GAUSS,
                            interp=O.NEAREST if interp == "nearest" else O.TRILINEAR)
        S = O.expand(cfg, model, q[r0:r1], d["x"], d["y"], d["z"])
        LL[r0:r1] = O.loglik(cfg, S, counts, d["mask"], sc)
    P, _, _ = O.softmax(LL)
    return P


def learned_proposal(a, E, W, d, device, dense_ms, dense_err):
    """The learned orientation proposal on the same data (rotations sorted
    into the 420 cells of the n=2 sampling): --train-iters dense iterations
    train the BF16 network on 90% of the patterns (10% held out); each
    proposed iteration then takes, per pattern, the cells holding the best of
    its previous log-posterior until they cover --top-k fine rotations (the
    configuration's 512 is reported beside it: it holds one step, but over 12
    chained iterations from this early state the posteriors' distant modes
    move outside its cells), adds
    the network's most probable cells up to a predicted mass of 0.999 (at most
    32 cells), and audits 64 patterns against every rotation: when one keeps
    less than 0.99 of its responsibility on its cells, the dense iteration
    runs instead.  Reports the timed chain of proposed iterations, the same
    selection without the network and the network alone, a forced fallback,
    the drift after 12 chained iterations, and errors against the dense
    iteration and the FP64 oracle."""
    import torch
    from emc_b200.proposal import LearnedProposal, sorted_rotations
    w = d["workload"]
    q, wt, cell, n_cells = sorted_rotations(d["q"], d["w"], coarse_n=2)
    N, R = d["counts"].shape[0], q.shape[0]
    ctx = E.Context(w.side, N, R, likelihood=a.likelihood, interp=a.interp, precision="mixed",
                    device=device)
    ctx.set_geometry(d["x"], d["y"], d["z"], d["mask"])
    ctx.set_rotations(q, wt)
    ctx.set_patterns(d["counts"])
    ctx.set_model(d["model0"])
    ctx.set_scaling(d["scaling0"])
    for _ in range(a.train_iters):
        ctx.iterate(stats=False)
    lp = LearnedProposal(ctx, cell, n_cells, bf16=True, seed=1)
    t0 = time.perf_counter()
    x, t_cur, lk = lp.features(), lp.targets(), lp.log_mass()
    perm = np.random.default_rng(0).permutation(N)
    held = torch.from_numpy(np.sort(perm[: N // 10])).cuda()
    train = torch.from_numpy(np.sort(perm[N // 10:])).cuda()
    losses = lp.train(x[train].contiguous(), t_cur[train].contiguous(), epochs=a.train_epochs,
                      batch=256, lr=2e-3)
    probs = lp.predict(x)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    top_k, max_cells, target, audit, min_cap = a.top_k, 32, 0.999, 64, 0.99

    def rel_err(m, ref):
        return float(np.linalg.norm(m - ref) / np.linalg.norm(ref))

    m0, s0 = ctx.get_model(), ctx.get_scaling()
    ctx.iterate(stats=False)  # the dense iteration from the same state
    m_dense, t_next = ctx.get_model(), lp.targets()

    def net_captured(scores, idx):
        """True mass of the step on the cells a network alone picks (its order,
        up to predicted mass 0.999, at most 16), for patterns idx."""
        sc, tn = scores[idx], t_next[idx]
        srt = torch.sort(sc, dim=1, descending=True)
        k = torch.clamp((torch.cumsum(srt.values, 1) < target).sum(1) + 1, max=16)
        sel = torch.arange(n_cells, device=sc.device)[None, :] < k[:, None]
        return float((torch.gather(tn, 1, srt.indices) * sel).sum(1).mean()), float(k.float().mean())

    untrained = LearnedProposal(ctx, cell, n_cells, bf16=True, seed=2)
    probs_u = untrained.predict(x)
    untrained.net.close()
    held_out = {"train_patterns": net_captured(probs, train)[0],
                "held_out_patterns": net_captured(probs, held)[0],
                "held_out_untrained": net_captured(probs_u, held)[0],
                "cells": net_captured(probs, held)[1]}

    def one_step(pr, keep):
        ctx.set_model(m0)
        ctx.set_scaling(s0)
        st = lp.iterate_topk(pr, keep, top_k, max_cells, target, audit, min_cap, a.keep_tail)
        cand = torch.isfinite(lp.log_mass())
        cap = (t_next * cand).sum(1)
        return st, ctx.get_model(), {
            "cells": round(st["pairs"] / N, 2), "rotations": round(st["evaluations"] / N, 1),
            "captured_min": float(cap.min()), "captured_mean": float(cap.mean()),
            "below_0.99": float((cap < 0.99).float().mean()), "fallback": st["fallback"],
            "model_err_vs_dense": rel_err(ctx.get_model(), m_dense)}

    variants = {}
    _, _, variants["no_network"] = one_step(None, lk)
    _, _, variants["network_only"] = one_step(probs, None)
    st1, m_prop, variants["with_network"] = one_step(probs, lk)
    variants["with_network"]["audit_min_captured"] = st1["audit_min_captured"]
    # responsibilities of sampled patterns against the FP64 oracle's dense ones
    cols = np.arange(0, N, max(1, N // a.oracle_patterns))[: a.oracle_patterns]
    P_prop = ctx.resp_columns(cols)
    P_orc = oracle_columns(dict(d, q=q), m0, s0, q, cols, a.likelihood, a.interp)
    l1 = np.abs(P_prop.astype(np.float64) - P_orc).sum(0)
    st_f, _, forced = one_step(None, torch.roll(lk, shifts=1, dims=0))

    # drift: 12 chained proposed iterations against 12 dense ones from the same state
    ctx.set_model(m0)
    ctx.set_scaling(s0)
    for _ in range(12):
        ctx.iterate(stats=False)
    m_d12 = ctx.get_model()

    def chain(k):
        ctx.set_model(m0)
        ctx.set_scaling(s0)
        keep, fb = lk, 0
        for _ in range(12):
            fb += lp.iterate_topk(probs, keep, k, max_cells, target, audit, min_cap,
                                  a.keep_tail)["fallback"]
            keep = lp.log_mass()
        return rel_err(ctx.get_model(), m_d12), fb

    drift, chain_fb = chain(top_k)
    # the configuration's own top-k (512 fine rotations): one step and 12 chained
    ctx.set_model(m0)
    ctx.set_scaling(s0)
    st512 = lp.iterate_topk(probs, lk, a.spec_top_k, max_cells, target, audit, min_cap, a.keep_tail)
    cap512 = (t_next * torch.isfinite(lp.log_mass())).sum(1)
    spec = {"top_k": a.spec_top_k, "cells": st512["pairs"] / N,
            "captured_min": float(cap512.min()),
            "model_err_vs_dense": rel_err(ctx.get_model(), m_dense)}
    spec["model_err_vs_dense_after_12"], spec["chain_fallbacks"] = chain(a.spec_top_k)

    # timed: chained proposed iterations (selection from the previous one)
    ctx.set_model(m0)
    ctx.set_scaling(s0)
    keep = lk
    for _ in range(2):
        lp.iterate_topk(probs, keep, top_k, max_cells, target, audit, min_cap, a.keep_tail)
        keep = lp.log_mass()
    ext = torch.cuda.ExternalStream(ctx.stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(ext):
        e0.record()
    evals = fallbacks = pairs = 0
    for _ in range(a.learned_steps):
        st = lp.iterate_topk(probs, keep, top_k, max_cells, target, audit, min_cap, a.keep_tail)
        keep = lp.log_mass()
        evals += st["evaluations"]
        pairs += st["pairs"]
        fallbacks += st["fallback"]
    with torch.cuda.stream(ext):
        e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.learned_steps
    ctx.set_profiling(True)
    stage = np.zeros(5)
    for i in range(3):
        lp.iterate_topk(probs, keep, top_k, max_cells, target, audit, min_cap, a.keep_tail)
        keep = lp.log_mass()
        if i >= 1:
            stage += ctx.stage_times()
    ctx.set_profiling(False)
    ctx.close()
    lp.net.close()
    return {
        "ms_per_step": ms, "top_k": top_k, "audit_patterns": audit, "min_captured": min_cap,
        **({"keep_tail": a.keep_tail} if a.keep_tail else {}),
        "fallback_iterations": fallbacks, "forced_fallback_iterations": st_f["fallback"],
        "cells_per_pattern": round(pairs / a.learned_steps / N, 2),
        "evaluated_fraction": evals / a.learned_steps / (N * R),
        "speedup_vs_dense_mixed": dense_ms / ms,
        "stages_ms": [round(float(v) / 2, 2) for v in stage],
        "one_step": variants, "held_out_captured": held_out,
        "model_err_vs_dense_after_12": drift, "chain_fallbacks": chain_fb, "spec_top_k": spec,
        "vs_fp64_oracle": {
            "resp_l1_max": float(l1.max()), "patterns": len(cols),
            "model_bound": variants["with_network"]["model_err_vs_dense"]
            + (dense_err or {}).get("model_rel_err", float("nan"))},
        "train_s": round(train_s, 1),
    }


# ------------------------------------------------------ batched datasets --

def batched_datasets(a, E, W, device, workloads, extra=None):
    """Six independent datasets (48 ... 128 px detectors), and `extra` (the
    headline dataset) with them when given, iterated (1) one
    after the other, each with its own launches, and (2) together: one
    persistent launch per contraction over the datasets' tiles (a dataset
    that fills the GPU alone keeps its own), the whole iteration captured in
    a CUDA graph and replayed."""
    import torch
    data = [W.make(w) for w in workloads] + ([extra] if extra is not None else [])
    ctxs, b = [], None
    try:
        for d in data:
            w = d["workload"]
            c = E.Context(w.side, d["counts"].shape[0], d["q"].shape[0], likelihood=a.likelihood,
                          interp=a.interp, precision="mixed", device=device)
            ctxs.append(c)
            c.set_geometry(d["x"], d["y"], d["z"], d["mask"])
            c.set_rotations(d["q"], d["w"])
            c.set_patterns_sparse(*E.photon_lists(d["counts"]))
            c.set_model(d["model0"])
            c.set_scaling(d["scaling0"])
        K = a.batch_steps

        def device_ms(stream, fn):
            ext = torch.cuda.ExternalStream(stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            with torch.cuda.stream(ext):
                e0.record()
            fn()
            with torch.cuda.stream(ext):
                e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1)

        # (1) one after the other (each context on its own stream, serialised),
        # after the three warm-up iterations the graph below also gets (an early
        # iteration whose responsibility lists outgrow their first capacity runs
        # the dense compress once and is not the steady state)
        for c in ctxs:
            for _ in range(3):
                c.iterate(stats=False)
        sep = 0.0
        for c in ctxs:
            sep += device_ms(c.stream, lambda c=c: [c.iterate(stats=False) for _ in range(K)]) / K
        # (2) one batch, CUDA graph
        b = E.Batch(ctxs)
        b.iterate()
        b.capture()
        b.launch(2)
        b.synchronize()
        ms = device_ms(b.stream, lambda: b.launch(K)) / K
        b.synchronize()
        ok = all(np.isfinite(c.get_model()).all() for c in ctxs)
    finally:
        if b is not None:
            b.close()
        for c in ctxs:
            c.close()
    assert ok, "batched iteration gave a non-finite model"
    return {"separate_ms": round(sep, 2), "graph_ms": round(ms, 2), "speedup": round(sep / ms, 3)}


# ------------------------------------------------------------------ ours --

def profile_case(a):
    """Small fixed cases whose kernels the summaries under profiles/ come from
    (run once plainly, then under ncu).  Prints wall-clock times per
    iteration, nothing else."""
    import torch
    import emc_b200 as E
    from emc_b200 import workloads as W
    from emc_b200.proposal import LearnedProposal, sorted_rotations
    if a.profile_case == "proposed":
        wl, dense, proposed = W.WORKLOADS["large128"], 2, 3
    elif a.profile_case == "expand":
        wl, dense, proposed = W.Workload("prof128", 128, 8, 2000, 500.0, 0.5, 6.0, 1), 3, 0
    else:
        wl, dense, proposed = W.Workload("prof128", 128, 8, 20000, 500.0, 0.5, 6.0, 1), 1, 2
    d = W.make(wl)
    q, w = d["q"], d["w"]
    if proposed:
        q, w, cell, n_cells = sorted_rotations(q, w)
    N, R = d["counts"].shape[0], q.shape[0]
    ctx = E.Context(wl.side, N, R, likelihood="poisson", precision="mixed")
    ctx.set_geometry(d["x"], d["y"], d["z"], d["mask"])
    ctx.set_rotations(q, w)
    ctx.set_patterns(d["counts"])
    ctx.set_model(d["model0"])
    ctx.set_scaling(d["scaling0"])
    for i in range(dense):
        t0 = time.perf_counter()
        ctx.iterate(stats=False)
        ctx.synchronize()
        print(f"dense {i}: {(time.perf_counter() - t0) * 1e3:.2f} ms", flush=True)
    if proposed:
        lp = LearnedProposal(ctx, cell, n_cells)
        keep = lp.log_mass()  # the dense posterior selects the first proposed iteration
        for i in range(proposed):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            st = lp.iterate_topk(None, keep, 2048, 32, audit=64)
            keep = lp.log_mass()
            ctx.synchronize()
            print(f"proposed {i}: {(time.perf_counter() - t0) * 1e3:.2f} ms, "
                  f"{st['pairs'] / N:.2f} cells per pattern", flush=True)
    ctx.close()


def main():
    a = parse()
    if a.impl == "reference":
        return reference_arm(a)
    if a.profile_case:
        return profile_case(a)
    import torch
    import emc_b200 as E
    from emc_b200 import workloads as W

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    wl = workload_of(a)
    d = W.make(wl, first_pattern=rank * wl.n_patterns)  # this rank's shard of one dataset
    N, R = d["counts"].shape[0], d["q"].shape[0]
    npa = int((d["mask"] != 0).sum())

    def make_ctx(precision):
        c = E.Context(wl.side, N, R, likelihood=a.likelihood, interp=a.interp,
                      precision=precision, device=local)
        c.set_geometry(d["x"], d["y"], d["z"], d["mask"])
        c.set_rotations(d["q"], d["w"])
        c.set_patterns(d["counts"])
        c.set_model(d["model0"])
        c.set_scaling(d["scaling0"])
        if a.rotation_chunk and precision == "mixed":
            c.set_rotation_chunk(a.rotation_chunk)
        if a.deterministic:
            c.set_deterministic(True)
        return c

    from emc_b200.parallel import ShardedIteration

    def timed(ctx, steps, warmup):
        """Device time per step (max over ranks), per-stage times, launches per step."""
        ext = torch.cuda.ExternalStream(ctx.stream)
        step = ShardedIteration(ctx)  # single GPU: expand, maximize, insert, normalise
        for _ in range(warmup):
            step()
        ctx.synchronize()
        l0 = ctx.launch_count
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(ext):
            e0.record()
        for _ in range(steps):
            step()
        with torch.cuda.stream(ext):
            e1.record()
        torch.cuda.synchronize()
        ctx.synchronize()
        ms = e0.elapsed_time(e1)
        launches = (ctx.launch_count - l0) / steps
        if dist:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        # stage times: events recorded inside each iteration, read one
        # iteration behind so the stream never drains
        ctx.set_profiling(True)
        stage, n = np.zeros(5), 0
        for i in range(min(steps, 8) + 1):
            step()
            if i >= 1:
                stage += ctx.stage_times()
                n += 1
        ctx.synchronize()
        ctx.set_profiling(False)
        return ms / steps, stage / max(n, 1), launches

    ctx = make_ctx(a.precision)
    clocks = ClockSampler(local)
    with clocks:
        ms_step, stage_ms, launches = timed(ctx, a.steps, a.warmup)
    clk = clocks.summary()
    value = N * R * world / (ms_step / 1e3)

    pk, pk_kind = peaks()
    # roofline of the dominant kernel: the maximize contraction
    gemm_ms = float(stage_ms[1])
    flops = 2.0 * N * R * npa
    achieved = flops / (gemm_ms / 1e3) / 1e12 if gemm_ms > 0 else None
    peak = pk["bf16_tflops_sustained"]
    roof = {"bound": "tensor", "kernel": "maximize contraction (tcgen05 cta_group::2 pairs, FP16 hi+lo)"
            if a.precision == "mixed" else "maximize contraction (FP32 CUDA cores)",
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak if achieved else None,
            "peak_kind": f"{pk_kind} bf16 dense, sustained",
            "traffic": MAXIMIZE_TRAFFIC_BYTES if a.workload == "large128" and N == 50_000
            and a.precision == "mixed" else None,
            "algorithmic_flops_per_launch": flops,
            "launch_ms": gemm_ms}
    stages = dict(zip(["expand", "maximize_contraction", "responsibility_pass", "compress_insert",
                       "normalise"], [round(float(x), 4) for x in stage_ms]))

    # e2e through the public API with host buffers (pinned), copies in the timed region
    e2e = None
    if not a.no_e2e:
        # sparse data (the 128^3 patterns are ~3% non-zero) crosses the bus as
        # photon lists (emc_set_patterns_sparse), dense data as images
        sparse = float(np.count_nonzero(d["counts"])) < 0.25 * d["counts"].size

        def pinned_copy(x):
            t = torch.empty(x.size, dtype={np.float32: torch.float32, np.int32: torch.int32,
                                           np.int64: torch.int64}[x.dtype.type], pin_memory=True)
            v = t.numpy().reshape(x.shape)
            v[:] = x
            return v

        if sparse:
            host_lists = tuple(pinned_copy(v) for v in E.photon_lists(d["counts"]))
            upload = lambda: ctx.set_patterns_sparse(*host_lists)  # noqa: E731
            up_bytes = sum(v.nbytes for v in host_lists)
        else:
            host_counts = pinned_copy(d["counts"])
            upload = lambda: ctx.set_patterns(host_counts)  # noqa: E731
            up_bytes = host_counts.nbytes
        pm = torch.empty(d["model0"].size, dtype=torch.float32, pin_memory=True).numpy()
        pm[:] = d["model0"]
        ps = torch.empty(N, dtype=torch.float32, pin_memory=True).numpy()
        ps[:] = 1.0
        ext = torch.cuda.ExternalStream(ctx.stream)
        steps_e = max(3, min(a.steps, 10))
        step = ShardedIteration(ctx)
        for _ in range(2):
            upload()
            ctx.set_model(pm)
            ctx.set_scaling(ps)
            step()
            m = ctx.get_model()
            s = ctx.get_scaling()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(ext):
            e0.record()
        parts = np.zeros(4)
        for _ in range(steps_e):
            t0 = time.perf_counter()
            upload()
            t1 = time.perf_counter()
            ctx.set_model(pm)
            ctx.set_scaling(ps)
            step()
            t2 = time.perf_counter()
            m = ctx.get_model()
            t3 = time.perf_counter()
            s = ctx.get_scaling()
            t4 = time.perf_counter()
            parts += [t1 - t0, t2 - t1, t3 - t2, t4 - t3]
        with torch.cuda.stream(ext):
            e1.record()
        torch.cuda.synchronize()
        ms_e = e0.elapsed_time(e1) / steps_e
        if dist:
            t = torch.tensor([ms_e], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms_e = float(t.item())
        assert np.isfinite(m).all() and np.isfinite(s).all()
        e2e = {"value": N * R * world / (ms_e / 1e3), "unit": UNIT, "ms_per_step": ms_e,
               "h2d_bytes_per_step": int(up_bytes + pm.nbytes + ps.nbytes),
               "d2h_bytes_per_step": int(m.nbytes + s.nbytes),
               "api": "photon lists" if sparse else "images"}

    ctx.close()

    # The error of this path against the FP64 oracle on a sample (the oracle
    # cannot run the full workload in seconds): the same patterns and an
    # evenly strided subset of the rotations through a context of that size;
    # the oracle's time on it is the CPU baseline.
    cpu = None
    err = None
    if rank == 0 and world == 1 and not a.no_cpu:
        rate, sample, (m_ref, s_ref, P_ref, _), n, rot = cpu_oracle_rate(
            d, a.likelihood, a.interp, a.cpu_seconds)
        cpu = {"value": rate, "unit": UNIT, "cores": cores(), "kind": "port",
               "sample": sample + " (C++/OpenMP FP64 oracle)"}
        sub = E.Context(wl.side, n, len(rot), likelihood=a.likelihood, interp=a.interp,
                        precision=a.precision, device=local)
        sub.set_geometry(d["x"], d["y"], d["z"], d["mask"])
        sub.set_rotations(d["q"][rot], d["w"][rot])
        sub.set_patterns(d["counts"][:n])
        sub.set_model(d["model0"])
        sub.set_scaling(d["scaling0"][:n])
        sub.expand()
        sub.maximize()
        P = sub.get_buffer(E.BUF_RESP)
        sub.compress()
        m_sub = sub.get_model()
        sub.close()
        diff = np.abs(P.astype(np.float64) - P_ref).sum(0)
        err = {"resp_l1_max": float(diff.max()), "resp_l1_mean": float(diff.mean()),
               "model_rel_err": float(np.linalg.norm(m_sub - m_ref) / np.linalg.norm(m_ref)),
               "patterns": n, "rotations": len(rot)}

    learned = None
    if rank == 0 and world == 1 and not a.no_learned and a.precision == "mixed":
        learned = learned_proposal(a, E, W, d, local, ms_step, err)

    batch = None
    if rank == 0 and world == 1 and not a.no_batch and a.precision == "mixed":
        def batch_case(*args, **kw):
            # a side measurement: its failure (say, device memory taken by
            # another process) is reported in its place, not the whole line lost
            try:
                return batched_datasets(a, E, W, local, *args, **kw)
            except (E.EmcError, RuntimeError, MemoryError) as ex:
                torch.cuda.synchronize()
                return {"unavailable": str(ex)[:120]}
        batch = {"large": batch_case(W.BATCH6),
                 "large_with_headline": batch_case(W.BATCH6, extra=d),
                 "small": batch_case(W.BATCH6_SMALL)}

    fp32 = None
    if rank == 0 and world == 1 and not a.no_fp32 and a.precision == "mixed":
        c32 = make_ctx("fp32")
        ms32, st32, _ = timed(c32, a.fp32_steps, 1)
        c32.close()
        sgemm = sgemm_tflops()
        fp32 = {"ms_per_step": ms32, "maximize_ms": float(st32[1]),
                "maximize_tflops": flops / (st32[1] / 1e3) / 1e12,
                "sgemm_tflops": sgemm}
        fp32["maximize_frac_of_sgemm"] = fp32["maximize_tflops"] / sgemm
        if a.likelihood == "poisson":
            # the same FP32 iteration with both contractions as gathers over
            # the non-zero counts (photon lists)
            c32 = make_ctx("fp32")
            c32.set_sparse_maximize(True)
            c32.set_sparse_compress(True)
            mss, sts, _ = timed(c32, a.fp32_steps, 1)
            c32.set_model(d["model0"])
            c32.set_scaling(d["scaling0"])
            c32.iterate(stats=False)
            m_sparse = c32.get_model()
            c32.close()
            c32 = make_ctx("fp32")
            c32.iterate(stats=False)
            m_plain = c32.get_model()
            c32.close()
            fp32["photon_lists"] = {
                "ms_per_step": mss, "maximize_ms": float(sts[1]),
                "model_err_vs_dense_fp32": float(np.linalg.norm(m_sparse - m_plain) /
                                                 np.linalg.norm(m_plain))}

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    # the plain FP32 iteration of the metric: the faster of the two FP32 forms
    # (dense CUDA-core contractions, or both contractions over photon lists)
    plain = None
    if fp32:
        plain = min(fp32["ms_per_step"], (fp32.get("photon_lists") or {}).get("ms_per_step", 1e30))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f16 hi+lo, f32 acc, f64 lse" if a.precision == "mixed" else "f32",
        "data": "synthetic (seeded)",
        "config": config_desc(a, d),
        "s_per_iter_mixed": ms_step / 1e3,
        "s_per_iter_learned": learned["ms_per_step"] / 1e3 if learned else None,
        "s_per_iter_plain_fp32": plain / 1e3 if plain else None,
        "speedup_learned_vs_plain_fp32": plain / learned["ms_per_step"] if plain and learned else None,
        "speedup_mixed_vs_plain_fp32": plain / ms_step if plain else None,
        "error_vs_fp64_oracle": {
            "mixed": {k: err[k] for k in ("resp_l1_max", "model_rel_err")} if err else None,
            "learned": learned["vs_fp64_oracle"] if learned else None},
        "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
        "gpu_launches": launches,
        "stages_ms": stages, "learned": learned, "plain_fp32": fp32, "batched": batch,
    }
    if learned:
        learned.pop("vs_fp64_oracle")
        # per variant: [cells per pattern, min captured mass, model error vs dense, fallback]
        learned["one_step"] = {k: [v["cells"], v["captured_min"], v["model_err_vs_dense"],
                                   v["fallback"]] for k, v in learned["one_step"].items()}
        learned["held_out_captured"] = [learned["held_out_captured"][k] for k in
                                        ("train_patterns", "held_out_patterns",
                                         "held_out_untrained")]
    for k in ("kernel", "peak_kind", "algorithmic_flops_per_launch"):
        roof.pop(k, None)
    line = compact(line)
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
