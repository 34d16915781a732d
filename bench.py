#!/usr/bin/env python
"""EMC iteration throughput on B200: pattern x rotation evaluations per second.

One step = one full EMC iteration (expand -> maximize -> compress, emc.c:989-1084)
over every pattern and rotation of the workload, inputs resident in HBM.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Default workload: 64^3 model, 64x64 detector with a radius-4 beamstop (4044
active pixels), 25,680 rotations (600-cell n=8, halved), 10,000 seeded
synthetic Poisson patterns (mean 2000 photons, lognormal scale sigma 0.5).
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
# DRAM bytes per launch of the maximize contraction on the default workload,
# from the ncu capture summarised in profiles/ (None until captured).
MAXIMIZE_TRAFFIC_BYTES = None


def parse():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="b200_64")
    ap.add_argument("--patterns", type=int, default=None, help="override the pattern count")
    ap.add_argument("--likelihood", default="poisson", choices=["poisson", "gauss"])
    ap.add_argument("--interp", default="nearest", choices=["nearest", "trilinear"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp32"])
    ap.add_argument("--fp32-steps", type=int, default=3, help="steps of the plain FP32 comparison")
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
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

def cpu_oracle_rate(d, likelihood, interp, seconds, want_resp_rows=None):
    """FP64 C++/OpenMP oracle (oracle/) on a bounded sample of the workload:
    every rotation, the first n patterns.  Returns (evals/s, sample text, P)."""
    from oracle import oracle as O
    w = d["workload"]
    R = d["q"].shape[0]

    def run(n):
        cfg = O.make_config(w.side, n, R, likelihood=O.LL_POISSON if likelihood == "poisson"
                            else O.LL_GAUSS, interp=O.NEAREST if interp == "nearest"
                            else O.TRILINEAR)
        t = time.perf_counter()
        _, _, P, _ = O.iterate(cfg, d["counts"][:n], d["mask"], d["q"], d["w"], d["x"], d["y"],
                               d["z"], d["model0"], d["scaling0"][:n], want_resp=True)
        return time.perf_counter() - t, P

    t8, _ = run(8)
    n = int(max(8, min(d["counts"].shape[0], 8 * seconds / max(t8, 1e-3) * 0.8)))
    n = max(8, (n // 8) * 8)
    t, P = run(n)
    return n * R / t, f"1 FP64 iteration, {n} patterns x {R} rotations ({t:.1f} s)", P, n


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
    from emc_b200 import workloads as W
    from oracle import oracle as O
    O.build() if not os.path.isfile(O.LIB_PATH) else None
    d = W.make(a.workload, n_patterns=a.patterns)
    w = d["workload"]
    N, R = d["counts"].shape[0], d["q"].shape[0]
    for _ in range(max(0, min(a.warmup, 1))):
        cpu_oracle_rate(d, a.likelihood, a.interp, 2.0)
    rates, samples = [], []
    per = max(2.0, 60.0 / max(1, a.steps))
    for _ in range(a.steps):
        r, s, _, _ = cpu_oracle_rate(d, a.likelihood, a.interp, per)
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


def config_desc(a, d):
    w = d["workload"]
    N, R = d["counts"].shape[0], d["q"].shape[0]
    npa = int((d["mask"] != 0).sum())
    return {"workload": f"{w.name}: {w.side}^3 model, {w.side}x{w.side} detector "
                        f"(beamstop r={w.beamstop:g}, {npa} active px), {R} rotations, {N} patterns, "
                        f"{a.likelihood} likelihood, {a.interp} interpolation",
            "precision": a.precision, "patterns": N, "rotations": R, "active_pixels": npa,
            "l2": "inputs larger than L2 (responsibility matrix and slice operands > 126 MB)"}


# ------------------------------------------------------------------ ours --

def main():
    a = parse()
    if a.impl == "reference":
        return reference_arm(a)
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
    w0 = W.WORKLOADS[a.workload]
    wl = W.Workload(w0.name, w0.side, w0.rot_n, a.patterns or w0.n_patterns, w0.mean_photons,
                    w0.scale_sigma, w0.beamstop, w0.iterations, seed=w0.seed)
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
    roof = {"bound": "tensor", "kernel": "maximize contraction (tcgen05, FP16 hi+lo)"
            if a.precision == "mixed" else "maximize contraction (FP32 CUDA cores)",
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak if achieved else None,
            "peak_kind": f"{pk_kind} bf16 dense, sustained",
            "traffic": MAXIMIZE_TRAFFIC_BYTES,
            "algorithmic_flops_per_launch": flops,
            "launch_ms": gemm_ms}
    stages = dict(zip(["expand", "maximize_contraction", "responsibility_pass", "compress_insert",
                       "normalise"], [round(float(x), 4) for x in stage_ms]))

    # e2e through the public API with host buffers (pinned), copies in the timed region
    e2e = None
    if not a.no_e2e:
        pinned = torch.empty(d["counts"].size, dtype=torch.float32, pin_memory=True)
        host_counts = pinned.numpy().reshape(d["counts"].shape)
        host_counts[:] = d["counts"]
        pm = torch.empty(d["model0"].size, dtype=torch.float32, pin_memory=True).numpy()
        pm[:] = d["model0"]
        ps = torch.empty(N, dtype=torch.float32, pin_memory=True).numpy()
        ps[:] = 1.0
        ext = torch.cuda.ExternalStream(ctx.stream)
        steps_e = max(3, min(a.steps, 10))
        step = ShardedIteration(ctx)
        for _ in range(2):
            ctx.set_patterns(host_counts)
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
            ctx.set_patterns(host_counts)
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
               "h2d_bytes_per_step": int(host_counts.nbytes + pm.nbytes + ps.nbytes),
               "d2h_bytes_per_step": int(m.nbytes + s.nbytes),
               "api": "emc_set_patterns/model/scaling + expand/maximize/compress (+ all-reduce) "
                      "+ emc_get_model/scaling",
               "host_ms": dict(zip(["set_patterns", "enqueue_iteration", "get_model",
                                    "get_scaling"], [round(x * 1e3 / steps_e, 3) for x in parts]))}

    # responsibility error of this path vs the FP64 oracle on a sample, and the CPU baseline
    cpu = None
    err = None
    if rank == 0 and world == 1 and not a.no_cpu:
        ctx.set_model(d["model0"])
        ctx.set_scaling(d["scaling0"])
        ctx.set_patterns(d["counts"])
        ctx.expand()
        ctx.maximize()
        P = ctx.get_buffer(E.BUF_RESP)
        rate, sample, P_ref, n = cpu_oracle_rate(d, a.likelihood, a.interp, a.cpu_seconds)
        cpu = {"value": rate, "unit": UNIT, "cores": cores(), "kind": "port",
               "sample": sample + " (C++/OpenMP FP64 oracle)"}
        diff = np.abs(P[:, :n].astype(np.float64) - P_ref).sum(0)
        err = {"resp_l1_max": float(diff.max()), "resp_l1_mean": float(diff.mean()),
               "sample_patterns": n, "vs": "FP64 oracle, same model and scaling"}
        ctx.compress()
    ctx.close()

    fp32 = None
    if not a.no_fp32 and a.precision == "mixed":
        c32 = make_ctx("fp32")
        ms32, st32, _ = timed(c32, a.fp32_steps, 1)
        c32.close()
        fp32 = {"value": N * R * world / (ms32 / 1e3), "ms_per_step": ms32,
                "stages_ms": [round(float(x), 3) for x in st32],
                "speedup_of_mixed": ms32 / ms_step}

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms_step, "s_per_iter": ms_step / 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f16 hi+lo operands, f32 accumulate, f64 lse" if a.precision == "mixed" else "f32",
        "data": "synthetic (seeded point-scatterer model, Poisson patterns)",
        "config": config_desc(a, d),
        "stages_ms": stages, "roofline": roof, "cpu_baseline": cpu, "error": err,
        "plain_fp32": fp32, "e2e": e2e, "clocks": clk, "gpu_launches": launches,
    }
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
