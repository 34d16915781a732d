"""Shared helpers of the parity tests: run the engine and the FP64 oracle on
the same seeded inputs and measure their differences."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def resp_l1(P, Pref):
    """max over patterns of sum_r |P - Pref| (responsibilities sum to 1 per pattern)."""
    return float(np.abs(np.asarray(P, np.float64) - Pref).sum(axis=0).max())


def oracle_cfg(d, likelihood="gauss", interp="nearest", sigma=0.4, floor=1e-10):
    w = d["workload"]
    return O.make_config(w.side, d["counts"].shape[0], d["q"].shape[0],
                         likelihood=O.LL_GAUSS if likelihood == "gauss" else O.LL_POISSON,
                         interp=O.NEAREST if interp == "nearest" else O.TRILINEAR,
                         sigma=sigma, poisson_floor=floor)


def make_ctx(d, likelihood="gauss", interp="nearest", precision="fp32", sigma=0.4, floor=1e-10):
    import emc_b200 as E
    w = d["workload"]
    ctx = E.Context(w.side, d["counts"].shape[0], d["q"].shape[0], likelihood=likelihood,
                    interp=interp, precision=precision, sigma=sigma, poisson_floor=floor)
    ctx.set_geometry(d["x"], d["y"], d["z"], d["mask"])
    ctx.set_rotations(d["q"], d["w"])
    ctx.set_patterns(d["counts"])
    ctx.set_model(d["model0"])
    ctx.set_scaling(d["scaling0"])
    return ctx


def active(d):
    return np.nonzero(d["mask"] != 0)[0]
