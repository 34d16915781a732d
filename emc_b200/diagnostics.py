"""Per-iteration output in the files the reference's viewer reads.

The viewer (viewer/*.py of the reference) loads, with numpy.loadtxt:
``likelihood.data`` (one value per iteration, likelihood_module.py:24),
``best_rot.data`` (one row of best rotation indices per iteration,
rotations_module.py:87), ``average_resp_%04d.data`` (the average
responsibility of every rotation, rotations_module.py:47).  The scaling
history it reads from ``best_scaling.h5`` (scaling_module.py:19) is written
here as text, ``best_scaling.data`` (one row per iteration), since this
package has no HDF5 writer; the model goes to ``model_%04d.raw`` (emc_model_save:
raw float32, the format emc_model_load reads).

``metrics.jsonl`` (MetricsLog) holds one JSON object per iteration for
tooling: the FP64 total log-likelihood and sum P log P, the model maximum,
the scaling statistics, the stage times, the throughput and any error
against the oracle the caller measured.
"""
from __future__ import annotations

import json
import os

import numpy as np

from . import Context, save_model


class OutputWriter:
    """Appends one iteration's record per call to `record`."""

    def __init__(self, directory: str, save_models: bool = True):
        self.dir = directory
        self.save_models = save_models
        os.makedirs(directory, exist_ok=True)

    def _path(self, name):
        return os.path.join(self.dir, name)

    def record(self, iteration: int, ctx: Context, sum_plogp: float):
        """The record of the iteration that `ctx` ran last: sum_r P log P (the
        reference's logged likelihood), best rotations, scaling, average
        responsibilities and the model."""
        o = ctx.orientation_stats()
        with open(self._path("likelihood.data"), "a") as f:
            f.write(f"{sum_plogp:.17g}\n")
        with open(self._path("best_rot.data"), "a") as f:
            f.write(" ".join(str(int(v)) for v in o["best_rot"]) + "\n")
        with open(self._path("best_scaling.data"), "a") as f:
            f.write(" ".join(f"{v:.9g}" for v in ctx.get_scaling()) + "\n")
        np.savetxt(self._path("average_resp_%.4d.data" % iteration), o["avg_resp"], fmt="%.9g")
        if self.save_models:
            save_model(self._path("model_%.4d.raw" % iteration), ctx.get_model(), ctx.side)
        return o


class MetricsLog:
    """Appends one JSON object per iteration to ``metrics.jsonl``."""

    def __init__(self, directory: str, name: str = "metrics.jsonl"):
        os.makedirs(directory, exist_ok=True)
        self.path = os.path.join(directory, name)

    def record(self, iteration: int, ctx, stats: dict, seconds: float | None = None,
               stages_ms=None, errors: dict | None = None) -> dict:
        """stats: the dict `Context.iterate()` returns (total_loglik and
        sum_plogp in FP64, model_max, total_resp); seconds: the iteration's
        time, for the pattern x rotation evaluations per second; stages_ms:
        `Context.stage_times()` when profiling is on; errors: e.g. the
        responsibility and model errors against the FP64 oracle."""
        sc = np.asarray(ctx.get_scaling(), np.float64)
        rec = {"iteration": int(iteration),
               "total_loglik": float(stats["total_loglik"]),
               "sum_plogp": float(stats["sum_plogp"]),
               "model_max": float(stats["model_max"]),
               "total_resp": float(stats["total_resp"]),
               "scaling": {"mean": float(sc.mean()), "min": float(sc.min()),
                           "max": float(sc.max())}}
        if stages_ms is not None:
            rec["stages_ms"] = [round(float(v), 4) for v in stages_ms]
        if seconds:
            rec["seconds"] = float(seconds)
            rec["evals_per_s"] = float(ctx.N) * float(ctx.R) / float(seconds)
        if errors:
            rec["errors"] = {k: float(v) for k, v in errors.items()}
        with open(self.path, "a") as f:
            f.write(json.dumps(rec) + "\n")
        return rec
