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
"""
from __future__ import annotations

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
