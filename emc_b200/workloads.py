"""Seeded synthetic EMC workloads with the shapes of the benchmark configurations.

No public dataset is involved: every workload is generated from a seed by the
library's own generator (emc_synthesize).  Geometry: lambda = 1 A and the
detector distance / pixel size chosen so that the pixel at the middle of the
detector edge sits at a 30 degree scattering angle; coordinates are in pixel
units, so q_max falls on the grid edge by construction.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import detector_coordinates, generate_rotations, random_model, synthesize

WAVELENGTH = 1e-10
DISTANCE = 1.0
EDGE_ANGLE_DEG = 30.0


@dataclass(frozen=True)
class Workload:
    name: str
    side: int
    rot_n: int            # 600-cell refinement (halved list: 420 / 3240 / 25680 / 86520)
    n_patterns: int
    mean_photons: float
    scale_sigma: float
    beamstop: float       # pixels; 0 = no mask
    iterations: int
    seed: int = 0


WORKLOADS = {
    # plain EMC on CPU, FP64 (32^3, 3240 rotations, 1000 patterns, 10 iterations)
    "cpu32": Workload("cpu32", 32, 4, 1000, 1000.0, 0.3, 0.0, 10),
    # plain FP32 drop-in / mixed precision on one B200 (64^3, 25680 rotations, 10k patterns)
    "b200_64": Workload("b200_64", 64, 8, 10_000, 2000.0, 0.5, 4.0, 20),
    # large case (128^3, 86520 rotations, 50k patterns, ~3% non-zero pixels)
    "large128": Workload("large128", 128, 12, 50_000, 500.0, 0.5, 6.0, 1),
    # small cases for tests
    "tiny16": Workload("tiny16", 16, 2, 64, 400.0, 0.3, 1.5, 3),
    "small32": Workload("small32", 32, 4, 256, 1000.0, 0.3, 2.0, 3),
}


# Batched case: six independent datasets of different detector sizes
# (48 ... 128 px, 2k ... 20k patterns), each with its model side equal to the
# detector side and an orientation sampling proportional to it (600-cell n
# from 5 at 48 px to 12 at 128 px), beamstop radius 6 and 500 photons on
# average as in large128.
BATCH6 = [Workload(f"batch{s}", s, n, N, 500.0, 0.5, 6.0, 1, seed=10 + i)
          for i, (s, n, N) in enumerate([(48, 5, 2000), (64, 6, 5000), (80, 8, 8000),
                                         (96, 9, 11000), (112, 10, 14000), (128, 12, 20000)])]


# The same detector sizes with 500 patterns and 3,240 rotations each: a
# dataset whose contractions alone fill about a third of the GPU.
BATCH6_SMALL = [Workload(f"small{s}", s, 4, 500, 500.0, 0.5, 6.0, 1, seed=20 + i)
                for i, s in enumerate([48, 64, 80, 96, 112, 128])]


def pixel_size(side: int) -> float:
    return math.tan(math.radians(EDGE_ANGLE_DEG)) * DISTANCE / (side / 2)


def make(w: Workload | str, n_patterns: int | None = None, first_pattern: int = 0):
    """Returns dict(x, y, z, mask, counts, rotations q, weights w, model0, true_model, ...).

    first_pattern selects a shard of the seeded pattern sequence (the model,
    mask and rotations do not depend on it)."""
    if isinstance(w, str):
        w = WORKLOADS[w]
    N = n_patterns or w.n_patterns
    x, y, z = detector_coordinates(w.side, WAVELENGTH, pixel_size(w.side), DISTANCE)
    d = synthesize(w.side, N, x, y, z, mean_photons=w.mean_photons, scale_sigma=w.scale_sigma,
                   beamstop_radius=w.beamstop, seed=w.seed, first_pattern=first_pattern)
    q, wt = generate_rotations(w.rot_n, halve=True)
    return dict(workload=w, x=x, y=y, z=z, mask=d["mask"], counts=d["counts"], q=q, w=wt,
                model0=random_model(w.side, w.seed), true_model=d["model"],
                true_rotations=d["rotations"], true_scales=d["scales"],
                scaling0=np.ones(N, np.float32))
