"""ctypes wrapper of the FP64 oracle (liboracle.so).  TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline /
reference leg import this module; the product package never does.  Each
function cites the reference lines it restates (paths inside FilipeMaia/emc).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

LL_GAUSS, LL_POISSON = 0, 1
NEAREST, TRILINEAR = 0, 1


class Config(C.Structure):
    _fields_ = [
        ("side", C.c_int32),
        ("likelihood", C.c_int32),
        ("interp", C.c_int32),
        ("pad_", C.c_int32),
        ("n_patterns", C.c_int64),
        ("n_rotations", C.c_int64),
        ("sigma", C.c_double),
        ("poisson_floor", C.c_double),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("sum_plogp", C.c_double),
        ("total_loglik", C.c_double),
        ("model_max", C.c_double),
        ("total_resp", C.c_double),
    ]


def reference_dir() -> str:
    """The reference checkout: $EMC_REFERENCE_DIR, else a sibling directory
    `reference` of the repository (absent on machines that only run tests)."""
    return os.environ.get("EMC_REFERENCE_DIR") or os.path.abspath(
        os.path.join(HERE, os.pardir, os.pardir, "reference"))


def build() -> None:
    """Compile liboracle.so (and oracle/_ref when the reference sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if os.path.isfile(os.path.join(reference_dir(), "emc.c")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={reference_dir()}"], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.isfile(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        P = C.c_void_p
        _lib.orc_n_to_samples.restype = C.c_int64
        _lib.orc_generate_rotations.restype = C.c_int64
        _lib.orc_generate_rotations.argtypes = [C.c_int, C.c_int, P, P]
        _lib.orc_coordinates.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, P, P, P]
        _lib.orc_rotation_matrix_f32.argtypes = [P, P]
        _lib.orc_expand.argtypes = [P] * 7
        _lib.orc_loglik.argtypes = [P] * 6
        _lib.orc_loglik_gauss_direct.argtypes = [P] * 6
        _lib.orc_softmax.argtypes = [C.c_int64, C.c_int64, P, P]
        _lib.orc_softmax.restype = C.c_double
        _lib.orc_update_scaling.argtypes = [P] * 6
        _lib.orc_compress.argtypes = [P] * 13
        _lib.orc_slice_average.argtypes = [P] * 7
        _lib.orc_insert.argtypes = [P] * 11
        _lib.orc_normalize_model.argtypes = [C.c_int64, P, P]
        _lib.orc_iterate.argtypes = [P] * 12
        _lib.orc_iterate_restricted.argtypes = [P] * 13
        _lib.orc_insert_shard.argtypes = [P] * 12
        _lib.orc_random_model.argtypes = [C.c_int, C.c_uint64, P]
        _lib.orc_synthesize.restype = C.c_int
        _lib.orc_synthesize.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int64, C.c_double,
                                        C.c_double, C.c_double, C.c_uint64, C.c_int64,
                                        P, P, P, P, P, P]
    return _lib


class _Keep:
    """Holds converted arrays alive until the C call that uses them returns."""

    def __init__(self):
        self.refs = []

    def __call__(self, a):
        if a is None:
            return None
        self.refs.append(a)
        return C.c_void_p(a.ctypes.data)


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def make_config(side, n_patterns, n_rotations, likelihood=LL_GAUSS, interp=NEAREST,
                sigma=0.4, poisson_floor=1e-10):
    return Config(side, likelihood, interp, 0, n_patterns, n_rotations, sigma, poisson_floor)


def generate_rotations(n: int, halve: bool = True):
    """600-cell sampling, emc.c:49-363 (halved: one of each +-q pair)."""
    L = lib()
    R = L.orc_generate_rotations(n, int(halve), None, None)
    q = np.zeros((R, 4), np.float64)
    w = np.zeros(R, np.float64)
    got = L.orc_generate_rotations(n, int(halve), _p(q), _p(w))
    if got < 0:
        raise RuntimeError("600-cell construction failed")
    return q[:got], w[:got]


def coordinates(side, wavelength, pixel_size, detector_distance):
    """emc.c:365-393; arrays indexed [y*side + x]."""
    n = side * side
    x, y, z = (np.zeros(n, np.float64) for _ in range(3))
    lib().orc_coordinates(side, wavelength, pixel_size, detector_distance, _p(x), _p(y), _p(z))
    return x, y, z


def rotation_matrix_f32(q):
    q = np.ascontiguousarray(q, np.float32)
    m = np.zeros(9, np.float32)
    lib().orc_rotation_matrix_f32(_p(q), _p(m))
    return m.reshape(3, 3)


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def _f64(a):
    return np.ascontiguousarray(a, np.float64)


def _i32(a):
    return np.ascontiguousarray(a, np.int32)


def expand(cfg, model, rot, cx, cy, cz):
    """emc_cuda.cu:51-111 (nearest) / trilinear; returns S[R][side*side]."""
    k = _Keep()
    npix = cfg.side * cfg.side
    S = np.zeros((cfg.n_rotations, npix), np.float64)
    lib().orc_expand(C.byref(cfg), k(_f64(model)), k(_f32(rot)), k(_f32(cx)), k(_f32(cy)),
                     k(_f32(cz)), _p(S))
    return S


def loglik(cfg, S, images, mask, scaling, direct=False):
    """emc_cuda.cu:113-150 (gauss) or sum K log W - phi sum W (poisson); LL[R][N]."""
    k = _Keep()
    LL = np.zeros((cfg.n_rotations, cfg.n_patterns), np.float64)
    fn = lib().orc_loglik_gauss_direct if direct else lib().orc_loglik
    fn(C.byref(cfg), k(_f64(S)), k(_f32(images)), k(_i32(mask)), k(_f64(scaling)), _p(LL))
    return LL


def softmax(LL):
    """emc_cuda.cu:445-476 in FP64; returns (P, lse, sum P log P)."""
    P = np.array(LL, np.float64, copy=True, order="C")
    R, N = P.shape
    lse = np.zeros(N, np.float64)
    plogp = lib().orc_softmax(R, N, _p(P), _p(lse))
    return P, lse, plogp


def update_scaling(cfg, S, images, mask, P, scaling):
    """emc_cuda.cu:195-228 (gauss) or the poisson MLE; returns new scaling."""
    k = _Keep()
    sc = _f64(scaling).copy()
    lib().orc_update_scaling(C.byref(cfg), k(_f64(S)), k(_f32(images)), k(_i32(mask)),
                             k(_f64(P)), _p(sc))
    return sc


def compress(cfg, P, images, mask, scaling, rot, rotw, cx, cy, cz):
    """emc_atomic.cu:76-133; returns (model_acc, weight_acc, T)."""
    k = _Keep()
    M = cfg.side ** 3
    model = np.zeros(M, np.float64)
    weight = np.zeros(M, np.float64)
    T = np.zeros(cfg.n_rotations, np.float64)
    lib().orc_compress(C.byref(cfg), k(_f64(P)), k(_f32(images)), k(_i32(mask)),
                       k(_f64(scaling)), k(_f32(rot)), k(_f32(rotw)), k(_f32(cx)),
                       k(_f32(cy)), k(_f32(cz)), _p(model), _p(weight), _p(T))
    return model, weight, T


def slice_average(cfg, P, images, mask, scaling):
    """emc_atomic.cu:76-113 / emc.c:541-555 without the /T_r; returns (U, T)."""
    k = _Keep()
    npix = cfg.side * cfg.side
    U = np.zeros((cfg.n_rotations, npix), np.float64)
    T = np.zeros(cfg.n_rotations, np.float64)
    lib().orc_slice_average(C.byref(cfg), k(_f64(P)), k(_f32(images)), k(_i32(mask)),
                            k(_f64(scaling)), _p(U), _p(T))
    return U, T


def insert(cfg, U, T, mask, rot, rotw, cx, cy, cz, model_acc=None, weight_acc=None,
           all_T=None):
    """emc_atomic.cu:17-73,115-133; accumulates into (model_acc, weight_acc).
    all_T: for a shard of the patterns, T_r over every shard (the skip test)."""
    k = _Keep()
    M = cfg.side ** 3
    model_acc = np.zeros(M, np.float64) if model_acc is None else model_acc
    weight_acc = np.zeros(M, np.float64) if weight_acc is None else weight_acc
    if all_T is None:
        lib().orc_insert(C.byref(cfg), k(_f64(U)), k(_f64(T)), k(_i32(mask)), k(_f32(rot)),
                         k(_f32(rotw)), k(_f32(cx)), k(_f32(cy)), k(_f32(cz)), _p(model_acc),
                         _p(weight_acc))
    else:
        lib().orc_insert_shard(C.byref(cfg), k(_f64(U)), k(_f64(T)), k(_f64(all_T)),
                               k(_i32(mask)), k(_f32(rot)), k(_f32(rotw)), k(_f32(cx)),
                               k(_f32(cy)), k(_f32(cz)), _p(model_acc), _p(weight_acc))
    return model_acc, weight_acc


def normalize_model(model, weight):
    """emc_cuda.cu:414-433 in FP64."""
    k = _Keep()
    m = _f64(model).copy()
    lib().orc_normalize_model(m.size, _p(m), k(_f64(weight)))
    return m


def iterate(cfg, images, mask, rot, rotw, cx, cy, cz, model, scaling, want_resp=False,
            allowed=None):
    """One EMC iteration in the order of emc.c:989-1084.

    allowed: optional [R][N] mask restricting each pattern's softmax to a
    candidate set of rotations (orc_iterate_restricted).
    Returns (model, scaling, P or None, stats dict)."""
    k = _Keep()
    npix = cfg.side * cfg.side
    if (np.asarray(images).size != cfg.n_patterns * npix or np.asarray(mask).size != npix
            or np.asarray(rot).shape != (cfg.n_rotations, 4) or np.asarray(rotw).size != cfg.n_rotations
            or np.asarray(scaling).size != cfg.n_patterns or np.asarray(model).size != npix * cfg.side):
        raise ValueError("oracle.iterate: array shapes do not match the configuration")
    m = _f64(model).copy()
    sc = _f64(scaling).copy()
    P = np.zeros((cfg.n_rotations, cfg.n_patterns), np.float64) if want_resp else None
    st = Stats()
    if allowed is None:
        lib().orc_iterate(C.byref(cfg), k(_f32(images)), k(_i32(mask)), k(_f32(rot)),
                          k(_f32(rotw)), k(_f32(cx)), k(_f32(cy)), k(_f32(cz)), _p(m), _p(sc),
                          _p(P), C.byref(st))
    else:
        al = k(np.ascontiguousarray(allowed, np.uint8))
        assert allowed.shape == (cfg.n_rotations, cfg.n_patterns)
        lib().orc_iterate_restricted(C.byref(cfg), k(_f32(images)), k(_i32(mask)), k(_f32(rot)),
                                     k(_f32(rotw)), k(_f32(cx)), k(_f32(cy)), k(_f32(cz)), al,
                                     _p(m), _p(sc), _p(P), C.byref(st))
    stats = {k: getattr(st, k) for k, _ in Stats._fields_}
    return m, sc, P, stats


# ------------------------------------------------------- synthetic inputs --

def random_model(side, seed=0):
    """Uniform [0, 1) model from the seeded counter-based stream."""
    m = np.zeros(side ** 3, np.float32)
    lib().orc_random_model(side, seed, _p(m))
    return m


def synthesize(side, n_patterns, x, y, z, mean_photons=1000.0, scale_sigma=0.3,
               beamstop_radius=0.0, n_scatterers=40, object_radius=0.3, seed=0, first_pattern=0):
    """Seeded synthetic dataset: dict(model, counts [N][side^2], mask)."""
    npix = side * side
    model = np.zeros(side ** 3, np.float32)
    counts = np.zeros((n_patterns, npix), np.float32)
    mask = np.zeros(npix, np.int32)
    k = _Keep()
    rc = lib().orc_synthesize(side, n_scatterers, object_radius, n_patterns, mean_photons,
                              scale_sigma, beamstop_radius, seed, first_pattern, k(_f32(x)),
                              k(_f32(y)), k(_f32(z)), _p(model), _p(counts), _p(mask))
    if rc != 0:
        raise ValueError("orc_synthesize: invalid arguments")
    return dict(model=model, counts=counts, mask=mask)


def make_workload(w, n_patterns=None, first_pattern=0, wavelength=1e-10, distance=1.0,
                  pixel_size=None):
    """A benchmark workload (an object with side, rot_n, n_patterns,
    mean_photons, scale_sigma, beamstop, seed) built with this library alone:
    the same arrays as the engine's own workload builder, in the same dict."""
    N = n_patterns or w.n_patterns
    x, y, z = (a.astype(np.float32) for a in coordinates(w.side, wavelength, pixel_size, distance))
    d = synthesize(w.side, N, x, y, z, mean_photons=w.mean_photons, scale_sigma=w.scale_sigma,
                   beamstop_radius=w.beamstop, seed=w.seed, first_pattern=first_pattern)
    q, wt = generate_rotations(w.rot_n, halve=True)
    return dict(workload=w, x=x, y=y, z=z, mask=d["mask"], counts=d["counts"],
                q=q.astype(np.float32), w=wt.astype(np.float32),
                model0=random_model(w.side, w.seed), true_model=d["model"],
                scaling0=np.ones(N, np.float32))
