"""emc_b200 -- B200 EMC engine (expand -> maximize -> compress).

Python host wrapper over libemc_b200.so (C ABI in include/emc_b200.h and the
reference-compatible include/emc.h).  The compute path is the CUDA library;
importing this module never falls back to a CPU implementation: if the
library is missing, ``lib()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libemc_b200.so")

GAUSS, POISSON = 0, 1
NEAREST, TRILINEAR = 0, 1
FP32, MIXED = 0, 1
_NAMES = {
    "gauss": GAUSS, "poisson": POISSON, "nearest": NEAREST, "trilinear": TRILINEAR,
    "fp32": FP32, "mixed": MIXED,
}
BUF_MODEL, BUF_WEIGHT, BUF_SCALING, BUF_RESP, BUF_SLICES, BUF_TOTALRESP, BUF_ACCUM = range(7)
BUF_TOTALRESP_ALL = 7
STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of device memory",
          4: "device wait timed out", 5: "call out of order", 6: "data out of exact range",
          7: "unsupported"}


class EmcError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Config(C.Structure):
    _fields_ = [("side", C.c_int32), ("likelihood", C.c_int32), ("interp", C.c_int32),
                ("precision", C.c_int32), ("n_patterns", C.c_int64), ("n_rotations", C.c_int64),
                ("sigma", C.c_float), ("poisson_floor", C.c_float), ("device", C.c_int32),
                ("flags", C.c_int32)]


class IterStats(C.Structure):
    _fields_ = [("sum_plogp", C.c_double), ("total_loglik", C.c_double),
                ("model_max", C.c_double), ("total_resp", C.c_double)]


class Tuning(C.Structure):
    _fields_ = [("maximize_raster", C.c_int32), ("compress_raster", C.c_int32),
                ("maximize_pair", C.c_int32), ("compress_pair", C.c_int32),
                ("maximize_sparse", C.c_int32), ("compress_sparse", C.c_int32)]


class SynthConfig(C.Structure):
    _fields_ = [("side", C.c_int32), ("n_scatterers", C.c_int32), ("object_radius", C.c_double),
                ("n_patterns", C.c_int64), ("mean_photons", C.c_double),
                ("scale_sigma", C.c_double), ("beamstop_radius", C.c_double),
                ("seed", C.c_uint64), ("first_pattern", C.c_int64)]


_lib = None


def lib():
    """The loaded CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.isfile(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m emc_b200.build`")
        L = C.CDLL(LIB_PATH)
        P, I64 = C.c_void_p, C.c_int64
        for name, args, res in [
            ("emc_create", [P, P], C.c_int), ("emc_destroy", [P], C.c_int),
            ("emc_set_geometry", [P, P, P, P, P], C.c_int), ("emc_set_rotations", [P, P, P], C.c_int),
            ("emc_set_patterns", [P, P], C.c_int), ("emc_set_model", [P, P], C.c_int),
            ("emc_set_scaling", [P, P], C.c_int), ("emc_iterate", [P, P], C.c_int),
            ("emc_expand", [P], C.c_int), ("emc_maximize", [P], C.c_int),
            ("emc_compress", [P], C.c_int), ("emc_synchronize", [P], C.c_int),
            ("emc_wait_probe", [P, C.c_uint32], C.c_int),
            ("emc_get_model", [P, P], C.c_int), ("emc_get_scaling", [P, P], C.c_int),
            ("emc_get_buffer", [P, C.c_int, P, C.c_size_t], C.c_int),
            ("emc_device_buffer", [P, C.c_int, P, P], C.c_int),
            ("emc_stream", [P], P), ("emc_active_pixels", [P], I64),
            ("emc_last_error", [P], C.c_char_p), ("emc_status_string", [C.c_int], C.c_char_p),
            ("emc_n_to_samples", [C.c_int], I64),
            ("emc_generate_rotations", [C.c_int, C.c_int, P, P], I64),
            ("emc_detector_coordinates", [C.c_int, C.c_double, C.c_double, C.c_double, P, P, P], None),
            ("emc_synthesize", [P, P, P, P, P, P, P, P, P], C.c_int),
            ("emc_random_model", [C.c_int, C.c_uint64, P], None),
            ("emc_legacy_last_status", [], C.c_int),
            ("emc_set_profiling", [P, C.c_int], C.c_int), ("emc_stage_times", [P, P], C.c_int),
            ("emc_launch_count", [P], I64),
            ("emc_compress_insert", [P], C.c_int), ("emc_normalize", [P], C.c_int),
            ("emc_partial_stats", [P, P, P], C.c_int),
            ("emc_get_tuning", [P, P], C.c_int), ("emc_set_tuning", [P, P], C.c_int),
            ("emc_orientation_stats", [P, P, P, P], C.c_int),
            ("emc_set_patterns_sparse", [P, P, P, P], C.c_int),
            ("emc_batch_create", [P, C.c_int32, P], C.c_int), ("emc_batch_destroy", [P], C.c_int),
            ("emc_batch_iterate", [P], C.c_int), ("emc_batch_capture", [P], C.c_int),
            ("emc_batch_launch", [P, C.c_int32], C.c_int),
            ("emc_batch_synchronize", [P], C.c_int), ("emc_batch_stream", [P], P),
            ("emc_batch_last_error", [P], C.c_char_p),
            ("emc_model_random_orientations", [C.c_int, I64, P, P, P, P, P, C.c_uint64, P, P],
             C.c_int),
            ("emc_model_load", [C.c_char_p, C.c_int, P], C.c_int),
            ("emc_model_save", [C.c_char_p, C.c_int, P], C.c_int),
            ("emc_autotune", [P, P, C.c_int32, P, P], C.c_int),
            ("emc_set_memory_limit", [P, C.c_size_t], C.c_int),
            ("emc_get_resp_columns", [P, I64, P, P], C.c_int),
            ("emc_memory_used", [P], C.c_size_t),
            ("emc_set_rotation_chunk", [P, C.c_int64, C.c_int64], C.c_int),
            ("emc_rotation_chunk", [P], C.c_int64),
            ("emc_set_deterministic", [P, C.c_int], C.c_int),
            ("emc_save_state", [P, C.c_char_p, I64], C.c_int),
            ("emc_load_state", [P, C.c_char_p, P], C.c_int),
        ]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


def _check(status, ctx=None):
    if status != 0:
        msg = lib().emc_last_error(ctx)
        raise EmcError(status, msg.decode() if msg else "")


# ------------------------------------------------------------ generators --

def generate_rotations(n: int, halve: bool = True):
    """600-cell rotation sampling (emc.c:49-363); halved to one of each +-q."""
    L = lib()
    R = L.emc_generate_rotations(n, int(halve), None, None)
    q = np.zeros((R, 4), np.float32)
    w = np.zeros(R, np.float32)
    got = L.emc_generate_rotations(n, int(halve), _ptr(q), _ptr(w))
    if got < 0:
        raise RuntimeError("rotation sampling failed")
    return q[:got], w[:got]


def detector_coordinates(side, wavelength, pixel_size, detector_distance):
    """Pixel coordinates with Ewald curvature (emc.c:365-393), [y*side+x]."""
    x, y, z = (np.zeros(side * side, np.float32) for _ in range(3))
    lib().emc_detector_coordinates(side, wavelength, pixel_size, detector_distance, _ptr(x), _ptr(y),
                                   _ptr(z))
    return x, y, z


def model_random_orientations(side, images, mask, x, y, z, seed=0, return_rotations=False):
    """emc_model_random_orientations: every image inserted with weight 1 at a
    uniformly random rotation, model = sum / weight (emc.c:896-914)."""
    imgs = np.ascontiguousarray(images, np.float32).reshape(-1, side * side)
    model = np.zeros(side ** 3, np.float32)
    quat = np.zeros((imgs.shape[0], 4), np.float32)
    _check(lib().emc_model_random_orientations(
        side, imgs.shape[0], _ptr(imgs), _ptr(np.ascontiguousarray(mask, np.int32)),
        _ptr(np.ascontiguousarray(x, np.float32)), _ptr(np.ascontiguousarray(y, np.float32)),
        _ptr(np.ascontiguousarray(z, np.float32)), seed, _ptr(model), _ptr(quat)))
    return (model, quat) if return_rotations else model


def photon_lists(counts):
    """Dense patterns [N][side^2] -> CSR photon lists (row_ptr, pixels, counts)
    of their non-zero pixels."""
    K = np.asarray(counts).reshape(np.asarray(counts).shape[0], -1)
    p, j = np.nonzero(K)
    row_ptr = np.zeros(K.shape[0] + 1, np.int64)
    np.cumsum(np.bincount(p, minlength=K.shape[0]), out=row_ptr[1:])
    return row_ptr, j.astype(np.int32), K[p, j].astype(np.float32)


def load_model(path, side):
    """emc_model_load: raw float32 side^3 file, |value| (emc.c:915-925)."""
    model = np.zeros(side ** 3, np.float32)
    _check(lib().emc_model_load(os.fsencode(path), side, _ptr(model)))
    return model


def save_model(path, model, side):
    m = np.ascontiguousarray(model, np.float32).reshape(-1)
    assert m.size == side ** 3
    _check(lib().emc_model_save(os.fsencode(path), side, _ptr(m)))


def random_model(side, seed=0):
    m = np.zeros(side ** 3, np.float32)
    lib().emc_random_model(side, seed, _ptr(m))
    return m


def synthesize(side, n_patterns, x, y, z, mean_photons=1000.0, scale_sigma=0.3,
               beamstop_radius=0.0, n_scatterers=40, object_radius=0.3, seed=0, first_pattern=0):
    """Seeded synthetic dataset: returns dict(model, counts, mask, rotations, scales).

    Patterns first_pattern .. first_pattern + n_patterns - 1 of the seeded
    sequence, so shards of one dataset can be generated independently."""
    sc = SynthConfig(side, n_scatterers, object_radius, n_patterns, mean_photons, scale_sigma,
                     beamstop_radius, seed, first_pattern)
    npix = side * side
    model = np.zeros(side ** 3, np.float32)
    counts = np.zeros((n_patterns, npix), np.float32)
    mask = np.zeros(npix, np.int32)
    rot = np.zeros((n_patterns, 4), np.float32)
    scales = np.zeros(n_patterns, np.float32)
    x, y, z = (np.ascontiguousarray(a, np.float32) for a in (x, y, z))
    _check(lib().emc_synthesize(C.byref(sc), _ptr(x), _ptr(y), _ptr(z), _ptr(model), _ptr(counts),
                                _ptr(mask), _ptr(rot), _ptr(scales)))
    return dict(model=model, counts=counts, mask=mask, rotations=rot, scales=scales)


class _CudaArray:
    """__cuda_array_interface__ of a float32 device buffer owned by the library."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False),
                                         "version": 2, "strides": None}


# --------------------------------------------------------------- context --

class Context:
    """One EMC dataset resident on a GPU (include/emc_b200.h)."""

    def __init__(self, side, n_patterns, n_rotations, likelihood="gauss", interp="nearest",
                 precision="fp32", sigma=0.4, poisson_floor=1e-10, device=0):
        cfg = Config(side, _NAMES[likelihood], _NAMES[interp], _NAMES[precision], n_patterns,
                     n_rotations, sigma, poisson_floor, device, 0)
        h = C.c_void_p()
        st = lib().emc_create(C.byref(cfg), C.byref(h))
        _check(st, None)
        self._h = h
        self.side, self.N, self.R = side, n_patterns, n_rotations
        self.M = side ** 3
        self.config = cfg

    def close(self):
        if getattr(self, "_h", None):
            lib().emc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _c(self, st):
        _check(st, self._h)

    @staticmethod
    def _f32(a):
        return np.ascontiguousarray(a, np.float32)

    def set_geometry(self, x, y, z, mask):
        x, y, z = (self._f32(a) for a in (x, y, z))
        m = np.ascontiguousarray(mask, np.int32)
        self._c(lib().emc_set_geometry(self._h, _ptr(x), _ptr(y), _ptr(z), _ptr(m)))

    def set_rotations(self, q, w):
        q, w = self._f32(q), self._f32(w)
        assert q.shape == (self.R, 4) and w.shape == (self.R,)
        self._c(lib().emc_set_rotations(self._h, _ptr(q), _ptr(w)))

    def set_patterns(self, counts):
        k = self._f32(counts)
        assert k.size == self.N * self.side * self.side
        self._c(lib().emc_set_patterns(self._h, _ptr(k)))

    def set_patterns_sparse(self, row_ptr, pixels, counts=None):
        """emc_set_patterns_sparse: photon lists in CSR form (see photon_lists)."""
        rp = np.ascontiguousarray(row_ptr, np.int64)
        assert rp.size == self.N + 1
        px = np.ascontiguousarray(pixels, np.int32)
        ct = None if counts is None else np.ascontiguousarray(counts, np.float32)
        self._c(lib().emc_set_patterns_sparse(self._h, _ptr(rp), _ptr(px),
                                              None if ct is None else _ptr(ct)))

    def set_model(self, model):
        m = self._f32(model)
        assert m.size == self.M
        self._c(lib().emc_set_model(self._h, _ptr(m)))

    def set_scaling(self, s):
        s = self._f32(s)
        assert s.size == self.N
        self._c(lib().emc_set_scaling(self._h, _ptr(s)))

    def iterate(self, stats=True):
        if not stats:
            self._c(lib().emc_iterate(self._h, None))
            return None
        st = IterStats()
        self._c(lib().emc_iterate(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in IterStats._fields_}

    def expand(self):
        self._c(lib().emc_expand(self._h))

    def maximize(self):
        self._c(lib().emc_maximize(self._h))

    def compress(self):
        self._c(lib().emc_compress(self._h))

    def compress_insert(self):
        self._c(lib().emc_compress_insert(self._h))

    def normalize(self):
        self._c(lib().emc_normalize(self._h))

    def partial_stats(self):
        a, b = C.c_double(), C.c_double()
        self._c(lib().emc_partial_stats(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def total_resp_all_tensor(self):
        """Zero-copy torch view (CUDA, float32 [R]) of T_r as the insertion's
        T_r <= 1e-10 skip test reads it, valid between maximize() and
        compress_insert(): a pattern-sharded caller sums it over the shards."""
        import torch
        ptr, nbytes = self.device_buffer(BUF_TOTALRESP_ALL)
        return torch.as_tensor(_CudaArray(ptr, nbytes // 4), device="cuda")

    def accumulator_tensor(self):
        """Zero-copy torch view (CUDA, float32 [2*side^3]) of the insertion
        accumulators, valid between compress_insert() and normalize()."""
        import torch
        ptr, nbytes = self.device_buffer(BUF_ACCUM)
        return torch.as_tensor(_CudaArray(ptr, nbytes // 4), device="cuda")

    def synchronize(self):
        self._c(lib().emc_synchronize(self._h))

    def wait_probe(self, limit_us=2000):
        """emc_wait_probe: one device wait that cannot succeed, given up after
        limit_us; raises EmcError with status EMC_ERR_TIMEOUT, after which the
        context is usable again."""
        self._c(lib().emc_wait_probe(self._h, int(limit_us)))

    @property
    def active_pixels(self):
        return int(lib().emc_active_pixels(self._h))

    @property
    def stream(self):
        return lib().emc_stream(self._h)

    def get_model(self):
        m = np.zeros(self.M, np.float32)
        self._c(lib().emc_get_model(self._h, _ptr(m)))
        return m

    def get_scaling(self):
        s = np.zeros(self.N, np.float32)
        self._c(lib().emc_get_scaling(self._h, _ptr(s)))
        return s

    def get_buffer(self, which):
        shapes = {BUF_MODEL: (self.M,), BUF_WEIGHT: (self.M,), BUF_SCALING: (self.N,),
                  BUF_RESP: (self.R, self.N), BUF_SLICES: (self.R, self.active_pixels),
                  BUF_TOTALRESP: (self.R,)}
        out = np.zeros(shapes[which], np.float32)
        self._c(lib().emc_get_buffer(self._h, which, _ptr(out), out.nbytes))
        return out

    def set_profiling(self, on=True):
        self._c(lib().emc_set_profiling(self._h, int(on)))

    def stage_times(self):
        """ms of [expand, maximize contraction, responsibility pass, compress, normalise]."""
        ms = np.zeros(5, np.float32)
        self._c(lib().emc_stage_times(self._h, _ptr(ms)))
        return ms

    @property
    def launch_count(self):
        return int(lib().emc_launch_count(self._h))

    def orientation_stats(self):
        """emc_orientation_stats: dict(best_rot [N], best_resp [N], avg_resp [R])."""
        best = np.zeros(self.N, np.int32)
        bp = np.zeros(self.N, np.float32)
        avg = np.zeros(self.R, np.float32)
        self._c(lib().emc_orientation_stats(self._h, _ptr(best), _ptr(bp), _ptr(avg)))
        return {"best_rot": best, "best_resp": bp, "avg_resp": avg}

    def get_tuning(self):
        """(maximize_raster, compress_raster, maximize_pair, compress_pair) of the
        tensor-core kernels."""
        t = Tuning()
        self._c(lib().emc_get_tuning(self._h, C.byref(t)))
        return t.maximize_raster, t.compress_raster, t.maximize_pair, t.compress_pair

    def set_tuning(self, maximize_raster, compress_raster, maximize_pair=None, compress_pair=None,
                   maximize_sparse=None):
        t = Tuning()
        self._c(lib().emc_get_tuning(self._h, C.byref(t)))
        t.maximize_raster, t.compress_raster = int(maximize_raster), int(compress_raster)
        if maximize_pair is not None:
            t.maximize_pair = int(maximize_pair)
        if compress_pair is not None:
            t.compress_pair = int(compress_pair)
        if maximize_sparse is not None:
            t.maximize_sparse = int(maximize_sparse)
        self._c(lib().emc_set_tuning(self._h, C.byref(t)))

    def set_sparse_maximize(self, on: bool):
        """FP32 poisson contexts: evaluate the log-likelihood as a gather over
        each pattern's photon list (its non-zero pixels) instead of the dense
        rotation x pixel contraction."""
        t = Tuning()
        self._c(lib().emc_get_tuning(self._h, C.byref(t)))
        t.maximize_sparse = int(bool(on))
        self._c(lib().emc_set_tuning(self._h, C.byref(t)))

    def set_sparse_compress(self, on: bool):
        """FP32 contexts: form the slice sums as a gather over each active
        pixel's non-zero counts instead of the dense rotation x pattern
        contraction."""
        t = Tuning()
        self._c(lib().emc_get_tuning(self._h, C.byref(t)))
        t.compress_sparse = int(bool(on))
        self._c(lib().emc_set_tuning(self._h, C.byref(t)))

    def tuning(self):
        """Every field of emc_tuning as a dict."""
        t = Tuning()
        self._c(lib().emc_get_tuning(self._h, C.byref(t)))
        return {k: getattr(t, k) for k, _ in Tuning._fields_}

    def autotune(self, candidates=(1, 2, 4, 8, 16)):
        """emc_autotune: returns (best (maximize, compress) band sizes, ms[2][n]);
        for FP32 contexts the choice is the dense or photon-list form of each
        contraction (see tuning())."""
        cand = np.ascontiguousarray(candidates, np.int32)
        ms = np.zeros((2, len(cand)), np.float32)
        t = Tuning()
        self._c(lib().emc_autotune(self._h, _ptr(cand), len(cand), _ptr(ms), C.byref(t)))
        return (t.maximize_raster, t.compress_raster), ms

    def resp_columns(self, patterns):
        """emc_get_resp_columns: responsibilities [R][n] of the given patterns
        in the last maximize (dense or proposed)."""
        pat = np.ascontiguousarray(patterns, np.int64)
        out = np.zeros((self.R, pat.size), np.float32)
        self._c(lib().emc_get_resp_columns(self._h, pat.size, _ptr(pat), _ptr(out)))
        return out

    def set_memory_limit(self, nbytes):
        """emc_set_memory_limit: cap on the device memory this context allocates."""
        self._c(lib().emc_set_memory_limit(self._h, int(nbytes)))

    @property
    def memory_used(self):
        return int(lib().emc_memory_used(self._h))

    def set_rotation_chunk(self, rows, capacity=0):
        """emc_set_rotation_chunk: the log-likelihood held for `rows`
        rotations at a time (a multiple of 256; 0 = all, -1 = what fits the
        memory limit); capacity = initial kept-entry capacity (0: default)."""
        self._c(lib().emc_set_rotation_chunk(self._h, int(rows), int(capacity)))

    def set_deterministic(self, on=True):
        """emc_set_deterministic: order-independent (bitwise reproducible)
        insertion sums and responsibility lists."""
        self._c(lib().emc_set_deterministic(self._h, int(bool(on))))

    @property
    def rotation_chunk(self):
        """Rotations the log-likelihood buffer holds (R when unchunked)."""
        return int(lib().emc_rotation_chunk(self._h))

    def save_state(self, path, iteration=0):
        """emc_save_state: model, weight grid, scaling and the iteration number."""
        self._c(lib().emc_save_state(self._h, os.fsencode(path), int(iteration)))

    def load_state(self, path):
        """emc_load_state; returns the saved iteration number."""
        it = C.c_int64()
        self._c(lib().emc_load_state(self._h, os.fsencode(path), C.byref(it)))
        return it.value

    def device_buffer(self, which):
        p, n = C.c_void_p(), C.c_size_t()
        self._c(lib().emc_device_buffer(self._h, which, C.byref(p), C.byref(n)))
        return p.value, n.value


class Batch:
    """emc_batch: several mixed-precision contexts iterated with one
    persistent launch per contraction, optionally replayed as a CUDA graph."""

    def __init__(self, contexts):
        self.contexts = list(contexts)
        arr = (C.c_void_p * len(self.contexts))(*[c._h for c in self.contexts])
        h = C.c_void_p()
        st = lib().emc_batch_create(arr, len(self.contexts), C.byref(h))
        if st != 0:
            raise EmcError(st, "emc_batch_create")
        self._h = h

    def _c(self, st):
        if st != 0:
            raise EmcError(st, lib().emc_batch_last_error(self._h).decode())

    def iterate(self):
        self._c(lib().emc_batch_iterate(self._h))

    def capture(self):
        self._c(lib().emc_batch_capture(self._h))

    def launch(self, iterations=1):
        self._c(lib().emc_batch_launch(self._h, iterations))

    def synchronize(self):
        self._c(lib().emc_batch_synchronize(self._h))

    @property
    def stream(self):
        return lib().emc_batch_stream(self._h)

    def close(self):
        if getattr(self, "_h", None):
            lib().emc_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
