"""Parity at the plain-FP32 drop-in configuration: 64^3 model, 64x64 detector
with a radius-4 beamstop (4,044 active pixels), all 25,680 rotations of the
halved n=8 600-cell sampling, seeded Poisson patterns of 2,000 photons on
average (lognormal scale sigma 0.5), 20 iterations from a random-uniform
model.  The engine and the FP64 oracle each run their own chain of 20
iterations from the same start; every iteration's responsibilities and the
model after the last one are compared.

Bars (written here, not loosened):
  * FP32 paths (the reference's gaussian likelihood through the drop-in
    include/emc.h API, driven as emc.c:961-1066 drives it; the poisson
    likelihood through the context API): responsibilities within 1e-5
    (max over patterns of the per-pattern L1 distance, which is relative
    because each pattern's responsibilities sum to 1) in every iteration,
    model within 1e-5 relative after 20 iterations;
  * mixed path (FP16 counts, FP16 hi+lo slice operand, FP32 accumulation,
    FP64 log-sum-exp), same data: responsibilities within 1e-3, model within
    1e-4 after 20 iterations.

The pattern count is cut to what the oracle iterates in a few minutes on the
host (the rotations, the geometry and the photon statistics are the
configuration's own): each pattern's responsibilities depend only on the
model, its scaling and that pattern, and the model is a sum over patterns.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from parity import make_ctx, oracle_cfg, rel, resp_l1

pytestmark = pytest.mark.gpu

N_PATTERNS = 128
ITERATIONS = 20

real = C.c_float


class Quaternion(C.Structure):
    _fields_ = [("q", real * 4)]


class Setup(C.Structure):
    _fields_ = [("side", C.c_int), ("wavelength", real), ("pixel_size", real),
                ("detector_size", C.c_int), ("detector_distance", real)]


class SpMatrix(C.Structure):
    _fields_ = [("rows", C.c_uint), ("cols", C.c_uint), ("data", C.POINTER(real))]


class SpIMatrix(C.Structure):
    _fields_ = [("rows", C.c_uint), ("cols", C.c_uint), ("data", C.POINTER(C.c_int))]


class Sp3Matrix(C.Structure):
    _fields_ = [("x", C.c_uint), ("y", C.c_uint), ("z", C.c_uint), ("data", C.POINTER(real))]


def _fp(a):
    return a.ctypes.data_as(C.POINTER(real))


@pytest.fixture(scope="module")
def cfg2():
    from emc_b200 import workloads as W
    d = W.make("b200_64", n_patterns=N_PATTERNS)
    assert d["q"].shape[0] == 25_680 and int((d["mask"] != 0).sum()) == 4044
    return d


def _oracle_chain(d, lik):
    """Yields (P, model, stats) of each oracle iteration (P from the state the
    iteration starts from, model after it)."""
    cfg = oracle_cfg(d, lik, "nearest")
    m, s = d["model0"].astype(np.float64), d["scaling0"].astype(np.float64)
    for _ in range(ITERATIONS):
        m, s, P, st = O.iterate(cfg, d["counts"], d["mask"], d["q"], d["w"], d["x"], d["y"],
                                d["z"], m, s, want_resp=True)
        yield P, m, st


def test_dropin_gauss_20_iterations(cfg2):
    """The reference's own API (include/emc.h) in the order of its main loop."""
    import torch

    import emc_b200 as E
    from emc_b200 import workloads as W
    L = E.lib()
    d = cfg2
    side, N, R = 64, d["counts"].shape[0], d["q"].shape[0]
    npix = side * side
    PP = C.POINTER(real)
    model_h = d["model0"].copy()
    weight_h = np.zeros(side ** 3, np.float32)
    model = Sp3Matrix(side, side, side, _fp(model_h))
    weight = Sp3Matrix(side, side, side, _fp(weight_h))
    mask_h = np.ascontiguousarray(d["mask"], np.int32)
    mask = SpIMatrix(side, side, mask_h.ctypes.data_as(C.POINTER(C.c_int)))
    coords = [np.ascontiguousarray(a, np.float32) for a in (d["x"], d["y"], d["z"])]
    cm = [SpMatrix(side, side, _fp(a)) for a in coords]
    imgs = [np.ascontiguousarray(d["counts"][p]) for p in range(N)]
    img_m = [SpMatrix(side, side, _fp(a)) for a in imgs]
    img_pp = (C.POINTER(SpMatrix) * N)(*[C.pointer(m) for m in img_m])
    quats = [Quaternion((real * 4)(*q)) for q in d["q"]]
    quat_pp = (C.POINTER(Quaternion) * R)(*[C.pointer(q) for q in quats])
    setup = Setup(side, 1e-10, W.pixel_size(side), 512, 1.0)
    slices, d_model, d_weight, d_rot, d_images, d_respons, d_scaling, d_x, d_y, d_z = (
        PP() for _ in range(10))
    d_mask = C.POINTER(C.c_int)()
    L.cuda_allocate_slices(C.byref(slices), setup, R)
    L.cuda_allocate_model(C.byref(d_model), C.byref(model))
    L.cuda_allocate_model(C.byref(d_weight), C.byref(weight))
    L.cuda_allocate_mask(C.byref(d_mask), C.byref(mask))
    L.cuda_allocate_rotations(C.byref(d_rot), quat_pp, R)
    L.cuda_allocate_coords(C.byref(d_x), C.byref(d_y), C.byref(d_z), *[C.byref(m) for m in cm])
    L.cuda_allocate_images(C.byref(d_images), img_pp, N)
    L.cuda_allocate_real(C.byref(d_respons), R * N * 4)
    L.cuda_allocate_scaling(C.byref(d_scaling), N)
    assert L.emc_legacy_last_status() == 0
    L.cuda_total_respons.restype = real
    L.cuda_update_slices.restype = real
    respons = np.zeros(R * N, np.float32)
    scaling = np.ones(N, np.float32)
    rotw = np.ascontiguousarray(d["w"], np.float32)
    errs = []
    for P_ref, m_ref, _ in _oracle_chain(d, "gauss"):
        L.cuda_get_slices(C.byref(model), d_model, slices, d_rot, d_x, d_y, d_z, R)
        L.cuda_calculate_responsabilities(slices, d_images, d_mask, real(0.4), d_scaling,
                                          d_respons, npix, N, R, _fp(respons))
        L.cuda_normalize_responsabilities(d_respons, R, N)
        L.cuda_total_respons(d_respons, _fp(respons), R * N)
        # the responsibilities stay on the device (emc_cuda.cu:484-505 copies nothing)
        P = torch.as_tensor(E._CudaArray(C.cast(d_respons, C.c_void_p).value, R * N),
                            device="cuda").cpu().numpy().reshape(R, N)
        errs.append(resp_l1(P, P_ref))
        L.cuda_reset_model(C.byref(model), d_model)
        L.cuda_reset_model(C.byref(weight), d_weight)
        L.cuda_update_scaling(d_images, slices, d_mask, d_respons, d_scaling, N, R, npix,
                              _fp(scaling))
        L.cuda_update_slices(d_images, slices, d_mask, d_respons, d_scaling, N, R, npix,
                             C.byref(model), d_model, d_x, d_y, d_z, d_rot, _fp(rotw), d_weight,
                             setup, img_pp)
        L.cuda_normalize_model(C.byref(model), d_model, d_weight)
        assert L.emc_legacy_last_status() == 0
    # cuda_update_slices leaves the unnormalised model in model_h (as
    # emc_cuda.cu:352 does); the normalised one is read from the device buffer
    t = torch.as_tensor(E._CudaArray(C.cast(d_model, C.c_void_p).value, side ** 3),
                        device="cuda")
    final = t.cpu().numpy()
    err_m = rel(final, m_ref)
    print(f"drop-in gauss: responsibility L1 per iteration {np.array2string(np.array(errs), precision=2)}; "
          f"model after {ITERATIONS} iterations {err_m:.3g}")
    assert max(errs) <= 1e-5, f"responsibility L1 {max(errs):.3g} (iteration {int(np.argmax(errs))})"
    assert err_m <= 1e-5, f"model error after {ITERATIONS} iterations: {err_m:.3g}"


def test_poisson_fp32_and_mixed_20_iterations(cfg2):
    """The poisson likelihood on the FP32 and the mixed path, each against the
    oracle's chain, iteration by iteration; the total log-likelihood
    (sum_p log sum_r e^LL_rp) is compared too."""
    import emc_b200 as E
    d = cfg2
    errs = {"fp32": [], "mixed": []}
    ll_err = {"fp32": [], "mixed": []}
    with make_ctx(d, "poisson", "nearest", "fp32") as c32, \
            make_ctx(d, "poisson", "nearest", "mixed") as cmx:
        for P_ref, m_ref, st_ref in _oracle_chain(d, "poisson"):
            for name, ctx in (("fp32", c32), ("mixed", cmx)):
                ctx.expand()
                ctx.maximize()
                P = ctx.get_buffer(E.BUF_RESP)
                ctx.compress()
                _, loglik = ctx.partial_stats()
                errs[name].append(resp_l1(P, P_ref))
                ll_err[name].append(abs(loglik - st_ref["total_loglik"])
                                    / abs(st_ref["total_loglik"]))
        e32, emx = rel(c32.get_model(), m_ref), rel(cmx.get_model(), m_ref)
    for name, em in (("fp32", e32), ("mixed", emx)):
        print(f"poisson {name}: responsibility L1 per iteration "
              f"{np.array2string(np.array(errs[name]), precision=2)}; total log-likelihood "
              f"max rel. {max(ll_err[name]):.3g}; model after {ITERATIONS} iterations {em:.3g}")
    assert max(errs["fp32"]) <= 1e-5, f"fp32 responsibility L1 {max(errs['fp32']):.3g}"
    assert e32 <= 1e-5, f"fp32 model error after {ITERATIONS} iterations: {e32:.3g}"
    assert max(errs["mixed"]) <= 1e-3, f"mixed responsibility L1 {max(errs['mixed']):.3g}"
    assert emx <= 1e-4, f"mixed model error after {ITERATIONS} iterations: {emx:.3g}"
