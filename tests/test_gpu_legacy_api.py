"""The reference-compatible C API (include/emc.h) driven the way the
reference's main loop drives it (emc.c:961-1066), checked against the oracle.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from parity import oracle_cfg, rel

pytestmark = pytest.mark.gpu

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


def test_reference_api_iteration():
    import emc_b200 as E
    from emc_b200 import workloads as W

    L = E.lib()
    d = W.make("tiny16")
    w = d["workload"]
    side, N, R = w.side, d["counts"].shape[0], d["q"].shape[0]
    npix = side * side
    PP = C.POINTER(real)
    pp = lambda: PP()  # noqa: E731

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

    slices, d_model, d_weight, d_rot, d_images, d_respons, d_scaling = (pp() for _ in range(7))
    d_x, d_y, d_z = pp(), pp(), pp()
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

    L.cuda_model_max.restype = real
    L.cuda_total_respons.restype = real
    L.cuda_update_slices.restype = real
    cfg = oracle_cfg(d, "gauss", "nearest")
    respons = np.zeros(R * N, np.float32)
    scaling = np.ones(N, np.float32)
    m_ref = d["model0"].astype(np.float64)
    s_ref = np.ones(N)
    rotw = np.ascontiguousarray(d["w"], np.float32)
    sigma = 0.4
    for it in range(2):
        mx = L.cuda_model_max(d_model, side ** 3)
        assert abs(mx - m_ref.max()) <= 1e-5 * m_ref.max()
        L.cuda_get_slices(C.byref(model), d_model, slices, d_rot, d_x, d_y, d_z, R)
        L.cuda_calculate_responsabilities(slices, d_images, d_mask, real(sigma), d_scaling, d_respons,
                                          npix, N, R, _fp(respons))
        S_ref = O.expand(cfg, m_ref.astype(np.float32), d["q"], d["x"], d["y"], d["z"])
        LL_ref = O.loglik(cfg, S_ref, d["counts"], d["mask"], s_ref)
        np.testing.assert_allclose(respons.reshape(R, N), LL_ref, rtol=2e-5,
                                   atol=2e-5 * np.abs(LL_ref).max())
        L.cuda_normalize_responsabilities(d_respons, R, N)
        P_ref, _, plogp_ref = O.softmax(LL_ref)
        plogp = L.cuda_total_respons(d_respons, _fp(respons), R * N)
        assert abs(plogp - plogp_ref) <= 1e-3 * abs(plogp_ref) + 1e-3
        L.cuda_reset_model(C.byref(model), d_model)
        L.cuda_reset_model(C.byref(weight), d_weight)
        L.cuda_update_scaling(d_images, slices, d_mask, d_respons, d_scaling, N, R, npix,
                              _fp(scaling))
        s_new = O.update_scaling(cfg, S_ref, d["counts"], d["mask"], P_ref, s_ref)
        assert rel(scaling, s_new) < 1e-4
        tot = L.cuda_update_slices(d_images, slices, d_mask, d_respons, d_scaling, N, R, npix,
                                   C.byref(model), d_model, d_x, d_y, d_z, d_rot, _fp(rotw),
                                   d_weight, setup, img_pp)
        assert abs(tot - N) < 1e-3 * N
        acc, wacc, _ = O.compress(cfg, P_ref, d["counts"], d["mask"], scaling.astype(np.float64),
                                  d["q"], d["w"], d["x"], d["y"], d["z"])
        # emc_cuda.cu:352 hands back the model before normalisation
        assert rel(model_h, acc) < 1e-4
        L.cuda_normalize_model(C.byref(model), d_model, d_weight)
        m_ref = O.normalize_model(acc, wacc)
        s_ref = s_new
        assert L.emc_legacy_last_status() == 0
