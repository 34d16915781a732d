"""CPU checks of the product library: it loads, exports every symbol its
headers declare, its host-side generators agree with the oracle, and its
error paths return status codes (no GPU is needed for any of this)."""
import os
import re

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(REPO, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", text)
    return sorted({n for n in names if n not in ("sizeof", "if", "return")})


@pytest.fixture(scope="module")
def L():
    import emc_b200 as E
    from emc_b200 import build as B
    B.build()
    return E.lib()


@pytest.mark.parametrize("header", ["emc.h", "emc_b200.h"])
def test_exports_every_declared_function(L, header):
    names = _declared(header)
    assert len(names) > 10
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_reference_entry_points_present(L):
    # the prototypes of the reference header emc.h:20-56
    for n in ["insert_slice", "cuda_update_slices", "cuda_update_scaling",
              "cuda_calculate_responsabilities", "cuda_get_slices", "cuda_allocate_slices",
              "cuda_model_max", "cuda_allocate_model", "cuda_allocate_mask", "cuda_reset_model",
              "cuda_normalize_model", "cuda_allocate_rotations", "cuda_allocate_images",
              "cuda_allocate_coords", "cuda_allocate_real", "cuda_allocate_scaling",
              "cuda_normalize_responsabilities", "cuda_total_respons"]:
        assert hasattr(L, n), n


def test_generators_match_oracle(L, orc):
    import emc_b200 as E
    for n in (2, 4):
        q, w = E.generate_rotations(n)
        qo, wo = orc.generate_rotations(n)
        np.testing.assert_allclose(q, qo, atol=1e-7)
        np.testing.assert_allclose(w, wo, rtol=1e-6)
    for side in (16, 33):
        x, y, z = E.detector_coordinates(side, 1e-10, 0.03, 1.0)
        xo, yo, zo = orc.coordinates(side, 1e-10, 0.03, 1.0)
        for a, b in ((x, xo), (y, yo), (z, zo)):
            np.testing.assert_allclose(a, b, atol=1e-5)


def test_synthetic_workloads(L):
    from emc_b200 import workloads as W
    a = W.make("tiny16")
    b = W.make("tiny16")
    for k in ("counts", "mask", "true_model", "model0", "true_rotations"):
        np.testing.assert_array_equal(a[k], b[k])  # seeded and thread-count independent
    c = W.make("b200_64", n_patterns=64)
    assert int((c["mask"] != 0).sum()) == 4044  # 64^2 with a radius-4 beamstop
    assert c["q"].shape == (25680, 4)
    assert np.all(c["counts"] >= 0) and np.all(c["counts"] == np.floor(c["counts"]))
    assert abs(c["counts"].sum(1).mean() / 2000.0 - 1) < 0.2


def test_insert_slice_host_matches_reference_fixture(L, golden):
    import ctypes as C
    # include/emc.h insert_slice is the reference CPU routine emc.c:491-539
    from test_gpu_legacy_api import Quaternion, Sp3Matrix, SpIMatrix, SpMatrix
    side = 16
    cx, cy, cz = (np.ascontiguousarray(a, np.float32) for a in golden["coord_curved"])
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    model = np.zeros(side ** 3, np.float32)
    weight = np.zeros(side ** 3, np.float32)
    m3, w3 = Sp3Matrix(side, side, side, fp(model)), Sp3Matrix(side, side, side, fp(weight))
    mask = np.ascontiguousarray(golden["insert_mask"], np.int32)
    mk = SpIMatrix(side, side, mask.ctypes.data_as(C.POINTER(C.c_int)))
    xm, ym, zm = (SpMatrix(side, side, fp(a)) for a in (cx, cy, cz))
    for r, vals, w in zip(golden["slice_rot"], golden["insert_vals"], golden["insert_w"]):
        v = np.ascontiguousarray(vals, np.float32)
        s = SpMatrix(side, side, fp(v))
        q = Quaternion((C.c_float * 4)(*r))
        L.insert_slice(C.byref(m3), C.byref(w3), C.byref(s), C.byref(mk), C.c_float(w),
                       C.byref(q), C.byref(xm), C.byref(ym), C.byref(zm))
    np.testing.assert_allclose(model, golden["insert_model"], rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(weight, golden["insert_weight"], rtol=1e-6, atol=1e-6)


def test_create_reports_errors_without_crashing(L):
    import emc_b200 as E
    with pytest.raises(E.EmcError) as ei:
        E.Context(1, 10, 10)  # side < 2
    assert ei.value.status == 1
    with pytest.raises(E.EmcError) as ei:
        E.Context(16, 10, 10, likelihood="poisson", poisson_floor=0.0)
    assert ei.value.status == 1
