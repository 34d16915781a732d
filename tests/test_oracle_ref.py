"""The FP64 oracle against outputs of the reference's own CPU functions.

tests/golden/ref_cpu.npz was written by tests/golden/make_golden.py, which
runs the reference's emc.c compiled from source (oracle/_ref).  These checks
pin the oracle: rotations, coordinates, slicing, insertion, likelihood,
scaling and slice averaging.
"""
import numpy as np


def test_rotation_counts(orc):
    # emc.c:43 n_to_samples and the counts emc.c:128,168,210,220 print
    for n, full in ((2, 840), (4, 6480), (8, 51360), (12, 173040)):
        assert orc.lib().orc_n_to_samples(n) == full
    for n, half in ((2, 420), (4, 3240), (8, 25680)):
        q, w = orc.generate_rotations(n, halve=True)
        assert q.shape == (half, 4)
        np.testing.assert_allclose(np.linalg.norm(q, axis=1), 1.0, atol=1e-12)
        assert abs(w.sum() - 1.0) < 1e-12


def test_rotations_match_reference(orc, golden):
    for n in (2, 4):
        q, w = orc.generate_rotations(n, halve=False)
        np.testing.assert_allclose(q, golden[f"rot{n}_q"], atol=2e-7)
        # reference accumulates the weight sum in float
        np.testing.assert_allclose(w, golden[f"rot{n}_w"], rtol=1e-4)


def test_halving_keeps_one_of_each_pair(orc):
    qf, wf = orc.generate_rotations(4, halve=False)
    qh, wh = orc.generate_rotations(4, halve=True)
    # every full-list quaternion is +-(a kept one), and weights are doubled
    d = np.abs(qf @ qh.T)
    assert np.all(d.max(axis=1) > 1 - 1e-12)
    np.testing.assert_allclose(np.sort(wh), np.sort(wf[np.isin(np.arange(len(qf)), np.where(
        [(q[np.nonzero(q)[0][0]] > 0) for q in qf])[0])]) * 2, rtol=1e-12)


def test_coordinates_match_reference(orc, golden):
    for name in ("refsetup", "curved"):
        side, wl, px, d = golden[f"coord_{name}_setup"]
        got = orc.coordinates(int(side), wl, px, d)
        ref = golden[f"coord_{name}"]
        for k in range(3):
            np.testing.assert_allclose(got[k], ref[k], atol=1e-6 * max(1.0, np.abs(ref[k]).max()))


def test_pixel_voxel_round_trip(golden):
    # emc.c:396-441: rint(coords) -> get_pixel_from_voxel lands within half a
    # pixel of the starting pixel (rint of the .5 pixel centres rounds to even,
    # so the reference's own never-called check is not an exact identity).  It
    # returns the -1 marker where the rounded voxel sits on the beam axis
    # (pixel_r == 0 gives 0/0 in emc.c:409).
    side = int(golden["coord_refsetup_setup"][0])
    pix = golden["pixel_from_voxel"].astype(np.float64)
    xs, ys = np.meshgrid(np.arange(side), np.arange(side), indexing="xy")
    ok = pix[:, 0] != -1
    assert ok.mean() > 0.95
    assert np.all(np.abs(pix[ok, 0] - xs.reshape(-1)[ok]) <= 0.5)
    assert np.all(np.abs(pix[ok, 1] - ys.reshape(-1)[ok]) <= 0.5)


def test_identity_rotation_reproduces_coordinates(orc):
    m = orc.rotation_matrix_f32([1, 0, 0, 0])
    np.testing.assert_array_equal(m, np.eye(3, dtype=np.float32))
    q, _ = orc.generate_rotations(4)
    for qq in q[::97]:
        m = orc.rotation_matrix_f32(qq).astype(np.float64)
        np.testing.assert_allclose(m @ m.T, np.eye(3), atol=1e-6)


def test_expand_matches_reference_get_slice(orc, golden):
    side = 16
    cx, cy, cz = golden["coord_curved"]
    rot = golden["slice_rot"]
    cfg = orc.make_config(side, 1, len(rot))
    S = orc.expand(cfg, golden["slice_model"], rot, cx, cy, cz)
    np.testing.assert_array_equal(S.astype(np.float32), golden["slice_out"])


def test_insert_matches_reference_insert_slice(orc, golden):
    side = 16
    cx, cy, cz = golden["coord_curved"]
    rot = golden["slice_rot"]
    R = len(rot)
    cfg = orc.make_config(side, R, R)
    U = golden["insert_vals"].astype(np.float64)
    T = np.ones(R)  # insert_slice(w) == insert with rotw = w, T = 1
    model, weight = orc.insert(cfg, U, T, golden["insert_mask"], rot, golden["insert_w"], cx, cy, cz)
    np.testing.assert_allclose(model, golden["insert_model"], rtol=2e-6, atol=1e-6)
    np.testing.assert_allclose(weight, golden["insert_weight"], rtol=2e-6, atol=1e-6)


def test_loglik_matches_reference(orc, golden):
    sl, im = golden["ll_slices"], golden["ll_images"]
    side = 16
    cfg = orc.make_config(side, im.shape[0], sl.shape[0], sigma=float(golden["ll_sigma"]))
    mask = golden["insert_mask"]
    for direct in (False, True):
        LL = orc.loglik(cfg, sl, im, mask, golden["ll_scaling"], direct=direct)
        np.testing.assert_allclose(LL, golden["ll_out"], rtol=2e-5)


def test_scaling_matches_reference_slice_weighting(orc, golden):
    sl, im = golden["ll_slices"], golden["ll_images"]
    mask = golden["insert_mask"]
    cfg = orc.make_config(16, im.shape[0], sl.shape[0])
    phi = orc.update_scaling(cfg, sl, im, mask, golden["ll_resp"], np.ones(im.shape[0]))
    power = ((im.astype(np.float64) ** 2) * (mask != 0)).sum(1)  # emc_cuda.cu:207-212
    np.testing.assert_allclose(phi, power / golden["sw_out"], rtol=2e-5)


def test_slice_average_matches_reference_update_slice(orc, golden):
    sl, im = golden["ll_slices"], golden["ll_images"]
    mask = golden["insert_mask"]
    cfg = orc.make_config(16, im.shape[0], sl.shape[0])
    U, T = orc.slice_average(cfg, golden["ll_resp"], im, mask, golden["ll_scaling"])
    np.testing.assert_allclose(U, golden["us_slices"], rtol=2e-5, atol=1e-6)
    np.testing.assert_allclose(T, golden["us_total"], rtol=1e-6)


def test_softmax_and_normalize_properties(orc):
    rng = np.random.default_rng(0)
    LL = rng.normal(0, 30, (50, 7))
    P, lse, plogp = orc.softmax(LL)
    np.testing.assert_allclose(P.sum(0), 1.0, atol=1e-12)
    np.testing.assert_allclose(lse, np.log(np.exp(LL - LL.max(0)).sum(0)) + LL.max(0), rtol=1e-12)
    assert abs(plogp - (P[P > 0] * np.log(P[P > 0])).sum()) < 1e-9
    model = rng.uniform(0, 2, 1000)
    weight = rng.uniform(0, 1, 1000)
    weight[::7] = 0
    m = orc.normalize_model(model, weight)
    assert np.all(m[::7] == 0)
    assert abs(m.mean() - 1.0) < 1e-12


def test_constant_model_round_trip(orc):
    # insert(expand(const)) / weight gives the constant back on every touched voxel
    side = 16
    x, y, z = orc.coordinates(side, 1e-10, 0.02, 1.0)
    q, w = orc.generate_rotations(2)
    R = len(q)
    cfg = orc.make_config(side, 1, R)
    model = np.full(side ** 3, 3.0)
    S = orc.expand(cfg, model, q, x, y, z)
    mask = np.ones(side * side, np.int32)
    acc, wacc = orc.insert(cfg, S, np.ones(R), mask, q, w, x, y, z)
    inner = (S > 0).all(0)
    assert inner.sum() > side * side // 2
    got = acc[wacc > 0] / wacc[wacc > 0]
    # voxels reached by the inclusive bound but not by expand's exclusive one see 0
    assert np.all((np.abs(got - 3.0) < 1e-12) | (got <= 3.0))
    assert np.mean(np.abs(got - 3.0) < 1e-12) > 0.9
