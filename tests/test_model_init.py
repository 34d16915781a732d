"""Model initialisation modes of the reference (emc.c:889-925) and the raw
model file format, on the CPU."""
import numpy as np
import pytest

from oracle import oracle as O


def test_random_orientations_model_matches_oracle_insertion():
    import emc_b200 as E
    from emc_b200 import workloads as W
    d = W.make("tiny16")
    side = d["workload"].side
    model, quat = E.model_random_orientations(side, d["counts"], d["mask"], d["x"], d["y"], d["z"],
                                              seed=7, return_rotations=True)
    n = d["counts"].shape[0]
    np.testing.assert_allclose(np.linalg.norm(quat, axis=1), 1.0, atol=1e-6)
    cfg = O.make_config(side, n, n)
    acc, wt = O.insert(cfg, d["counts"].astype(np.float64), np.ones(n), d["mask"], quat,
                       np.ones(n, np.float32), d["x"], d["y"], d["z"])
    ref = np.where(wt > 0, acc / np.where(wt > 0, wt, 1), 0.0)
    np.testing.assert_allclose(model, ref, rtol=1e-6, atol=1e-6)
    again = E.model_random_orientations(side, d["counts"], d["mask"], d["x"], d["y"], d["z"], seed=7)
    np.testing.assert_array_equal(model, again)
    other = E.model_random_orientations(side, d["counts"], d["mask"], d["x"], d["y"], d["z"], seed=8)
    assert not np.array_equal(model, other)


def test_random_rotations_are_uniform():
    """Shoemake's construction: the rotated z axis is uniform on the sphere."""
    import emc_b200 as E
    side = 8
    n = 20000
    imgs = np.zeros((n, side * side), np.float32)
    mask = np.zeros(side * side, np.int32)
    xyz = [np.zeros(side * side, np.float32)] * 3
    _, q = E.model_random_orientations(side, imgs, mask, *xyz, seed=1, return_rotations=True)
    a, b, c, dd = q.T.astype(np.float64)
    zz = a * a - b * b - c * c + dd * dd  # z component of R e_z for q = (a, b, c, d), a real
    assert abs(zz.mean()) < 0.02 and abs((zz ** 2).mean() - 1 / 3) < 0.02


def test_model_file_round_trip(tmp_path):
    import emc_b200 as E
    side = 12
    m = np.random.default_rng(0).standard_normal(side ** 3).astype(np.float32)
    p = tmp_path / "model.raw"
    E.save_model(str(p), m, side)
    np.testing.assert_array_equal(E.load_model(str(p), side), np.abs(m))
    with pytest.raises(E.EmcError) as ei:
        E.load_model(str(p), side + 1)
    assert ei.value.status == 6
