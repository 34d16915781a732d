"""The oracle's own synthetic-input generator (used where only the oracle may
run, e.g. the timed CPU baseline) gives the engine's workloads bit for bit:
same coordinates, mask, counts, rotations, weights and initial model."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize("name,n", [("tiny16", None), ("small32", None), ("large128", 24)])
def test_oracle_workload_equals_engine_workload(name, n):
    from emc_b200 import workloads as W
    w = W.WORKLOADS[name]
    a = W.make(w, n_patterns=n, first_pattern=5)
    b = O.make_workload(w, n_patterns=n, first_pattern=5, wavelength=W.WAVELENGTH,
                        distance=W.DISTANCE, pixel_size=W.pixel_size(w.side))
    for k in ("x", "y", "z", "mask", "counts", "q", "w", "model0", "true_model", "scaling0"):
        assert a[k].dtype == b[k].dtype and a[k].shape == b[k].shape, k
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_oracle_iterate_rejects_mismatched_shapes():
    from emc_b200 import workloads as W
    d = W.make("tiny16")
    cfg = O.make_config(16, d["counts"].shape[0] + 1, d["q"].shape[0])
    with pytest.raises(ValueError):
        O.iterate(cfg, d["counts"], d["mask"], d["q"], d["w"], d["x"], d["y"], d["z"],
                  d["model0"], d["scaling0"])
