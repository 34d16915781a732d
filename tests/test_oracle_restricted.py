"""The oracle's restricted iteration (softmax over a per-pattern candidate set
of rotations), the reference semantics of the learned proposal's iteration."""
import numpy as np
import pytest

from oracle import oracle as O
from parity import oracle_cfg


@pytest.fixture(scope="module")
def tiny():
    from emc_b200 import workloads as W
    return W.make("tiny16")


def _args(d):
    return (d["counts"], d["mask"], d["q"], d["w"], d["x"], d["y"], d["z"],
            d["model0"].astype(np.float64), d["scaling0"].astype(np.float64))


def test_all_allowed_equals_plain_iteration(tiny):
    d = tiny
    cfg = oracle_cfg(d, "poisson")
    R, N = d["q"].shape[0], d["counts"].shape[0]
    m0, s0, P0, st0 = O.iterate(cfg, *_args(d), want_resp=True)
    m1, s1, P1, st1 = O.iterate(cfg, *_args(d), want_resp=True, allowed=np.ones((R, N), np.uint8))
    np.testing.assert_array_equal(m0, m1)
    np.testing.assert_array_equal(s0, s1)
    np.testing.assert_array_equal(P0, P1)


def test_restriction_zeroes_responsibility_outside_the_set(tiny):
    d = tiny
    cfg = oracle_cfg(d, "gauss")
    R, N = d["q"].shape[0], d["counts"].shape[0]
    rng = np.random.default_rng(1)
    allowed = (rng.random((R, N)) < 0.2).astype(np.uint8)
    allowed[0] = 1  # every pattern keeps a candidate
    m, s, P, st = O.iterate(cfg, *_args(d), want_resp=True, allowed=allowed)
    assert np.all(P[allowed == 0] == 0.0)
    np.testing.assert_allclose(P.sum(0), 1.0, rtol=1e-12)
    assert np.isfinite(m).all() and np.isfinite(s).all()
