"""Photon-list forms of the FP32 path: the poisson log-likelihood gathered
over each pattern's non-zero pixels, and the slice sums gathered over each
pixel's non-zero counts, give the responsibilities, scaling and model of the
dense FP32 contractions and of the FP64 oracle.

Tolerances: against the oracle, the FP32 bars of the dense path
(responsibilities within 1e-4 per-pattern L1, models within 1e-5 relative);
against the dense FP32 path twice that for the responsibilities (both carry
FP32 rounding of log-likelihoods of magnitude ~1e4, summed in another order)
and 1e-5 for scaling and model.
"""
import numpy as np
import pytest

from oracle import oracle as O
from parity import make_ctx, oracle_cfg, rel, resp_l1

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    from emc_b200 import workloads as W
    return W.make("small32")


def _stage(ctx):
    import emc_b200 as E
    ctx.expand()
    ctx.maximize()
    P = ctx.get_buffer(E.BUF_RESP)
    phi = ctx.get_scaling()
    ctx.compress()
    return P, phi, ctx.get_model()


@pytest.mark.parametrize("interp", ["nearest", "trilinear"])
def test_sparse_matches_dense_and_oracle(small, interp):
    d = small
    with make_ctx(d, "poisson", interp, "fp32") as ctx:
        P0, phi0, m0 = _stage(ctx)
    with make_ctx(d, "poisson", interp, "fp32") as ctx:
        ctx.set_sparse_maximize(True)
        P1, phi1, m1 = _stage(ctx)
    assert resp_l1(P1, P0) <= 2e-4, resp_l1(P1, P0)
    assert rel(phi1, phi0) <= 1e-5
    assert rel(m1, m0) <= 1e-5
    cfg = oracle_cfg(d, "poisson", interp)
    S = O.expand(cfg, d["model0"], d["q"], d["x"], d["y"], d["z"])
    LL = O.loglik(cfg, S, d["counts"], d["mask"], d["scaling0"])
    P_ref, _, _ = O.softmax(LL)
    assert resp_l1(P1, P_ref) <= 1e-4, (resp_l1(P1, P_ref), resp_l1(P0, P_ref))


def test_sparse_ragged_and_empty_patterns():
    """Empty patterns (no photons), a pattern count that is not a multiple of
    the 16-pattern block and a rotation count that is neither a multiple of
    the 512-rotation block nor of the 4 rotations a thread gathers;
    iterations against the oracle."""
    from emc_b200 import workloads as W
    d = dict(W.make("tiny16"))
    counts = d["counts"][:45].copy()
    counts[[0, 17, 44]] = 0.0
    d["counts"], d["scaling0"] = counts, d["scaling0"][:45]
    d["q"], d["w"] = d["q"][:301], d["w"][:301]
    cfg = oracle_cfg(d, "poisson", "nearest")
    m_ref, s_ref = d["model0"].astype(np.float64), d["scaling0"].astype(np.float64)
    with make_ctx(d, "poisson", "nearest", "fp32") as ctx:
        ctx.set_sparse_maximize(True)
        for _ in range(3):
            ctx.iterate()
            m_ref, s_ref, _, _ = O.iterate(cfg, d["counts"], d["mask"], d["q"], d["w"], d["x"],
                                           d["y"], d["z"], m_ref, s_ref)
        model = ctx.get_model()
    assert rel(model, m_ref) <= 1e-4, rel(model, m_ref)


def test_sparse_follows_new_patterns(small):
    """A second pattern upload rebuilds the photon lists."""
    d = small
    other = np.ascontiguousarray(d["counts"][::-1])
    with make_ctx(d, "poisson", "nearest", "fp32") as ctx:
        ctx.set_sparse_maximize(True)
        _stage(ctx)
        ctx.set_patterns(other)
        ctx.set_model(d["model0"])
        ctx.set_scaling(np.ascontiguousarray(d["scaling0"][::-1]))
        P1, _, m1 = _stage(ctx)
    d2 = dict(d, counts=other, scaling0=np.ascontiguousarray(d["scaling0"][::-1]))
    with make_ctx(d2, "poisson", "nearest", "fp32") as ctx:
        P0, _, m0 = _stage(ctx)
    assert resp_l1(P1, P0) <= 2e-4
    assert rel(m1, m0) <= 1e-5


@pytest.mark.parametrize("lik,prec", [("poisson", "mixed"), ("gauss", "fp32")])
def test_sparse_rejected_outside_fp32_poisson(small, lik, prec):
    import emc_b200 as E
    with make_ctx(small, lik, "nearest", prec) as ctx:
        with pytest.raises(E.EmcError) as ei:
            ctx.set_sparse_maximize(True)
        assert ei.value.status == 7
        if prec == "mixed":
            # the mixed compress_sparse form is the responsibility lists
            ctx.set_sparse_compress(True)
            assert ctx.tuning()["compress_sparse"] == 1


@pytest.mark.parametrize("lik", ["poisson", "gauss"])
def test_sparse_slice_sums_match_dense_and_oracle(small, lik):
    """Slice sums gathered over each pixel's non-zero counts (FP32, both
    likelihoods): the model of the dense FP32 compress and of the oracle's
    insertion from the engine's own responsibilities."""
    import emc_b200 as E
    d = small
    with make_ctx(d, lik, "nearest", "fp32") as ctx:
        P0, phi0, m0 = _stage(ctx)
    with make_ctx(d, lik, "nearest", "fp32") as ctx:
        ctx.set_sparse_compress(True)
        P1, phi1, m1 = _stage(ctx)
        T1 = ctx.get_buffer(E.BUF_TOTALRESP)
    np.testing.assert_array_equal(P1, P0)  # the maximize is unchanged
    assert rel(m1, m0) <= 1e-5, rel(m1, m0)
    cfg = oracle_cfg(d, lik, "nearest")
    acc, wacc, T = O.compress(cfg, P1.astype(np.float64), d["counts"], d["mask"],
                              phi1.astype(np.float64), d["q"], d["w"], d["x"], d["y"], d["z"])
    assert rel(m1, O.normalize_model(acc, wacc)) <= 1e-5
    np.testing.assert_allclose(T1, T, rtol=1e-4, atol=1e-6)


def test_sparse_iteration_both_gathers_ragged():
    """Photon-list maximize and slice sums together over three iterations
    with empty patterns and ragged sizes, against the oracle."""
    from emc_b200 import workloads as W
    d = dict(W.make("tiny16"))
    counts = d["counts"][:45].copy()
    counts[[0, 17, 44]] = 0.0
    d["counts"], d["scaling0"] = counts, d["scaling0"][:45]
    d["q"], d["w"] = d["q"][:301], d["w"][:301]
    cfg = oracle_cfg(d, "poisson", "nearest")
    m_ref, s_ref = d["model0"].astype(np.float64), d["scaling0"].astype(np.float64)
    with make_ctx(d, "poisson", "nearest", "fp32") as ctx:
        ctx.set_sparse_maximize(True)
        ctx.set_sparse_compress(True)
        for _ in range(3):
            ctx.iterate()
            m_ref, s_ref, _, _ = O.iterate(cfg, d["counts"], d["mask"], d["q"], d["w"], d["x"],
                                           d["y"], d["z"], m_ref, s_ref)
        model = ctx.get_model()
    assert rel(model, m_ref) <= 1e-4, rel(model, m_ref)


def test_fp32_autotune_picks_forms_and_restores_state(small):
    """emc_autotune on an FP32 context times the dense and the photon-list
    forms, keeps the faster of each, and leaves model and scaling as they
    were; the chosen forms give the dense iteration's model."""
    d = small
    with make_ctx(d, "poisson", "nearest", "fp32") as ctx:
        ctx.iterate()
        m_dense = ctx.get_model()
    with make_ctx(d, "poisson", "nearest", "fp32") as ctx:
        m0 = ctx.get_model()
        _, ms = ctx.autotune((1,))
        assert ms[0, 0] > 0 and ms[1, 0] > 0
        t = ctx.tuning()
        assert t["maximize_sparse"] in (0, 1) and t["compress_sparse"] in (0, 1)
        np.testing.assert_array_equal(ctx.get_model(), m0)
        ctx.iterate()
        assert rel(ctx.get_model(), m_dense) <= 1e-5
