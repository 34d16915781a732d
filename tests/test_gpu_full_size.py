"""Full benchmark sizes, checked through size-independent properties.

At 64^3 / 25,680 rotations / 10,000 patterns and at the 128^3 / 86,520
rotation geometry, one iteration of each path must give responsibilities that
sum to one per pattern, a total responsibility equal to the pattern count, a
model normalised to mean 1; the mixed and FP32 paths must agree; and the
responsibilities of sampled patterns must match the FP64 oracle (a pattern's
responsibilities depend only on the model, the scaling and that pattern).
"""
import numpy as np
import pytest

from oracle import oracle as O
from parity import make_ctx, oracle_cfg, rel

pytestmark = pytest.mark.gpu


def _one_iteration(d, precision, lik="poisson"):
    import emc_b200 as E
    with make_ctx(d, likelihood=lik, precision=precision) as ctx:
        ctx.expand()
        ctx.maximize()
        P_cols = ctx.get_buffer(E.BUF_RESP)[:, :8].copy()
        colsum = None
        if precision == "fp32":
            colsum = ctx.get_buffer(E.BUF_RESP).sum(axis=0, dtype=np.float64)
        ctx.compress()
        model = ctx.get_model()
        T = ctx.get_buffer(E.BUF_TOTALRESP)
        scaling = ctx.get_scaling()
    return P_cols, colsum, model, T, scaling


@pytest.mark.parametrize("workload,n_patterns", [("b200_64", None), ("large128", 4000)])
def test_full_size_properties(workload, n_patterns):
    from emc_b200 import workloads as W
    d = W.make(workload, n_patterns=n_patterns)
    N, R = d["counts"].shape[0], d["q"].shape[0]
    Pm, _, mm, Tm, sm = _one_iteration(d, "mixed")
    Pf, colsum, mf, Tf, sf = _one_iteration(d, "fp32")
    for model, T in ((mm, Tm), (mf, Tf)):
        assert np.isfinite(model).all() and model.min() >= 0
        assert abs(model.astype(np.float64).mean() - 1.0) < 1e-4
        assert abs(T.astype(np.float64).sum() - N) < 1e-3 * N
    np.testing.assert_allclose(colsum, 1.0, atol=1e-3)
    # the two precisions agree
    assert rel(mm, mf) < 1e-3, rel(mm, mf)
    assert rel(sm, sf) < 1e-4, rel(sm, sf)
    np.testing.assert_allclose(Tm, Tf, atol=1e-3 * max(1.0, Tf.max()))
    # sampled patterns against the FP64 oracle (first 8 patterns, every rotation)
    if R * (W.WORKLOADS[workload].side ** 2) <= 2e8:
        n = 8
        cfg = oracle_cfg(dict(d, counts=d["counts"][:n]), "poisson")
        _, _, P_ref, _ = O.iterate(cfg, d["counts"][:n], d["mask"], d["q"], d["w"], d["x"], d["y"],
                                   d["z"], d["model0"], d["scaling0"][:n], want_resp=True)
        for P in (Pm, Pf):
            err = np.abs(P.astype(np.float64) - P_ref).sum(axis=0).max()
            assert err < 2e-3, err


# Bars of the benchmark geometry against the FP64 oracle: the mixed path must
# hold responsibility L1 <= 1e-2 per pattern and model <= 1e-3 relative; the
# FP32 path the FP32 bars of the parity tests.
LARGE_BARS = {"mixed": (1e-2, 1e-3), "fp32": (1e-4, 1e-5)}


@pytest.mark.parametrize("precision", ["mixed", "fp32"])
def test_large128_sample_vs_oracle(precision):
    """The 128^3 benchmark geometry (128x128 detector, radius-6 beamstop,
    16,272 active pixels, 500 photons on average, ~3% non-zero pixels) on
    every 43rd of its 86,520 rotations and its first 384 patterns: one
    iteration of the engine against the oracle's from the same model."""
    import emc_b200 as E
    from emc_b200 import workloads as W
    d = W.make("large128", n_patterns=384)
    rot = np.arange(0, d["q"].shape[0], 43)
    d = dict(d, q=d["q"][rot], w=d["w"][rot])
    cfg = oracle_cfg(d, "poisson")
    m_ref, s_ref, P_ref, _ = O.iterate(cfg, d["counts"], d["mask"], d["q"], d["w"], d["x"],
                                       d["y"], d["z"], d["model0"], d["scaling0"],
                                       want_resp=True)
    with make_ctx(d, "poisson", "nearest", precision) as ctx:
        ctx.expand()
        ctx.maximize()
        P = ctx.get_buffer(E.BUF_RESP)
        ctx.compress()
        model, scaling = ctx.get_model(), ctx.get_scaling()
    err_p = float(np.abs(P.astype(np.float64) - P_ref).sum(axis=0).max())
    err_m, err_s = rel(model, m_ref), rel(scaling, s_ref)
    print(f"large128 sample ({precision}): responsibility L1 {err_p:.3g}, scaling {err_s:.3g}, "
          f"model {err_m:.3g}")
    bar_p, bar_m = LARGE_BARS[precision]
    assert err_p <= bar_p, f"responsibility L1 {err_p:.3g}"
    assert err_m <= bar_m, f"model error {err_m:.3g}"
