"""Engine vs FP64 oracle on the same seeded inputs, stage by stage and over
whole iterations, for every likelihood / interpolation / precision mode.

Tolerances (stated per check):
  * voxel choice and slicing are exact (bit-identical slices);
  * FP32 path: responsibilities within 1e-4 (per-pattern L1), scaling and
    models within 1e-5 relative;
  * mixed path (FP16 hi+lo operands, FP32 accumulation, FP64 log-sum-exp):
    responsibilities within 1e-3 (per-pattern L1), models within 1e-4.
"""
import numpy as np
import pytest

from oracle import oracle as O
from parity import active, make_ctx, oracle_cfg, rel, resp_l1

pytestmark = pytest.mark.gpu

MODES = [
    ("gauss", "nearest", "fp32"),
    ("poisson", "nearest", "fp32"),
    ("gauss", "trilinear", "fp32"),
    ("poisson", "trilinear", "fp32"),
    ("gauss", "nearest", "mixed"),
    ("poisson", "nearest", "mixed"),
    ("poisson", "trilinear", "mixed"),
]
TOL = {"fp32": dict(resp=1e-4, scale=1e-5, model=1e-5),
       "mixed": dict(resp=1e-3, scale=1e-4, model=1e-4)}


@pytest.fixture(scope="module")
def small():
    from emc_b200 import workloads as W
    return W.make("small32")


@pytest.fixture(scope="module")
def tiny():
    from emc_b200 import workloads as W
    return W.make("tiny16")


def _sigma(lik):
    return 0.4 if lik == "gauss" else 0.4


@pytest.mark.parametrize("lik,interp,prec", MODES)
def test_stages_match_oracle(small, lik, interp, prec):
    import emc_b200 as E
    d = small
    tol = TOL[prec]
    cfg = oracle_cfg(d, lik, interp)
    act = active(d)
    with make_ctx(d, lik, interp, prec) as ctx:
        # expand: slices on the active pixels are exact
        ctx.expand()
        S_ref = O.expand(cfg, d["model0"], d["q"], d["x"], d["y"], d["z"])
        S = ctx.get_buffer(E.BUF_SLICES)
        if prec == "fp32" and lik == "gauss" and interp == "nearest":
            np.testing.assert_array_equal(S, S_ref[:, act].astype(np.float32))
        elif prec == "fp32" and lik == "gauss":
            # trilinear weights are FP32 products on the GPU, FP64 in the oracle
            np.testing.assert_allclose(S, S_ref[:, act], rtol=1e-6, atol=1e-6)
        elif prec == "fp32":
            Lref = np.log(np.maximum(S_ref[:, act], 1e-10)).astype(np.float32)
            np.testing.assert_allclose(S, Lref, rtol=2e-6, atol=2e-6)
        else:
            ref = np.log(np.maximum(S_ref[:, act], 1e-10)) if lik == "poisson" else S_ref[:, act]
            assert np.abs(S - ref).max() <= 1e-6 * max(1.0, np.abs(ref).max())
        # maximize: responsibilities and the new scaling
        ctx.maximize()
        P = ctx.get_buffer(E.BUF_RESP)
        LL = O.loglik(cfg, S_ref, d["counts"], d["mask"], d["scaling0"])
        P_ref, lse, _ = O.softmax(LL)
        err_p = resp_l1(P, P_ref)
        assert err_p <= tol["resp"], f"responsibility L1 {err_p:.3g}"
        phi = ctx.get_scaling()
        phi_ref = O.update_scaling(cfg, S_ref, d["counts"], d["mask"], P_ref, d["scaling0"])
        assert rel(phi, phi_ref) <= max(tol["scale"], 10 * err_p), rel(phi, phi_ref)
        # compress: from the engine's own P and phi, the oracle inserts the same model
        ctx.compress()
        model = ctx.get_model()
        acc, wacc, T = O.compress(cfg, P.astype(np.float64), d["counts"], d["mask"],
                                  phi.astype(np.float64), d["q"], d["w"], d["x"], d["y"], d["z"])
        m_ref = O.normalize_model(acc, wacc)
        assert rel(model, m_ref) <= tol["model"], rel(model, m_ref)
        np.testing.assert_allclose(ctx.get_buffer(E.BUF_TOTALRESP), T, rtol=1e-4, atol=1e-6)


@pytest.mark.parametrize("lik,interp,prec", [MODES[0], MODES[1], MODES[4], MODES[5]])
def test_iterations_match_oracle(tiny, lik, interp, prec):
    d = tiny
    cfg = oracle_cfg(d, lik, interp)
    iters = d["workload"].iterations
    m_ref, s_ref = d["model0"].astype(np.float64), d["scaling0"].astype(np.float64)
    with make_ctx(d, lik, interp, prec) as ctx:
        for it in range(iters):
            st = ctx.iterate()
            m_ref, s_ref, _, st_ref = O.iterate(cfg, d["counts"], d["mask"], d["q"], d["w"], d["x"],
                                               d["y"], d["z"], m_ref, s_ref)
            assert abs(st["total_resp"] - d["counts"].shape[0]) < 1e-3 * d["counts"].shape[0]
        model = ctx.get_model()
    err = rel(model, m_ref)
    limit = {"fp32": 1e-4, "mixed": 1e-3}[prec]
    assert err <= limit, f"model error after {iters} iterations: {err:.3g}"


def test_mixed_rejects_inexact_counts(tiny):
    import emc_b200 as E
    d = dict(tiny)
    counts = d["counts"].copy()
    counts[0, 0] = 0.5
    w = d["workload"]
    ctx = E.Context(w.side, counts.shape[0], d["q"].shape[0], precision="mixed")
    ctx.set_geometry(d["x"], d["y"], d["z"], np.ones_like(d["mask"]))
    with pytest.raises(E.EmcError) as ei:
        ctx.set_patterns(counts)
    assert ei.value.status == 6
    ctx.close()


def test_stage_order_is_enforced(tiny):
    import emc_b200 as E
    with make_ctx(tiny) as ctx:
        with pytest.raises(E.EmcError) as ei:
            ctx.compress()
        assert ei.value.status == 5
        ctx.iterate()
        ctx.synchronize()


@pytest.mark.parametrize("prec", ["fp32", "mixed"])
def test_accumulator_view_and_split_compress(tiny, prec):
    """compress == compress_insert + normalize, and the zero-copy torch view of
    the accumulators (what a pattern-sharded run all-reduces) holds the model
    and weight sums."""
    import torch
    d = tiny
    M = d["workload"].side ** 3
    with make_ctx(d, precision=prec) as a, make_ctx(d, precision=prec) as b:
        a.iterate()
        b.expand()
        b.maximize()
        b.compress_insert()
        b.synchronize()
        acc = b.accumulator_tensor()
        assert acc.is_cuda and acc.numel() == 2 * M
        h = acc.double().cpu().numpy()
        msum, wsum = (h[:M], h[M:]) if prec == "fp32" else (h[0::2], h[1::2])
        expect = np.where(wsum > 0, msum / np.where(wsum > 0, wsum, 1), 0.0)
        expect /= expect.mean()
        b.normalize()
        model = b.get_model()
        torch.cuda.synchronize()
        np.testing.assert_allclose(model, a.get_model(), rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(model, expect, rtol=1e-5, atol=1e-6)


def test_autotune_keeps_results_and_restores_state(tiny):
    """emc_autotune times candidate tile orders from the current state and
    restores it; the tile order changes no result."""
    d = tiny
    with make_ctx(d, "poisson", "nearest", "mixed") as ctx:
        m0 = ctx.get_model()
        best, ms = ctx.autotune((1, 2, 4))
        assert ms.shape == (2, 3) and np.all(ms > 0)
        assert best[0] in (1, 2, 4) and best[1] in (1, 2, 4)
        np.testing.assert_array_equal(ctx.get_model(), m0)
        ctx.set_tuning(1, 1)
        ctx.iterate()
        m1 = ctx.get_model()
        ctx.set_model(m0)
        ctx.set_scaling(d["scaling0"])
        ctx.set_tuning(3, 5)
        assert ctx.get_tuning()[:2] == (3, 5)
        ctx.iterate()
        assert rel(ctx.get_model(), m1) < 1e-6


@pytest.mark.parametrize("lik", ["poisson", "gauss"])
def test_pair_maximize_matches_oracle_and_one_sm_kernel(small, lik):
    """Both contractions on SM pairs (cta_group::2: 256-pattern / 256-rotation
    tiles, half of the B operand per SM) give the responsibilities and the
    model of the one-SM kernels and of the oracle."""
    import emc_b200 as E
    d = small
    cfg = oracle_cfg(d, lik, "nearest")
    S = O.expand(cfg, d["model0"], d["q"], d["x"], d["y"], d["z"])
    LL = O.loglik(cfg, S, d["counts"], d["mask"], d["scaling0"])
    P_ref, _, _ = O.softmax(LL)
    with make_ctx(d, lik, "nearest", "mixed") as ctx:
        ctx.expand()
        ctx.maximize()
        P1 = ctx.get_buffer(E.BUF_RESP)
        ctx.compress()
        m1 = ctx.get_model()
        ctx.set_model(d["model0"])
        ctx.set_scaling(d["scaling0"])
        ctx.set_tuning(1, 6, 1, 1)
        assert ctx.get_tuning()[2:] == (1, 1)
        ctx.expand()
        ctx.maximize()
        P2 = ctx.get_buffer(E.BUF_RESP)
        ctx.compress()
        m2 = ctx.get_model()
    assert resp_l1(P2, P1) <= 1e-4, resp_l1(P2, P1)
    assert resp_l1(P2, P_ref) <= TOL["mixed"]["resp"], resp_l1(P2, P_ref)
    assert rel(m2, m1) <= 1e-5, rel(m2, m1)


def test_pair_maximize_at_size():
    """Many pair tiles (3,000 patterns: the last 256-pattern tile half past
    the padded rows; 25,680 rotations): same responsibilities and model as
    the one-SM kernel."""
    import emc_b200 as E
    from emc_b200 import workloads as W
    d = W.make("b200_64", n_patterns=3000)
    out = []
    for pair in (0, 1):
        with make_ctx(d, "poisson", "nearest", "mixed") as ctx:
            ctx.set_tuning(1, 6, pair, pair)
            ctx.expand()
            ctx.maximize()
            P = ctx.get_buffer(E.BUF_RESP)
            ctx.compress()
            out.append((P, ctx.get_model(), ctx.get_scaling()))
    assert resp_l1(out[1][0], out[0][0]) <= 1e-4
    assert rel(out[1][1], out[0][1]) <= 1e-5
    assert rel(out[1][2], out[0][2]) <= 1e-6


@pytest.mark.parametrize("lik,interp", [("poisson", "nearest"), ("gauss", "nearest"),
                                        ("poisson", "trilinear")])
def test_list_compress_matches_dense_contraction(small, lik, interp):
    """The mixed compress from responsibility lists (per rotation, the
    patterns with a non-zero operand entry, times their photon lists; the
    default) gives the model of the dense tensor-core compress on one SM and
    on SM pairs, and the oracle's compress of the engine's responsibilities."""
    import emc_b200 as E
    d = small
    cfg = oracle_cfg(d, lik, interp)
    out = {}
    for mode in ("lists", "dense", "dense_pairs"):
        with make_ctx(d, lik, interp, "mixed") as ctx:
            assert ctx.tuning()["compress_sparse"] == 1
            if mode != "lists":
                ctx.set_sparse_compress(False)
                ctx.set_tuning(1, 2, 0, 1 if mode == "dense_pairs" else 0)
            ctx.expand()
            ctx.maximize()
            P, phi = ctx.get_buffer(E.BUF_RESP), ctx.get_scaling()
            ctx.compress()
            out[mode] = (ctx.get_model(), ctx.get_buffer(E.BUF_TOTALRESP), P, phi)
    m, T, P, phi = out["lists"]
    acc, wacc, T_ref = O.compress(cfg, P.astype(np.float64), d["counts"], d["mask"],
                                  phi.astype(np.float64), d["q"], d["w"], d["x"], d["y"], d["z"])
    assert rel(m, O.normalize_model(acc, wacc)) <= 1e-5, rel(m, O.normalize_model(acc, wacc))
    np.testing.assert_allclose(T, T_ref, rtol=1e-4, atol=1e-6)
    # the dense contraction rounds the operand to FP16 hi + lo: within the
    # mixed path's model tolerance of the lists
    for mode in ("dense", "dense_pairs"):
        assert rel(out[mode][0], m) <= TOL["mixed"]["model"], (mode, rel(out[mode][0], m))
