"""Deterministic insertion: the same iterations run twice give bitwise the
same model, weight and scaling (fixed-point insertion sums, responsibility
lists in (rotation, pattern) order, slices summed in list order), in both
precisions, with the compress from lists, the dense tensor-core compress and
rotation chunks.  After one iteration the exact sums are within 1e-6 of the
FP32 atomic ones, and over three they hold the oracle bars."""
import numpy as np
import pytest

from parity import make_ctx, oracle_cfg, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    from emc_b200 import workloads as W
    return W.make("small32")


def _run(d, lik, interp, prec, det=True, lists=None, chunk=0, iters=3):
    import emc_b200 as E
    with make_ctx(d, lik, interp, prec) as ctx:
        if det:
            ctx.set_deterministic(True)
        if lists is not None:
            ctx.set_sparse_compress(lists)
        if chunk:
            ctx.set_rotation_chunk(chunk)
        for _ in range(iters):
            ctx.iterate()
        return ctx.get_model(), ctx.get_buffer(E.BUF_WEIGHT), ctx.get_scaling()


CASES = [
    ("poisson", "nearest", "mixed", None, 0),      # compress from responsibility lists
    ("poisson", "trilinear", "mixed", None, 0),
    ("gauss", "nearest", "mixed", None, 0),
    ("poisson", "nearest", "mixed", False, 0),     # dense tensor-core compress
    ("poisson", "nearest", "mixed", None, 512),    # rotation chunks
    ("gauss", "nearest", "fp32", None, 0),
    ("poisson", "trilinear", "fp32", True, 0),     # photon-list slice sums
]


@pytest.mark.parametrize("lik,interp,prec,lists,chunk", CASES)
def test_two_runs_are_bitwise_equal(small, lik, interp, prec, lists, chunk):
    a = _run(small, lik, interp, prec, lists=lists, chunk=chunk)
    b = _run(small, lik, interp, prec, lists=lists, chunk=chunk)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    # the exact sums against the FP32 atomics of the default mode, one
    # iteration (later iterations carry the atomics' own rounding forward)
    e = _run(small, lik, interp, prec, lists=lists, chunk=chunk, iters=1)
    c = _run(small, lik, interp, prec, det=False, lists=lists, chunk=chunk, iters=1)
    assert rel(e[0], c[0]) <= 1e-6, rel(e[0], c[0])
    assert rel(e[1], c[1]) <= 1e-6, rel(e[1], c[1])
    assert rel(e[2], c[2]) <= 1e-6, rel(e[2], c[2])


@pytest.mark.parametrize("prec,tol", [("mixed", 1e-4), ("fp32", 1e-5)])
def test_deterministic_iterations_match_the_oracle(small, prec, tol):
    from oracle import oracle as O
    d = small
    cfg = oracle_cfg(d, "poisson", "nearest")
    m_ref, s_ref = d["model0"].astype(np.float64), d["scaling0"].astype(np.float64)
    for _ in range(3):
        m_ref, s_ref, _, _ = O.iterate(cfg, d["counts"], d["mask"], d["q"], d["w"], d["x"], d["y"],
                                       d["z"], m_ref, s_ref)
    m, _, s = _run(d, "poisson", "nearest", prec)
    assert rel(m, m_ref) <= tol, rel(m, m_ref)
    assert rel(s, s_ref) <= tol


def test_deterministic_mode_is_refused_where_it_does_not_apply(small):
    import torch

    import emc_b200 as E
    from emc_b200.proposal import LearnedProposal, sorted_rotations
    d = small
    q, w, cell, n_cells = sorted_rotations(d["q"], d["w"], coarse_n=1)
    d = dict(d, q=q, w=w)
    with make_ctx(d, "poisson", "nearest", "mixed") as ctx:
        ctx.set_deterministic(True)
        with pytest.raises(E.EmcError) as ei:
            E.Batch([ctx])
        assert ei.value.status == 7
        lp = LearnedProposal(ctx, cell, n_cells)
        probs = torch.full((ctx.N, n_cells), 1.0 / n_cells, device="cuda")
        with pytest.raises(E.EmcError) as ei:
            lp.iterate_topk(probs, None, top_k=1, max_cells=4)
        assert ei.value.status == 7
        ctx.set_deterministic(False)
        lp.iterate_topk(probs, None, top_k=1, max_cells=4)
