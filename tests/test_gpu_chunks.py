"""Rotation chunks of the mixed path: the log-likelihood held for one chunk of
rotations at a time, an online log-sum-exp over the tile partials of the
chunks so far, and the responsibilities kept as the entries of at least 1e-30
under that running log-sum-exp.

Against the unchunked iteration: lse, scaling and sum P log P come from the
same tile partials and are identical; responsibilities, T_r and model differ
only by the order of FP32/FP64 sums (tolerances 1e-5 per-pattern L1 and 1e-6
relative).  Against the FP64 oracle over three iterations at the mixed
path's bar (model and scaling 1e-4 relative).
"""
import numpy as np
import pytest

from parity import make_ctx, oracle_cfg, rel, resp_l1

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    from emc_b200 import workloads as W
    return W.make("small32")


def _one_iteration(d, lik, interp, rows, capacity=0):
    import emc_b200 as E
    with make_ctx(d, lik, interp, "mixed") as ctx:
        ctx.set_rotation_chunk(rows, capacity)
        assert ctx.rotation_chunk == (ctx.R if rows == 0 else rows)
        ctx.expand()
        ctx.maximize()
        out = dict(P=ctx.get_buffer(E.BUF_RESP), phi=ctx.get_scaling(),
                   T=ctx.get_buffer(E.BUF_TOTALRESP), stats=ctx.partial_stats(),
                   orient=ctx.orientation_stats(), cols=ctx.resp_columns([0, 5, 255]))
        ctx.compress()
        out["model"] = ctx.get_model()
        return out


# 3,240 rotations: chunks of 512 (six and one of 168), 256 (twelve and one
# of 168), 1,024 (three and one of 168) and 2,816 (one and one of 424)
@pytest.mark.parametrize("lik,interp,rows", [
    ("poisson", "nearest", 512), ("gauss", "nearest", 256), ("poisson", "trilinear", 1024),
    ("poisson", "nearest", 2816)])
def test_chunked_iteration_matches_unchunked(small, lik, interp, rows):
    one = _one_iteration(small, lik, interp, 0)
    ch = _one_iteration(small, lik, interp, rows)
    np.testing.assert_array_equal(ch["phi"], one["phi"])
    assert ch["stats"] == one["stats"]
    assert resp_l1(ch["P"], one["P"]) <= 1e-5, resp_l1(ch["P"], one["P"])
    assert rel(ch["T"], one["T"]) <= 1e-6
    assert rel(ch["model"], one["model"]) <= 1e-6, rel(ch["model"], one["model"])
    np.testing.assert_array_equal(ch["orient"]["best_rot"], one["orient"]["best_rot"])
    np.testing.assert_allclose(ch["orient"]["best_resp"], one["orient"]["best_resp"], rtol=1e-6)
    np.testing.assert_allclose(ch["cols"], one["cols"], rtol=1e-5, atol=1e-30)
    # every entry the chunked pass dropped is below 1e-30
    assert one["P"][ch["P"] == 0].max(initial=0.0) < 1e-30


def test_chunked_iterations_match_the_oracle(small):
    """Three chunked iterations (chunks of 768: four and one of 168) against
    the FP64 oracle."""
    from oracle import oracle as O
    d = small
    cfg = oracle_cfg(d, "poisson", "nearest")
    m_ref, s_ref = d["model0"].astype(np.float64), d["scaling0"].astype(np.float64)
    with make_ctx(d, "poisson", "nearest", "mixed") as ctx:
        ctx.set_rotation_chunk(768)
        for _ in range(3):
            ctx.iterate()
            m_ref, s_ref, _, _ = O.iterate(cfg, d["counts"], d["mask"], d["q"], d["w"], d["x"],
                                           d["y"], d["z"], m_ref, s_ref)
        assert rel(ctx.get_model(), m_ref) <= 1e-4, rel(ctx.get_model(), m_ref)
        assert rel(ctx.get_scaling(), s_ref) <= 1e-4


def test_kept_entry_overflow_grows_and_reruns(small):
    """Arrays for 64 kept entries: the iteration keeps more, grows them, runs
    its chunks again and ends where the default capacity does."""
    a = _one_iteration(small, "poisson", "nearest", 512)
    b = _one_iteration(small, "poisson", "nearest", 512, capacity=64)
    np.testing.assert_array_equal(b["P"], a["P"])
    np.testing.assert_array_equal(b["phi"], a["phi"])
    assert rel(b["model"], a["model"]) <= 1e-6


def test_chunks_chosen_from_the_memory_limit(small):
    """Under a memory limit that leaves less than the unchunked log-likelihood
    and compress operand (besides a reserve of 4 N (side^2 + active pixels)
    bytes + 1 GiB for patterns and lists), emc_set_geometry chooses chunks of
    the most rotations whose log-likelihood fits in half of what is left;
    rows = -1 chooses again.  Both iterate like the unchunked context."""
    import emc_b200 as E
    d = small
    w = d["workload"]
    N, R = d["counts"].shape[0], d["q"].shape[0]
    one = _one_iteration(d, "poisson", "nearest", 0)
    npad = (N + 127) // 128 * 128
    rpad = (R + 255) // 256 * 256
    y_bytes = 4 * R * npad
    big = y_bytes + 4 * rpad * npad  # Y and the dense compress operand P'
    with make_ctx(d, "poisson", "nearest", "mixed") as ctx:
        assert ctx.rotation_chunk == R
        reserve = 4 * N * (w.side ** 2 + ctx.active_pixels) + (1 << 30)
    ctx = E.Context(w.side, N, R, likelihood="poisson", interp="nearest", precision="mixed")
    try:
        ctx.set_geometry(d["x"], d["y"], d["z"], d["mask"])
        before_y = ctx.memory_used - big  # what emc_set_geometry holds besides Y and P'
    finally:
        ctx.close()
    # room for a third of Y beyond the reserve: chunks of about R / 6 rotations
    limit = before_y + reserve + y_bytes // 3
    ctx = E.Context(w.side, N, R, likelihood="poisson", interp="nearest", precision="mixed")
    try:
        ctx.set_memory_limit(limit)
        ctx.set_geometry(d["x"], d["y"], d["z"], d["mask"])
        expect = (y_bytes // 6) // (4 * npad) // 256 * 256
        assert ctx.rotation_chunk == max(expect, 256) < R, (ctx.rotation_chunk, expect)
        ctx.set_rotations(d["q"], d["w"])
        ctx.set_patterns(d["counts"])
        ctx.set_model(d["model0"])
        ctx.set_scaling(d["scaling0"])
        ctx.iterate()
        assert ctx.memory_used <= limit
        assert rel(ctx.get_model(), one["model"]) <= 1e-6
        ctx.set_rotation_chunk(-1)
        assert 256 <= ctx.rotation_chunk < R and ctx.rotation_chunk % 256 == 0
        ctx.set_model(d["model0"])
        ctx.set_scaling(d["scaling0"])
        ctx.iterate()
        assert rel(ctx.get_model(), one["model"]) <= 1e-6
    finally:
        ctx.close()


def test_chunk_arguments_are_checked(small):
    import emc_b200 as E
    d = small
    with make_ctx(d, "poisson", "nearest", "mixed") as ctx:
        for rows, status in ((300, 1), (-2, 1)):
            with pytest.raises(E.EmcError) as ei:
                ctx.set_rotation_chunk(rows)
            assert ei.value.status == status
        ctx.set_rotation_chunk(512)
        with pytest.raises(E.EmcError) as ei:
            E.Batch([ctx])
        assert ei.value.status == 7
        ctx.set_rotation_chunk(10 ** 9)  # more than R: one chunk
        assert ctx.rotation_chunk == ctx.R
    with make_ctx(d, "poisson", "nearest", "fp32") as ctx:
        with pytest.raises(E.EmcError) as ei:
            ctx.set_rotation_chunk(512)
        assert ei.value.status == 7


def test_chunked_cell_masses_match_unchunked(small):
    """Cell masses and log masses after a chunked iteration (from the kept
    entries) against the unchunked iteration's (from Y): equal where the
    mass is above the kept entries' 1e-30 floor."""
    from emc_b200.proposal import LearnedProposal, sorted_rotations
    q, w, cell, n_cells = sorted_rotations(small["q"], small["w"], coarse_n=1)
    d = dict(small, q=q, w=w)
    out = {}
    for rows in (0, 512):
        with make_ctx(d, "poisson", "nearest", "mixed") as ctx:
            ctx.set_rotation_chunk(rows)
            lp = LearnedProposal(ctx, cell, n_cells)
            ctx.iterate()
            out[rows] = (lp.targets().cpu().numpy(), lp.log_mass().cpu().numpy())
    (t0, l0), (t1, l1) = out[0], out[512]
    np.testing.assert_allclose(t1, t0, rtol=1e-5, atol=1e-7)
    big = l0 > np.log(1e-25)
    assert big.any()
    assert np.abs(l1[big] - l0[big]).max() <= 1e-4


def test_proposed_iterations_on_a_chunked_context(small):
    """The learned-proposal iteration on a chunked context: the dense
    iteration before it runs in chunks (its log cell masses come from the
    kept entries), and the proposed iteration, over the same candidates,
    gives the model and scaling of the unchunked context's."""
    import torch

    from emc_b200.proposal import LearnedProposal, sorted_rotations
    q, w, cell, n_cells = sorted_rotations(small["q"], small["w"], coarse_n=1)
    d = dict(small, q=q, w=w)
    N = d["counts"].shape[0]
    rng = np.random.default_rng(3)
    z = rng.standard_normal((N, n_cells)) * 2.0
    probs = np.exp(z - z.max(1, keepdims=True))
    probs = torch.from_numpy((probs / probs.sum(1, keepdims=True)).astype(np.float32)).cuda()
    out = {}
    for rows in (0, 512):
        with make_ctx(d, "poisson", "nearest", "mixed") as ctx:
            ctx.set_rotation_chunk(rows)
            lp = LearnedProposal(ctx, cell, n_cells)
            ctx.iterate()
            assert np.isfinite(lp.log_mass().cpu().numpy().max(axis=1)).all()
            # the same candidates for both contexts: from the fixed probabilities
            st = lp.iterate_topk(probs, None, top_k=1, max_cells=8, mass_target=0.9)
            assert st["fallback"] == 0
            out[rows] = (ctx.get_model(), ctx.get_scaling(), st["pairs"])
    assert out[512][2] == out[0][2]
    assert rel(out[512][1], out[0][1]) <= 1e-5
    assert rel(out[512][0], out[0][0]) <= 1e-5
