"""Orientation diagnostics (best rotation, its responsibility, average
responsibility per rotation) and the viewer-readable output files."""
import numpy as np
import pytest

from parity import make_ctx, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["fp32", "mixed"])
def test_orientation_stats_match_the_responsibilities(prec):
    import emc_b200 as E
    from emc_b200 import workloads as W
    d = W.make("tiny16")
    with make_ctx(d, "poisson", "nearest", prec) as ctx:
        ctx.iterate()
        ctx.expand()
        ctx.maximize()
        P = ctx.get_buffer(E.BUF_RESP)
        o = ctx.orientation_stats()
        N = P.shape[1]
        agree = o["best_rot"] == P.argmax(0)
        assert agree.mean() >= 0.99
        # where the index differs the two rotations carry the same responsibility
        np.testing.assert_allclose(P[o["best_rot"], np.arange(N)], P.max(0), rtol=1e-5, atol=1e-7)
        np.testing.assert_allclose(o["best_resp"], P.max(0), rtol=1e-4, atol=1e-7)
        np.testing.assert_allclose(o["avg_resp"], P.sum(1) / N, rtol=1e-4, atol=1e-8)


def test_orientation_stats_of_a_proposed_iteration():
    import torch
    from emc_b200 import workloads as W
    from emc_b200.proposal import LearnedProposal
    from oracle import oracle as O
    from parity import oracle_cfg
    from test_gpu_proposal import _proposal_case
    d, cell, n_cells, probs, allowed = _proposal_case(W.make("tiny16"), 7)
    cfg = oracle_cfg(d, "poisson", "nearest")
    _, _, P_ref, _ = O.iterate(cfg, d["counts"], d["mask"], d["q"], d["w"], d["x"], d["y"], d["z"],
                               d["model0"].astype(np.float64), d["scaling0"].astype(np.float64),
                               want_resp=True, allowed=allowed)
    with make_ctx(d, "poisson", "nearest", "mixed") as ctx:
        lp = LearnedProposal(ctx, cell, n_cells)
        lp.iterate(torch.from_numpy(probs).cuda(), 7, threshold=0.0)
        o = ctx.orientation_stats()
    N = P_ref.shape[1]
    assert np.all(allowed[o["best_rot"], np.arange(N)] == 1)
    assert (o["best_rot"] == P_ref.argmax(0)).mean() >= 0.95
    np.testing.assert_allclose(o["best_resp"], P_ref[o["best_rot"], np.arange(N)], atol=2e-3)
    np.testing.assert_allclose(o["avg_resp"], P_ref.sum(1) / N, atol=1e-5)


def test_output_files_read_back_like_the_viewer(tmp_path):
    import emc_b200 as E
    from emc_b200 import workloads as W
    from emc_b200.diagnostics import OutputWriter
    d = W.make("tiny16")
    out = OutputWriter(str(tmp_path))
    with make_ctx(d, "poisson", "nearest", "mixed") as ctx:
        for it in range(2):
            st = ctx.iterate()
            out.record(it, ctx, st["sum_plogp"])
        model = ctx.get_model()
    N, R = d["counts"].shape[0], d["q"].shape[0]
    assert np.loadtxt(tmp_path / "likelihood.data").shape == (2,)
    best = np.loadtxt(tmp_path / "best_rot.data")
    assert best.shape == (2, N) and best.min() >= 0 and best.max() < R
    assert np.loadtxt(tmp_path / "best_scaling.data").shape == (2, N)
    avg = np.loadtxt(tmp_path / "average_resp_0001.data")
    assert avg.shape == (R,) and abs(avg.sum() - 1.0) < 1e-3
    np.testing.assert_array_equal(E.load_model(str(tmp_path / "model_0001.raw"), 16), model)


@pytest.mark.parametrize("prec", ["fp32", "mixed"])
def test_photon_list_ingest_equals_dense_patterns(prec):
    """emc_set_patterns_sparse (CSR photon lists, as (pixel, count) pairs or
    one entry per photon) gives the iteration of the dense upload."""
    import emc_b200 as E
    from emc_b200 import workloads as W
    d = W.make("small32")
    with make_ctx(d, "poisson", "nearest", prec) as ctx:
        m0 = ctx.get_model()
        ctx.iterate()
        m_dense, s_dense = ctx.get_model(), ctx.get_scaling()
        rp, px, ct = E.photon_lists(d["counts"])
        assert px.size == np.count_nonzero(d["counts"])
        for photons in (False, True):
            if photons:  # one entry per photon, in shuffled order within a pattern
                rep = ct.astype(np.int64)
                px2 = np.repeat(px, rep)
                rp2 = np.zeros_like(rp)
                np.cumsum(np.add.reduceat(rep, rp[:-1]) * (np.diff(rp) > 0), out=rp2[1:])
                rng = np.random.default_rng(0)
                for p in range(len(rp2) - 1):
                    rng.shuffle(px2[rp2[p]:rp2[p + 1]])
                ctx.set_patterns_sparse(rp2, px2)
            else:
                ctx.set_patterns_sparse(rp, px, ct)
            ctx.set_model(m0)
            ctx.set_scaling(d["scaling0"])
            ctx.iterate()
            assert rel(ctx.get_model(), m_dense) < 1e-6
            assert rel(ctx.get_scaling(), s_dense) < 1e-6
        bad = px.copy()
        bad[0] = 32 * 32
        with pytest.raises(E.EmcError):
            ctx.set_patterns_sparse(rp, bad, ct)
