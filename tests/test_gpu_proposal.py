"""Learned rotation proposal: the network's gradients against a float64 torch
autograd reference of the same architecture, and the proposal end to end
(trained on dense responsibilities; captured responsibility mass; model of a
proposed iteration against the dense iteration; fallback)."""
import numpy as np
import pytest

from parity import make_ctx, rel

pytestmark = pytest.mark.gpu


def _torch_reference(params, x, t, in_side, n_out):
    """Forward + backward of the network in float64 (CPU), same parameter layout:
    W[co][ci][3][3] then b[co] for three stride-2 convolutions, Wfc[c][f], bfc[c]."""
    import torch
    import torch.nn.functional as F
    ch = [1, 16, 32, 64]
    p = torch.tensor(params, dtype=torch.float64)
    off, views = 0, []
    for l in range(3):
        n = ch[l + 1] * ch[l] * 9
        views.append(p[off:off + n].view(ch[l + 1], ch[l], 3, 3))
        off += n
        views.append(p[off:off + ch[l + 1]])
        off += ch[l + 1]
    nf = 64 * (in_side // 8) ** 2
    views.append(p[off:off + n_out * nf].view(n_out, nf))
    off += n_out * nf
    views.append(p[off:off + n_out])
    leaves = [v.clone().requires_grad_(True) for v in views]
    h = torch.tensor(x, dtype=torch.float64).view(-1, 1, in_side, in_side)
    for l in range(3):
        h = F.relu(F.conv2d(h, leaves[2 * l], leaves[2 * l + 1], stride=2, padding=1))
    z = h.reshape(h.shape[0], -1) @ leaves[6].T + leaves[7]
    tt = torch.tensor(t, dtype=torch.float64)
    loss = -(tt * F.log_softmax(z, dim=1)).sum(1).mean()
    loss.backward()
    return float(loss.detach()), np.concatenate([v.grad.reshape(-1).numpy() for v in leaves])


@pytest.mark.parametrize("bf16,tol", [(False, 1e-4), (True, 5e-2)])
def test_network_gradients_match_float64_reference(bf16, tol):
    import torch
    from emc_b200.proposal import ProposalNet
    in_side, n_out, B = 16, 10, 5
    net = ProposalNet(in_side, n_out, bf16=bf16, seed=3)
    rng = np.random.default_rng(0)
    params = (rng.standard_normal(net.num_params) * 0.2).astype(np.float32)
    if bf16:  # the forward pass sees bf16 weights: give the reference the same values
        params = torch.tensor(params).bfloat16().float().numpy()
    net.set_params(params)
    x = rng.uniform(0, 2, (B, in_side * in_side)).astype(np.float32)
    t = rng.uniform(0, 1, (B, n_out)).astype(np.float32)
    t /= t.sum(1, keepdims=True)
    loss, g = net.gradients(torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda())
    loss_ref, g_ref = _torch_reference(params.astype(np.float64), x.astype(np.float64),
                                       t.astype(np.float64), in_side, n_out)
    assert abs(loss - loss_ref) <= tol * abs(loss_ref)
    # per tensor relative error (layout W1 b1 W2 b2 W3 b3 Wfc bfc)
    sizes = [16 * 9, 16, 32 * 144, 32, 64 * 288, 64, n_out * 64 * 4, n_out]
    o = 0
    for sz in sizes:
        assert rel(g[o:o + sz], g_ref[o:o + sz]) <= tol, (o, rel(g[o:o + sz], g_ref[o:o + sz]))
        o += sz
    net.close()


def test_learned_proposal_end_to_end():
    import torch
    from emc_b200 import workloads as W
    from emc_b200.proposal import LearnedProposal, sorted_rotations
    d = W.make("b200_64", n_patterns=3000)
    q, w, cell, n_cells = sorted_rotations(d["q"], d["w"], coarse_n=2)
    d = dict(d, q=q, w=w)
    members = np.bincount(cell, minlength=n_cells)
    m = int(np.ceil(512 / members.mean()))  # about 512 fine rotations per pattern
    with make_ctx(d, likelihood="poisson", precision="mixed") as ctx:
        for _ in range(3):
            ctx.iterate()
        lp = LearnedProposal(ctx, cell, n_cells, bf16=True, seed=1)
        x, t = lp.features(), lp.targets()
        np.testing.assert_allclose(t.sum(1).cpu().numpy(), 1.0, atol=1e-4)

        def captured(probs):
            top = torch.topk(probs, m, dim=1).indices
            return torch.gather(t, 1, top).sum(1).cpu().numpy()

        before = captured(lp.predict(x))
        losses = lp.train(x, t, epochs=25, batch=256, lr=2e-3)
        probs = lp.predict(x)
        after = captured(probs)
        assert losses[-1] < losses[0]
        # what the trained network gains over the untrained one: the true
        # responsibility mass on the evaluated rotations
        assert after.mean() > 0.95 and after.mean() > before.mean() + 0.3, (before.mean(), after.mean())
        m0, s0 = ctx.get_model(), ctx.get_scaling()
        st = lp.iterate(probs, m, threshold=0.0)
        assert st["fallback"] == 0
        assert st["mean_mass"] > 0.9 and st["pairs"] == 3000 * m
        frac = st["evaluations"] / (3000 * len(q))
        assert frac < 0.03, frac
        m_prop = ctx.get_model()
        ctx.set_model(m0)
        ctx.set_scaling(s0)
        ctx.iterate()
        m_dense = ctx.get_model()
        err = rel(m_prop, m_dense)
        print(f"proposal: captured mass untrained {before.mean():.4f} trained {after.mean():.4f} "
              f"(min {after.min():.4f}); evaluated fraction {frac:.4f}; model error vs dense {err:.2e}")
        assert err < 2e-2, err
        # the fallback runs the dense iteration
        ctx.set_model(m0)
        ctx.set_scaling(s0)
        st = lp.iterate(probs, m, threshold=1.01)
        assert st["fallback"] == 1
        assert rel(ctx.get_model(), m_dense) < 1e-5


def _select(probs, max_cells, mass_target, min_cells=1, keep=None, keep_mass=0.0):
    """The candidate cells emc_iterate_proposed takes: with keep, first the
    most probable cells under keep that hold keep > 0 until at least
    min_cells are taken and their (FP32) keep sum reaches keep_mass; then
    cells in order of probs until at least min_cells are taken and their
    (FP32) probs sum reaches mass_target, at most max_cells."""
    N, n_cells = probs.shape
    sel = np.zeros((N, n_cells), bool)
    for p in range(N):
        tot, n = np.float32(0), 0
        if keep is not None:
            ktot = np.float32(0)
            for k in np.argsort(-keep[p], kind="stable"):
                if n >= max_cells or (n >= min_cells and not ktot < np.float32(keep_mass)):
                    break
                if not keep[p, k] > 0:
                    break
                sel[p, k] = True
                n += 1
                ktot = np.float32(ktot + keep[p, k])
                tot = np.float32(tot + max(probs[p, k], np.float32(0)))
        for k in np.argsort(-probs[p], kind="stable"):
            if n >= max_cells or (mass_target < 1.0 and n >= min_cells and tot >= mass_target):
                break
            if sel[p, k]:
                continue
            sel[p, k] = True
            n += 1
            tot = np.float32(tot + probs[p, k])
    return sel


def _proposal_case(d, max_cells, mass_target=1.0, seed=0, min_cells=1, keep=False, keep_mass=0.0):
    """Rotations sorted by coarse cell (n=1: 60 uneven cells), distinct random
    cell probabilities (and, with keep, a second random posterior with half
    of each row zero), and the allowed[r][p] mask of the selected cells."""
    from emc_b200.proposal import sorted_rotations
    q, w, cell, n_cells = sorted_rotations(d["q"], d["w"], coarse_n=1)
    d = dict(d, q=q, w=w)
    N = d["counts"].shape[0]
    rng = np.random.default_rng(seed)
    z = rng.standard_normal((N, n_cells)) * 2.0
    probs = np.exp(z - z.max(1, keepdims=True))
    probs = (probs / probs.sum(1, keepdims=True)).astype(np.float32)
    kp = None
    if keep:
        z = rng.standard_normal((N, n_cells)) * 3.0
        kp = np.exp(z - z.max(1, keepdims=True)) * (rng.random((N, n_cells)) < 0.5)
        kp[:3] = 0.0  # patterns with no kept cell at all
        kp = kp.astype(np.float32)
    sel = _select(probs, max_cells, mass_target, min_cells, kp, keep_mass)
    allowed = sel[:, cell].T.astype(np.uint8)  # [R][N]
    if keep:
        return d, cell, n_cells, probs, allowed, kp
    return d, cell, n_cells, probs, allowed


@pytest.mark.parametrize("lik,interp,prec,tol,max_cells,mass_target,min_cells,keep,keep_mass,pair", [
    ("poisson", "nearest", "fp32", 1e-5, 7, 1.0, 1, False, 0.0, False),
    ("gauss", "nearest", "fp32", 1e-4, 7, 1.0, 1, False, 0.0, False),
    ("poisson", "nearest", "mixed", 1e-4, 7, 1.0, 1, False, 0.0, False),
    ("gauss", "nearest", "mixed", 1e-4, 7, 1.0, 1, False, 0.0, False),
    ("poisson", "trilinear", "mixed", 1e-4, 7, 1.0, 1, False, 0.0, False),
    ("poisson", "nearest", "mixed", 1e-4, 12, 0.6, 1, False, 0.0, False),
    ("poisson", "nearest", "mixed", 1e-4, 12, 0.7, 3, False, 0.0, False),
    ("poisson", "nearest", "mixed", 1e-4, 12, 0.7, 3, True, 0.0, False),
    ("poisson", "nearest", "mixed", 1e-4, 12, 0.5, 2, True, 1.1, False),
    ("poisson", "nearest", "mixed", 1e-4, 7, 1.0, 1, False, 0.0, True),
    ("poisson", "nearest", "mixed", 1e-4, 12, 0.5, 2, True, 1.1, True),
])
def test_proposed_iteration_matches_restricted_oracle(lik, interp, prec, tol, max_cells,
                                                      mass_target, min_cells, keep, keep_mass,
                                                      pair):
    """One proposed iteration (the top cells of 60 uneven cells per pattern:
    a fixed 7, adaptive up to a predicted mass of 0.6, at least 3 and then up
    to 0.7, the 3 top cells of a second posterior first, or that posterior's
    cells up to a mass of 1.1 first; pair: the grouped maximize on SM pairs)
    against the FP64 oracle's iteration restricted to the same candidate
    rotations."""
    import torch
    from emc_b200 import workloads as W
    from emc_b200.proposal import LearnedProposal
    from oracle import oracle as O
    from parity import oracle_cfg
    case = _proposal_case(W.make("tiny16"), max_cells, mass_target, min_cells=min_cells, keep=keep,
                          keep_mass=keep_mass)
    d, cell, n_cells, probs, allowed = case[:5]
    kp = torch.from_numpy(case[5]).cuda() if keep else None
    cfg = oracle_cfg(d, lik, interp)
    m_ref, s_ref, P_ref, st_ref = O.iterate(cfg, d["counts"], d["mask"], d["q"], d["w"], d["x"],
                                            d["y"], d["z"], d["model0"].astype(np.float64),
                                            d["scaling0"].astype(np.float64), want_resp=True,
                                            allowed=allowed)
    t_ref = np.zeros((P_ref.shape[1], n_cells))
    np.add.at(t_ref.T, cell, P_ref)  # responsibility mass per (pattern, cell)
    with make_ctx(d, lik, interp, prec) as ctx:
        if pair:
            ctx.set_tuning(1, 6, 1, 0)
        lp = LearnedProposal(ctx, cell, n_cells, bf16=True)
        st = lp.iterate(torch.from_numpy(probs).cuda(), max_cells, mass_target, threshold=0.0,
                        min_cells=min_cells, keep=kp, keep_mass=keep_mass)
        assert st["fallback"] == 0
        assert st["evaluations"] == int(allowed.sum())
        assert rel(ctx.get_scaling(), s_ref) <= tol, rel(ctx.get_scaling(), s_ref)
        assert rel(ctx.get_model(), m_ref) <= tol, rel(ctx.get_model(), m_ref)
        assert abs(st["sum_plogp"] - st_ref["sum_plogp"]) <= 1e-3 * abs(st_ref["sum_plogp"]) + 1e-3
        assert abs(st["total_loglik"] - st_ref["total_loglik"]) <= 1e-5 * abs(st_ref["total_loglik"])
        t = lp.targets().cpu().numpy()
        assert np.abs(t - t_ref).max() <= 1e-3


def test_proposed_iteration_with_every_cell_is_the_dense_iteration():
    import torch
    from emc_b200 import workloads as W
    from emc_b200.proposal import LearnedProposal
    d, cell, n_cells, probs, _ = _proposal_case(W.make("tiny16"), 60)
    with make_ctx(d, "poisson", "nearest", "mixed") as ctx:
        m0, s0 = ctx.get_model(), ctx.get_scaling()
        ctx.iterate()
        m_dense, s_dense = ctx.get_model(), ctx.get_scaling()
        ctx.set_model(m0)
        ctx.set_scaling(s0)
        lp = LearnedProposal(ctx, cell, n_cells)
        st = lp.iterate(torch.from_numpy(probs).cuda(), n_cells, threshold=0.0)
        assert st["evaluations"] == ctx.N * ctx.R
        assert rel(ctx.get_model(), m_dense) <= 1e-4
        assert rel(ctx.get_scaling(), s_dense) <= 1e-4


def _select_topk(probs, log_keep, mcnt, top_k, m, mass_target, keep_tail=0.0):
    """The candidate cells emc_iterate_topk takes: cells in order of log_keep
    (finite values) until they hold at least top_k fine rotations and (with
    keep_tail) all but keep_tail of exp(log_keep), then cells in order of
    probs until the (FP32) probs total of all taken cells reaches mass_target
    (at least one cell), at most m."""
    N, n_cells = (probs if probs is not None else log_keep).shape
    sel = np.zeros((N, n_cells), bool)
    for p in range(N):
        tot, n, covered, held = np.float32(0), 0, 0, 0.0
        if log_keep is not None:
            for k in np.argsort(-log_keep[p], kind="stable"):
                if n >= m or not log_keep[p, k] > -np.inf:
                    break
                if covered >= top_k and not (keep_tail > 0 and held < 1.0 - keep_tail):
                    break
                sel[p, k] = True
                n += 1
                covered += mcnt[k]
                held += float(np.exp(np.float64(log_keep[p, k])))
                if probs is not None:
                    tot = np.float32(tot + max(probs[p, k], np.float32(0)))
        if probs is not None:
            for k in np.argsort(-probs[p], kind="stable"):
                if n >= m or (n > 0 and tot >= np.float32(mass_target)):
                    break
                if sel[p, k]:
                    continue
                sel[p, k] = True
                n += 1
                tot = np.float32(tot + max(probs[p, k], np.float32(0)))
    return sel


@pytest.mark.parametrize("prec,use_probs,use_keep,tol,tail", [
    ("fp32", True, True, 1e-5, 0.0), ("mixed", True, True, 1e-4, 0.0),
    ("mixed", False, True, 1e-4, 0.0), ("mixed", True, False, 1e-4, 0.0),
    ("mixed", False, True, 1e-4, 1e-3)])
def test_topk_iteration_matches_restricted_oracle(prec, use_probs, use_keep, tol, tail):
    """emc_iterate_topk (cells holding each pattern's best previous
    log-posterior until 20 fine rotations are covered, then network cells up
    to a predicted mass of 0.6, at most 9 of 60 uneven cells) against the
    FP64 oracle restricted to the same candidates: model, scaling, the
    exported responsibilities, and the log cell masses of the iteration."""
    import torch

    import emc_b200 as E
    from emc_b200 import workloads as W
    from emc_b200.proposal import LearnedProposal, sorted_rotations
    from oracle import oracle as O
    from parity import oracle_cfg, resp_l1
    d = W.make("tiny16")
    q, w, cell, n_cells = sorted_rotations(d["q"], d["w"], coarse_n=1)
    d = dict(d, q=q, w=w)
    N = d["counts"].shape[0]
    mcnt = np.bincount(cell, minlength=n_cells)
    rng = np.random.default_rng(5)
    z = rng.standard_normal((N, n_cells)) * 2.0
    probs = np.exp(z - z.max(1, keepdims=True))
    probs = (probs / probs.sum(1, keepdims=True)).astype(np.float32)
    z = rng.standard_normal((N, n_cells)) * 3.0
    z[rng.random((N, n_cells)) < 0.6] = -np.inf
    z[:, 0] = np.maximum(z[:, 0], -5.0)
    lk = (z - np.log(np.exp(z).sum(1, keepdims=True))).astype(np.float32)  # log-posterior
    lk[:2] = -np.inf  # patterns with no previous posterior at all
    if not use_probs:
        lk[:2, 0] = 0.0
    sel = _select_topk(probs if use_probs else None, lk if use_keep else None, mcnt, 20, 9, 0.6,
                       tail)
    allowed = sel[:, cell].T.astype(np.uint8)
    cfg = oracle_cfg(d, "poisson", "nearest")
    m_ref, s_ref, P_ref, st_ref = O.iterate(cfg, d["counts"], d["mask"], d["q"], d["w"], d["x"],
                                            d["y"], d["z"], d["model0"], d["scaling0"],
                                            want_resp=True, allowed=allowed)
    t_ref = np.zeros((N, n_cells))
    np.add.at(t_ref.T, cell, P_ref)
    with make_ctx(d, "poisson", "nearest", prec) as ctx:
        lp = LearnedProposal(ctx, cell, n_cells)
        st = lp.iterate_topk(torch.from_numpy(probs).cuda() if use_probs else None,
                             torch.from_numpy(lk).cuda() if use_keep else None, top_k=20,
                             max_cells=9, mass_target=0.6, keep_tail=tail)
        assert st["fallback"] == 0 and st["audited"] == 0
        assert st["evaluations"] == int(allowed.sum()) and st["pairs"] == int(sel.sum())
        assert rel(ctx.get_model(), m_ref) <= tol, rel(ctx.get_model(), m_ref)
        assert rel(ctx.get_scaling(), s_ref) <= tol
        P = ctx.get_buffer(E.BUF_RESP)
        assert resp_l1(P, P_ref) <= 10 * tol, resp_l1(P, P_ref)
        assert (P[allowed == 0] == 0).all()
        lm = lp.log_mass().cpu().numpy()
        assert np.isneginf(lm[~sel]).all()
        big = t_ref > 1e-30
        assert np.abs(lm[big] - np.log(t_ref[big])).max() <= 1e-2


@pytest.mark.parametrize("coarse_n", [1, 2])
def test_grouped_forms_agree(coarse_n):
    """The grouped maximize on SM pairs and on one SM, each with the compress
    from responsibility lists and with the grouped tensor-core compress, give
    the same scaling and model; 60 or 420 uneven cells, ragged slot counts
    (301 patterns)."""
    import torch

    from emc_b200 import workloads as W
    from emc_b200.proposal import LearnedProposal, sorted_rotations
    d = W.make("tiny16", n_patterns=301)
    q, w, cell, n_cells = sorted_rotations(d["q"], d["w"], coarse_n=coarse_n)
    d = dict(d, q=q, w=w)
    N = d["counts"].shape[0]
    rng = np.random.default_rng(11)
    z = rng.standard_normal((N, n_cells)) * 2.0
    probs = np.exp(z - z.max(1, keepdims=True))
    probs = torch.from_numpy((probs / probs.sum(1, keepdims=True)).astype(np.float32)).cuda()
    out = {}
    for pair in (1, 0):
        for lists in (True, False):
            with make_ctx(d, "poisson", "nearest", "mixed") as ctx:
                ctx.set_tuning(1, 6, pair, 0)
                ctx.set_sparse_compress(lists)
                lp = LearnedProposal(ctx, cell, n_cells)
                st = lp.iterate_topk(probs, None, top_k=1, max_cells=9, mass_target=0.8)
                assert st["fallback"] == 0
                out[pair, lists] = (ctx.get_model(), ctx.get_scaling(), st["pairs"])
    ref = out[1, True]
    for key, (m, phi, pairs) in out.items():
        assert pairs == ref[2]
        assert rel(phi, ref[1]) <= 1e-6, (key, rel(phi, ref[1]))
        assert rel(m, ref[0]) <= 1e-5, (key, rel(m, ref[0]))


@pytest.mark.parametrize("prec", ["fp32", "mixed"])
def test_log_mass_of_a_dense_iteration(prec):
    """emc_cell_log_mass after a dense maximize: log of the oracle's per-cell
    responsibility mass, down the tail (cells with mass > 1e-200)."""
    from emc_b200 import workloads as W
    from emc_b200.proposal import LearnedProposal, sorted_rotations
    from oracle import oracle as O
    from parity import oracle_cfg
    d = W.make("tiny16")
    q, w, cell, n_cells = sorted_rotations(d["q"], d["w"], coarse_n=1)
    d = dict(d, q=q, w=w)
    cfg = oracle_cfg(d, "poisson", "nearest")
    _, _, P_ref, _ = O.iterate(cfg, d["counts"], d["mask"], d["q"], d["w"], d["x"], d["y"],
                               d["z"], d["model0"], d["scaling0"], want_resp=True)
    t_ref = np.zeros((d["counts"].shape[0], n_cells))
    np.add.at(t_ref.T, cell, P_ref)
    with make_ctx(d, "poisson", "nearest", prec) as ctx:
        lp = LearnedProposal(ctx, cell, n_cells)
        ctx.iterate()
        lm = lp.log_mass().cpu().numpy()
    big = t_ref > 1e-200
    err = np.abs(lm[big] - np.log(t_ref[big]))
    # relative errors of tail masses follow the log-likelihood's absolute error
    assert err.max() <= (2e-3 if prec == "fp32" else 5e-2), err.max()
    assert big.sum() > 0.5 * big.size


@pytest.mark.parametrize("prec", ["fp32", "mixed"])
def test_audit_triggers_the_dense_fallback(prec):
    """With candidates drawn from the previous iteration's log-posterior, the
    audited patterns keep their responsibility and the grouped stages run;
    with every pattern handed another pattern's cells, the audit sees the
    responsibility outside the candidates and the dense iteration runs (same
    model as emc_iterate)."""
    import torch
    from emc_b200 import workloads as W
    from emc_b200.proposal import LearnedProposal, sorted_rotations
    d = W.make("b200_64", n_patterns=600)
    q, w, cell, n_cells = sorted_rotations(d["q"], d["w"], coarse_n=2)
    d = dict(d, q=q, w=w)
    with make_ctx(d, "poisson", "nearest", prec) as ctx:
        lp = LearnedProposal(ctx, cell, n_cells)
        for _ in range(3):
            ctx.iterate()
        lk = lp.log_mass()
        m0, s0 = ctx.get_model(), ctx.get_scaling()
        ctx.iterate()
        m_dense = ctx.get_model()
        ctx.set_model(m0)
        ctx.set_scaling(s0)
        st = lp.iterate_topk(None, lk, top_k=512, max_cells=16, audit=64, min_captured=0.99)
        assert st["fallback"] == 0 and st["audited"] == 64, st
        assert st["audit_min_captured"] >= 0.99, st
        assert rel(ctx.get_model(), m_dense) < 1e-3
        ctx.set_model(m0)
        ctx.set_scaling(s0)
        wrong = torch.roll(lk, shifts=1, dims=0)  # pattern p gets pattern p-1's cells
        st = lp.iterate_topk(None, wrong, top_k=512, max_cells=16, audit=64, min_captured=0.99)
        assert st["fallback"] == 1 and st["audit_min_captured"] < 0.99, st
        assert rel(ctx.get_model(), m_dense) < 1e-5


def test_topk_at_the_large_geometry_holds_the_bar_against_the_dense_fp64_oracle():
    """The 128^3 benchmark geometry (16,272 active pixels, 500 photons, ~3%
    non-zero pixels) on every 43rd of its 86,520 rotations (2,013, sorted
    into the 60 cells of the n=1 sampling) and 384 patterns: after two dense
    iterations, one top-k proposed iteration (512 fine rotations from the
    previous log-posterior, 64 patterns audited) against the oracle's DENSE
    iteration from the same state: per-pattern responsibility L1 <= 1e-2 and
    model error <= 1e-3 (the mixed path's own error included)."""
    import emc_b200 as E
    from emc_b200 import workloads as W
    from emc_b200.proposal import LearnedProposal, sorted_rotations
    from oracle import oracle as O
    from parity import oracle_cfg, resp_l1
    d = W.make("large128", n_patterns=384)
    rot = np.arange(0, d["q"].shape[0], 43)
    q, w, cell, n_cells = sorted_rotations(d["q"][rot], d["w"][rot], coarse_n=1)
    d = dict(d, q=q, w=w)
    with make_ctx(d, "poisson", "nearest", "mixed") as ctx:
        lp = LearnedProposal(ctx, cell, n_cells)
        ctx.iterate()
        ctx.iterate()
        lk = lp.log_mass()
        m0, s0 = ctx.get_model(), ctx.get_scaling()
        st = lp.iterate_topk(None, lk, top_k=512, max_cells=n_cells, audit=64, min_captured=0.99)
        P = ctx.get_buffer(E.BUF_RESP)
        cols = ctx.resp_columns([0, 5, 383])
        np.testing.assert_array_equal(cols, P[:, [0, 5, 383]])
        model = ctx.get_model()
    cfg = oracle_cfg(d, "poisson")
    m_ref, _, P_ref, _ = O.iterate(cfg, d["counts"], d["mask"], d["q"], d["w"], d["x"], d["y"],
                                   d["z"], m0, s0, want_resp=True)
    err_p, err_m = resp_l1(P, P_ref), rel(model, m_ref)
    print(f"top-k at 128^3 ({st['pairs'] / 384:.1f} cells, "
          f"{st['evaluations'] / 384:.0f} rotations per pattern of {len(q)}; audit min captured "
          f"{st['audit_min_captured']:.6f}): responsibility L1 {err_p:.3g}, model {err_m:.3g} "
          f"vs the dense FP64 oracle")
    assert st["fallback"] == 0
    assert err_p <= 1e-2 and err_m <= 1e-3


@pytest.mark.parametrize("prec", ["fp32", "mixed"])
def test_resp_columns_match_the_full_export(prec):
    import emc_b200 as E
    from emc_b200 import workloads as W
    d = W.make("tiny16")
    with make_ctx(d, "poisson", "nearest", prec) as ctx:
        ctx.expand()
        ctx.maximize()
        cols = ctx.resp_columns([3, 0, 63, 3])
        P = ctx.get_buffer(E.BUF_RESP)
        np.testing.assert_array_equal(cols, P[:, [3, 0, 63, 3]])
        with pytest.raises(E.EmcError):
            ctx.resp_columns([64])
