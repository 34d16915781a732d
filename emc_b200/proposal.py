"""Learned rotation proposal: host-side orchestration.

Fine rotations are grouped into coarse cells (nearest rotation of a coarse
600-cell sampling, 420 rotations for n = 2); the proposal network (emc_net,
CUDA kernels in emc_b200/csrc/net.cu) learns to predict, from a pattern's
2x-downsampled log(1 + K), the posterior over cells that dense EMC
iterations produce; emc_iterate_proposed then evaluates each pattern only
against the fine rotations of its candidate cells (those holding most of its
responsibility in the previous iteration, then the network's most probable
ones), with the dense iteration as the fallback.  torch provides device
buffers only.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import Context, _check, _ptr, generate_rotations, lib

_bound = False


def _bind():
    global _bound
    if _bound:
        return
    L = lib()
    P, I64 = C.c_void_p, C.c_int64
    for name, args, res in [
        ("emc_set_cells", [P, P, C.c_int32], C.c_int),
        ("emc_pattern_features", [P, C.c_int32, P], C.c_int),
        ("emc_cell_targets", [P, P], C.c_int),
        ("emc_iterate_proposed",
         [P, P, P, C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_float, P], C.c_int),
        ("emc_net_create", [C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int, P], C.c_int),
        ("emc_net_destroy", [P], C.c_int),
        ("emc_net_num_params", [P], I64),
        ("emc_net_get_params", [P, P], C.c_int),
        ("emc_net_set_params", [P, P], C.c_int),
        ("emc_net_forward", [P, P, I64, P], C.c_int),
        ("emc_net_gradients", [P, P, P, I64, P, P], C.c_int),
        ("emc_net_train_step", [P, P, P, I64, C.c_float, P], C.c_int),
        ("emc_net_last_error", [P], C.c_char_p),
        ("emc_iterate_topk", [P, P, P, P, P], C.c_int),
        ("emc_cell_log_mass", [P, P], C.c_int),
    ]:
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _bound = True


class ProposalStats(C.Structure):
    _fields_ = [("mean_mass", C.c_double), ("min_mass", C.c_double), ("pairs", C.c_int64),
                ("evaluations", C.c_int64), ("fallback", C.c_int32), ("audited", C.c_int32),
                ("sum_plogp", C.c_double), ("total_loglik", C.c_double),
                ("audit_mean_captured", C.c_double), ("audit_min_captured", C.c_double)]


class TopkConfig(C.Structure):
    _fields_ = [("top_k", C.c_int32), ("max_cells", C.c_int32), ("mass_target", C.c_float),
                ("audit_patterns", C.c_int32), ("min_captured", C.c_float),
                ("keep_tail", C.c_float)]


def assign_cells(q_fine, q_coarse, chunk=8192):
    """Nearest coarse rotation of every fine rotation (|<q, q'>| largest: q and
    -q are the same rotation)."""
    q_fine = np.asarray(q_fine, np.float64)
    q_coarse = np.asarray(q_coarse, np.float64)
    out = np.empty(len(q_fine), np.int32)
    for i in range(0, len(q_fine), chunk):
        out[i:i + chunk] = np.argmax(np.abs(q_fine[i:i + chunk] @ q_coarse.T), axis=1)
    return out


def sorted_rotations(q, w, coarse_n=2):
    """(q, w, cell, n_cells) with the fine rotations sorted by their coarse cell."""
    qc, _ = generate_rotations(coarse_n)
    cell = assign_cells(q, qc)
    perm = np.argsort(cell, kind="stable")
    return (np.ascontiguousarray(q[perm]), np.ascontiguousarray(w[perm]),
            np.ascontiguousarray(cell[perm]), len(qc))


class ProposalNet:
    """The network of emc_b200/csrc/net.cu (BF16, or FP32 with bf16=False)."""

    def __init__(self, in_side, n_out, bf16=True, seed=0, device=0):
        _bind()
        h = C.c_void_p()
        _check(lib().emc_net_create(in_side, n_out, int(bf16), seed, device, C.byref(h)))
        self._h, self.in_side, self.n_out = h, in_side, n_out

    def close(self):
        if getattr(self, "_h", None):
            lib().emc_net_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, st):
        if st != 0:
            from . import EmcError
            raise EmcError(st, lib().emc_net_last_error(self._h).decode())

    @property
    def num_params(self):
        return int(lib().emc_net_num_params(self._h))

    def get_params(self):
        p = np.zeros(self.num_params, np.float32)
        self._c(lib().emc_net_get_params(self._h, _ptr(p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        self._c(lib().emc_net_set_params(self._h, _ptr(p)))

    def forward(self, x):
        """x: CUDA float32 tensor [B][in_side^2] -> probs [B][n_out]."""
        import torch
        torch.cuda.synchronize()
        probs = torch.empty((x.shape[0], self.n_out), dtype=torch.float32, device=x.device)
        self._c(lib().emc_net_forward(self._h, x.data_ptr(), x.shape[0], probs.data_ptr()))
        return probs

    def gradients(self, x, t):
        import torch
        torch.cuda.synchronize()
        g = np.zeros(self.num_params, np.float32)
        loss = C.c_double()
        self._c(lib().emc_net_gradients(self._h, x.data_ptr(), t.data_ptr(), x.shape[0],
                                        C.byref(loss), _ptr(g)))
        return loss.value, g

    def train_step(self, x, t, lr):
        import torch
        torch.cuda.synchronize()
        loss = C.c_double()
        self._c(lib().emc_net_train_step(self._h, x.data_ptr(), t.data_ptr(), x.shape[0], lr,
                                         C.byref(loss)))
        return loss.value


class LearnedProposal:
    """Features, targets, training and prediction for one Context whose
    rotations are sorted by cell (see sorted_rotations)."""

    def __init__(self, ctx: Context, cell, n_cells, bf16=True, seed=0, device=0):
        _bind()
        self.ctx, self.n_cells = ctx, n_cells
        self.in_side = ctx.side // 2
        cell = np.ascontiguousarray(cell, np.int32)
        ctx._c(lib().emc_set_cells(ctx._h, _ptr(cell), n_cells))
        self.net = ProposalNet(self.in_side, n_cells, bf16=bf16, seed=seed, device=device)

    def features(self):
        import torch
        x = torch.empty((self.ctx.N, self.in_side ** 2), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        self.ctx._c(lib().emc_pattern_features(self.ctx._h, self.in_side, x.data_ptr()))
        return x

    def targets(self):
        """Cell posterior of the last maximize (dense, or proposed: 0 outside
        the candidate cells), [N][n_cells]."""
        import torch
        t = torch.empty((self.ctx.N, self.n_cells), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        self.ctx._c(lib().emc_cell_targets(self.ctx._h, t.data_ptr()))
        return t

    def train(self, x, t, epochs=10, batch=256, lr=2e-3, seed=0):
        import torch
        g = torch.Generator(device="cpu").manual_seed(seed)
        losses = []
        n = x.shape[0]
        for ep in range(epochs):
            perm = torch.randperm(n, generator=g).cuda()
            tot, cnt = 0.0, 0
            for i in range(0, n - batch + 1, batch):
                idx = perm[i:i + batch]
                xb, tb = x[idx].contiguous(), t[idx].contiguous()
                tot += self.net.train_step(xb, tb, lr) * batch
                cnt += batch
            losses.append(tot / max(cnt, 1))
        return losses

    def predict(self, x, batch=2048):
        import torch
        out = torch.empty((x.shape[0], self.n_cells), dtype=torch.float32, device="cuda")
        for i in range(0, x.shape[0], batch):
            out[i:i + batch] = self.net.forward(x[i:i + batch].contiguous())
        torch.cuda.synchronize()
        return out

    def iterate(self, probs, max_cells, mass_target=1.0, threshold=0.99, min_cells=1, keep=None,
                keep_mass=0.0):
        """One proposed iteration (emc_iterate_proposed).  Per pattern: with
        `keep` (e.g. the previous iteration's `targets()`) first its most
        probable cells under keep until at least min_cells are taken and their
        keep mass reaches keep_mass; then the most probable cells under
        `probs` until at least min_cells are taken and their predicted mass
        reaches mass_target, at most max_cells.  The dense iteration runs
        instead when the mean predicted mass is below threshold.  Returns the
        iteration's statistics as a dict."""
        import torch
        if keep is not None:
            if tuple(keep.shape) != tuple(probs.shape) or keep.dtype != torch.float32:
                raise ValueError("keep must be a float32 tensor shaped like probs")
            keep = keep.contiguous()
        torch.cuda.synchronize()
        st = ProposalStats()
        self.ctx._c(lib().emc_iterate_proposed(self.ctx._h, probs.data_ptr(),
                                               None if keep is None else keep.data_ptr(),
                                               int(min_cells), int(max_cells), mass_target,
                                               keep_mass, threshold, C.byref(st)))
        return {k: getattr(st, k) for k, _ in ProposalStats._fields_}

    def log_mass(self):
        """Log-posterior mass of every cell in the last maximize (dense, or
        proposed: -inf outside the candidate cells), [N][n_cells]."""
        import torch
        t = torch.empty((self.ctx.N, self.n_cells), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        self.ctx._c(lib().emc_cell_log_mass(self.ctx._h, t.data_ptr()))
        return t

    def iterate_topk(self, probs=None, log_keep=None, top_k=512, max_cells=32, mass_target=0.999,
                     audit=0, min_captured=0.99, keep_tail=0.0):
        """One proposed iteration of emc_iterate_topk: per pattern the cells
        holding the best of its previous log-posterior until they hold top_k
        fine rotations (log_keep, e.g. log_mass() of the previous iteration),
        then the network's most probable cells up to a predicted mass of
        mass_target (probs), at most max_cells (with keep_tail > 0 the
        log_keep cells continue until they hold all but keep_tail of the
        previous posterior); `audit` sampled patterns are
        evaluated against every rotation and the dense iteration runs when one
        of them holds less than min_captured of its responsibility."""
        import torch
        for t in (probs, log_keep):
            if t is not None and (t.dtype != torch.float32 or tuple(t.shape) !=
                                  (self.ctx.N, self.n_cells)):
                raise ValueError("probs / log_keep must be float32 [N][n_cells] tensors")
        torch.cuda.synchronize()
        cfg = TopkConfig(int(top_k), int(max_cells), float(mass_target), int(audit),
                         float(min_captured), float(keep_tail))
        st = ProposalStats()
        self.ctx._c(lib().emc_iterate_topk(
            self.ctx._h, None if probs is None else probs.contiguous().data_ptr(),
            None if log_keep is None else log_keep.contiguous().data_ptr(), C.byref(cfg),
            C.byref(st)))
        return {k: getattr(st, k) for k, _ in ProposalStats._fields_}
