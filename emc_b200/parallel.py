"""Pattern-sharded EMC across ranks (one process per GPU).

An EMC iteration is per pattern everywhere except insertion: every rank
expands the same model against the same rotations, evaluates its own patterns
(responsibilities, scaling), and inserts their slice averages into its own
accumulators.  The exchanges are the element-wise sums of those
accumulators -- 2 x side^3 floats, model and weight sums -- before
normalisation, and of the R per-rotation responsibility totals that decide
which rotations the insertion skips; the ranks then normalise identical sums and hold identical
models.  The reference is single-GPU; patterns are the natural unit to
shard, and this costs one all-reduce per iteration.

The per-iteration statistics (sum P log P, sum of log-sum-exps) are sums over
patterns and are reduced the same way.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def shard_range(n_total: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous, balanced (first pattern, count) of rank's share."""
    base, extra = divmod(n_total, world)
    count = base + (1 if rank < extra else 0)
    first = rank * base + min(rank, extra)
    return first, count


class ShardedIteration:
    """Drives one EMC iteration over a pattern shard and sums the insertion
    accumulators across the process group.

    `ctx` is an emc_b200.Context (or any object with the same stage methods:
    expand, maximize, compress_insert, accumulator_tensor, synchronize,
    normalize, partial_stats)."""

    def __init__(self, ctx, group=None):
        self.ctx = ctx
        self.group = group

    def _sum(self, t) -> None:
        c = self.ctx
        if t.is_cuda:
            # enqueued on the library's stream: it waits for the stage that
            # wrote t, and the next stage (enqueued after it) waits for it
            with torch.cuda.stream(torch.cuda.ExternalStream(c.stream)):
                dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        else:
            c.synchronize()
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)

    def __call__(self) -> None:
        c = self.ctx
        sharded = dist.is_initialized() and dist.get_world_size(self.group) > 1
        c.expand()
        c.maximize()
        if sharded:
            # the insertion skips rotations whose total responsibility over
            # ALL patterns is <= 1e-10 (emc_atomic.cu:128): sum T_r first
            self._sum(c.total_resp_all_tensor())
        c.compress_insert()
        if sharded:
            self._sum(c.accumulator_tensor())
        c.normalize()

    def stats(self) -> dict:
        plogp, loglik = self.ctx.partial_stats()
        t = torch.tensor([plogp, loglik], dtype=torch.float64)
        if dist.is_initialized() and dist.get_world_size(self.group) > 1:
            backend = dist.get_backend(self.group)
            if backend == "nccl":
                t = t.cuda()
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
            t = t.cpu()
        return {"sum_plogp": float(t[0]), "total_loglik": float(t[1])}
