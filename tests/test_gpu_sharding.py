"""Pattern sharding on the GPU: two contexts holding the two halves of a
dataset, their insertion accumulators summed between compress and
normalisation, reproduce the single-context iteration; and the NCCL
all-reduce of the accumulator view runs on the library's stream."""
import numpy as np
import pytest

from parity import make_ctx, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["mixed", "fp32"])
def test_two_shards_equal_one_context(prec):
    import torch
    from emc_b200 import workloads as W
    w = W.WORKLOADS["small32"]
    full = W.make(w)
    N = full["counts"].shape[0]
    halves = [W.make(w, n_patterns=N // 2, first_pattern=k * (N // 2)) for k in (0, 1)]
    np.testing.assert_array_equal(np.concatenate([h["counts"] for h in halves]), full["counts"])
    with make_ctx(full, "poisson", "nearest", prec) as c:
        c.iterate()
        m_ref, s_ref = c.get_model(), c.get_scaling()
    ctxs = [make_ctx(h, "poisson", "nearest", prec) for h in halves]
    try:
        for c in ctxs:
            c.expand()
            c.maximize()
            c.synchronize()
        # the insertion's skip test reads T_r summed over both shards
        ts = [c.total_resp_all_tensor() for c in ctxs]
        t_all = ts[0] + ts[1]
        torch.cuda.synchronize()
        for t in ts:
            t.copy_(t_all)
        torch.cuda.synchronize()
        for c in ctxs:
            c.compress_insert()
            c.synchronize()
        accs = [c.accumulator_tensor() for c in ctxs]
        total = accs[0] + accs[1]
        torch.cuda.synchronize()
        for a in accs:
            a.copy_(total)
        torch.cuda.synchronize()
        for c in ctxs:
            c.normalize()
        for c in ctxs:
            assert rel(c.get_model(), m_ref) < 1e-5, rel(c.get_model(), m_ref)
        s = np.concatenate([c.get_scaling() for c in ctxs])
        assert rel(s, s_ref) < 1e-6
    finally:
        for c in ctxs:
            c.close()


def test_nccl_allreduce_of_the_accumulators_single_rank():
    import os
    import torch
    import torch.distributed as dist
    from emc_b200 import workloads as W
    from emc_b200.parallel import ShardedIteration
    if not dist.is_nccl_available():
        pytest.skip("NCCL not available")
    d = W.make("tiny16")
    with make_ctx(d, "poisson", "nearest", "mixed") as c:
        c.iterate()
        m_ref = c.get_model()
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ.setdefault("MASTER_PORT", "29533")
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        with make_ctx(d, "poisson", "nearest", "mixed") as c:
            c.expand()
            c.maximize()
            c.compress_insert()
            c.synchronize()
            acc = c.accumulator_tensor()
            before = acc.clone()
            torch.cuda.synchronize()
            with torch.cuda.stream(torch.cuda.ExternalStream(c.stream)):
                dist.all_reduce(acc, op=dist.ReduceOp.SUM)
            torch.cuda.synchronize()
            assert torch.equal(acc, before)  # one rank: the sum is the input
            c.normalize()
            assert rel(c.get_model(), m_ref) < 1e-5
            st = ShardedIteration(c)
            st()
            assert np.isfinite(st.stats()["sum_plogp"])
    finally:
        dist.destroy_process_group()
