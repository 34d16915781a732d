"""Host-side failure handling: inputs the engine cannot use are refused with a
status (and leave the context usable), a forced device-memory budget makes
allocations fail cleanly with EMC_ERR_OOM, and a checkpointed state resumes
the iteration where it stopped.  No GPU fault is provoked: every failure here
is made on the host."""
import os

import numpy as np
import pytest

from parity import make_ctx, rel

pytestmark = pytest.mark.gpu

ERR_ARG, ERR_OOM, ERR_STATE, ERR_RANGE = 1, 3, 5, 6


@pytest.fixture(scope="module")
def tiny():
    from emc_b200 import workloads as W
    return W.make("tiny16")


@pytest.mark.parametrize("prec", ["fp32", "mixed"])
def test_nonfinite_counts_are_refused(tiny, prec):
    import emc_b200 as E
    d = tiny
    bad = d["counts"].copy()
    bad[3, 40] = np.nan
    neg = d["counts"].copy()
    neg[1, 7] = -1.0
    with make_ctx(d, precision=prec) as ctx:
        for counts in (bad, neg):
            with pytest.raises(E.EmcError) as ei:
                ctx.set_patterns(counts)
            assert ei.value.status == ERR_RANGE
            # no patterns now: iterating is a state error, not a NaN model
            with pytest.raises(E.EmcError) as ei:
                ctx.iterate()
            assert ei.value.status == ERR_STATE
        ctx.set_patterns(d["counts"])
        ctx.iterate()
        assert np.isfinite(ctx.get_model()).all()


def test_nonfinite_model_scaling_rotations_geometry_are_refused(tiny):
    import emc_b200 as E
    d = tiny
    w = d["workload"]
    with make_ctx(d) as ctx:
        m = d["model0"].copy()
        m[5] = np.inf
        s = d["scaling0"].copy()
        s[2] = 0.0
        wt = d["w"].copy()
        wt[0] = -1.0
        q = d["q"].copy()
        q[4, 1] = np.nan
        for call in (lambda: ctx.set_model(m), lambda: ctx.set_scaling(s),
                     lambda: ctx.set_rotations(d["q"], wt), lambda: ctx.set_rotations(q, d["w"])):
            with pytest.raises(E.EmcError) as ei:
                call()
            assert ei.value.status == ERR_RANGE
        ctx.iterate()  # the refused calls changed nothing
        assert np.isfinite(ctx.get_model()).all()
    x = d["x"].copy()
    x[0] = np.nan
    ctx = E.Context(w.side, d["counts"].shape[0], d["q"].shape[0])
    with pytest.raises(E.EmcError) as ei:
        ctx.set_geometry(x, d["y"], d["z"], d["mask"])
    assert ei.value.status == ERR_RANGE
    ctx.close()


@pytest.mark.parametrize("prec", ["fp32", "mixed"])
def test_memory_budget_fails_cleanly(tiny, prec):
    """A budget smaller than the working set: the allocation that would pass
    it fails with EMC_ERR_OOM before calling cudaMalloc; destroying the
    context frees what it held."""
    import torch

    import emc_b200 as E
    d = tiny
    w = d["workload"]
    torch.cuda.synchronize()
    ctx = E.Context(w.side, d["counts"].shape[0], d["q"].shape[0], precision=prec)
    held = ctx.memory_used
    assert held > 0
    with pytest.raises(E.EmcError) as ei:
        ctx.set_memory_limit(held - 1)
    assert ei.value.status == ERR_ARG
    ctx.set_memory_limit(held + 4096)
    with pytest.raises(E.EmcError) as ei:
        ctx.set_geometry(d["x"], d["y"], d["z"], d["mask"])
    assert ei.value.status == ERR_OOM and "limit" in str(ei.value)
    assert ctx.memory_used <= held + 4096
    ctx.close()
    # the same context with room iterates normally
    with make_ctx(d, precision=prec) as ok:
        ok.iterate()


@pytest.mark.parametrize("prec", ["fp32", "mixed"])
def test_checkpoint_resume_continues_the_run(tiny, tmp_path, prec):
    """Two iterations, save, two more; a fresh context loaded from the file
    runs the same two iterations to the same model (insertion sums in a
    different order at most) and scaling."""
    import emc_b200 as E
    d = tiny
    path = os.path.join(tmp_path, "state.bin")
    with make_ctx(d, "poisson", precision=prec) as a:
        a.iterate()
        a.iterate()
        a.save_state(path, iteration=2)
        w2 = a.get_buffer(E.BUF_WEIGHT)
        a.iterate()
        a.iterate()
        m4, s4 = a.get_model(), a.get_scaling()
    with make_ctx(d, "poisson", precision=prec) as b:
        b.set_model(np.ones_like(d["model0"]))
        assert b.load_state(path) == 2
        np.testing.assert_array_equal(b.get_buffer(E.BUF_WEIGHT), w2)
        b.iterate()
        b.iterate()
        assert rel(b.get_model(), m4) < 1e-6
        assert rel(b.get_scaling(), s4) < 1e-6
    # a state of another shape, or a damaged file, is refused
    from emc_b200 import workloads as W
    other = W.make("tiny16", n_patterns=32)
    with make_ctx(other, "poisson", precision=prec) as c:
        with pytest.raises(E.EmcError) as ei:
            c.load_state(path)
        assert ei.value.status == ERR_RANGE
    with open(path, "r+b") as f:
        f.truncate(os.path.getsize(path) - 4)
    with make_ctx(d, "poisson", precision=prec) as c:
        with pytest.raises(E.EmcError) as ei:
            c.load_state(path)
        assert ei.value.status == ERR_RANGE


@pytest.mark.parametrize("prec", ["fp32", "mixed"])
def test_checkpoint_resume_is_bitwise_in_deterministic_mode(tiny, tmp_path, prec):
    """With the order-independent insertion sums, a run resumed from its
    checkpoint ends bitwise where the uninterrupted run does."""
    import emc_b200 as E
    d = tiny
    path = os.path.join(tmp_path, "state_det.bin")
    with make_ctx(d, "poisson", precision=prec) as a:
        a.set_deterministic(True)
        a.iterate()
        a.iterate()
        a.save_state(path, iteration=2)
        a.iterate()
        a.iterate()
        m4, s4, w4 = a.get_model(), a.get_scaling(), a.get_buffer(E.BUF_WEIGHT)
    with make_ctx(d, "poisson", precision=prec) as b:
        b.set_deterministic(True)
        assert b.load_state(path) == 2
        b.iterate()
        b.iterate()
        np.testing.assert_array_equal(b.get_model(), m4)
        np.testing.assert_array_equal(b.get_scaling(), s4)
        np.testing.assert_array_equal(b.get_buffer(E.BUF_WEIGHT), w4)
