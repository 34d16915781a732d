"""Several datasets of different detector sizes iterated by one persistent
launch per contraction (emc_batch), directly and replayed as a CUDA graph,
against the same datasets iterated one by one."""
import numpy as np
import pytest

from parity import make_ctx, rel

pytestmark = pytest.mark.gpu


def _datasets():
    from emc_b200 import workloads as W
    ws = [W.Workload("b16", 16, 2, 64, 400.0, 0.3, 1.5, 1, seed=1),
          W.Workload("b24", 24, 3, 200, 600.0, 0.3, 2.0, 1, seed=2),
          W.Workload("b32", 32, 4, 300, 1000.0, 0.3, 2.0, 1, seed=3)]
    return [W.make(w) for w in ws]


@pytest.mark.parametrize("lists", [True, False])
def test_batched_iteration_matches_separate_iterations(lists):
    """With responsibility lists each dataset compresses from its own lists
    (their count kept on the device); without, the batched dense compress
    contraction covers them all."""
    import emc_b200 as E
    ds = _datasets()
    solo = [make_ctx(d, "poisson", "nearest", "mixed") for d in ds]
    for c in solo:
        c.set_sparse_compress(lists)
        c.iterate()
        c.iterate()
    refs = [(c.get_model(), c.get_scaling()) for c in solo]
    for c in solo:
        c.close()
    ctxs = [make_ctx(d, "poisson", "nearest", "mixed") for d in ds]
    try:
        for c in ctxs:
            c.set_sparse_compress(lists)
        with E.Batch(ctxs) as b:
            b.iterate()
            b.iterate()
            b.synchronize()
            for c, (m, s) in zip(ctxs, refs):
                assert rel(c.get_model(), m) < 1e-5, rel(c.get_model(), m)
                assert rel(c.get_scaling(), s) < 1e-5
            # stats and diagnostics of each dataset stay available
            o = ctxs[1].orientation_stats()
            assert o["avg_resp"].shape == (ctxs[1].R,)
    finally:
        for c in ctxs:
            c.close()


def test_overflowing_lists_fall_back_and_grow():
    """Lists started with room for 16 entries overflow in the first
    iteration: the gated dense compress runs instead, synchronize gives the
    lists room and records the graph again, and every iteration ends where
    the separate iterations do."""
    import emc_b200 as E
    ds = _datasets()
    # the same sequence one by one: the dense compress, then lists
    solo = [make_ctx(d, "poisson", "nearest", "mixed") for d in ds]
    refs = []
    for c in solo:
        ms = []
        for k in range(3):
            c.set_sparse_compress(k > 0)
            c.iterate()
            ms.append(c.get_model())
        refs.append(ms)
        c.close()
    ctxs = [make_ctx(d, "poisson", "nearest", "mixed") for d in ds]
    try:
        for c in ctxs:
            c.set_rotation_chunk(0, 16)
        with E.Batch(ctxs) as b:
            b.capture()
            b.launch(1)      # overflows: the dense compress
            b.synchronize()  # grows the lists, records the graph again
            for c, ms in zip(ctxs, refs):
                assert rel(c.get_model(), ms[0]) < 1e-5, rel(c.get_model(), ms[0])
            b.launch(1)
            b.synchronize()
            b.iterate()
            b.synchronize()
            for c, ms in zip(ctxs, refs):
                assert rel(c.get_model(), ms[2]) < 1e-5, rel(c.get_model(), ms[2])
    finally:
        for c in ctxs:
            c.close()


def test_graph_replay_matches_batched_iterations():
    import emc_b200 as E
    ds = _datasets()
    ctxs = [make_ctx(d, "gauss", "nearest", "mixed") for d in ds]
    try:
        with E.Batch(ctxs) as b:
            l_eager = [c.launch_count for c in ctxs]
            b.iterate()
            b.synchronize()
            l_eager = [c.launch_count - l for c, l in zip(ctxs, l_eager)]
            after1 = [c.get_model() for c in ctxs]
            for c, d in zip(ctxs, ds):
                c.set_model(d["model0"])
                c.set_scaling(d["scaling0"])
            b.capture()
            b.launch(1)
            b.synchronize()
            for c, m in zip(ctxs, after1):
                assert rel(c.get_model(), m) < 1e-5
            l0 = [c.launch_count for c in ctxs]
            b.launch(3)
            b.synchronize()
            # a replay counts the launches of an eager batched iteration
            assert [c.launch_count - l for c, l in zip(ctxs, l0)] == [3 * d for d in l_eager]
            for c in ctxs:
                m = c.get_model()
                assert np.isfinite(m).all() and abs(m.astype(np.float64).mean() - 1.0) < 1e-4
    finally:
        for c in ctxs:
            c.close()


def test_a_dataset_that_fills_the_gpu_keeps_its_own_launches():
    """A dataset whose maximize alone fills the persistent grid for eight
    waves (2,048 patterns x 25,680 rotations: 16 x 101 tiles) runs its own
    contraction launches inside the batch's graph, the other dataset the
    batched ones; both end where their separate iterations do."""
    import emc_b200 as E
    from emc_b200 import workloads as W
    ds = [W.make(W.Workload("b32r", 32, 8, 2048, 1000.0, 0.3, 2.0, 1, seed=4)),
          W.make(W.Workload("b16", 16, 2, 64, 400.0, 0.3, 1.5, 1, seed=1))]
    solo = [make_ctx(d, "poisson", "nearest", "mixed") for d in ds]
    for c in solo:
        c.iterate()
        c.iterate()
    refs = [(c.get_model(), c.get_scaling()) for c in solo]
    for c in solo:
        c.close()
    ctxs = [make_ctx(d, "poisson", "nearest", "mixed") for d in ds]
    try:
        with E.Batch(ctxs) as b:
            b.capture()
            l0, l1 = ctxs[0].launch_count, ctxs[1].launch_count
            b.launch(2)
            b.synchronize()
            # the same launches but for its own maximize and dense compress
            # (the other dataset's dense compress is its own too: lists), and
            # the batched maximize counted on the first context
            assert (ctxs[0].launch_count - l0) - (ctxs[1].launch_count - l1) == 2 * 2
            for c, (m, s) in zip(ctxs, refs):
                assert rel(c.get_model(), m) < 1e-5, rel(c.get_model(), m)
                assert rel(c.get_scaling(), s) < 1e-5
    finally:
        for c in ctxs:
            c.close()


def test_batch_rejects_fp32_contexts():
    import emc_b200 as E
    from emc_b200 import workloads as W
    d = W.make("tiny16")
    with make_ctx(d, "poisson", "nearest", "fp32") as c:
        with pytest.raises(E.EmcError):
            E.Batch([c])


def test_batched_pair_maximize_matches_separate_iterations():
    """Both batched contractions on SM pairs (chosen when the datasets that
    use pairs on their own hold most of the work) against one-by-one
    iterations."""
    import emc_b200 as E
    ds = _datasets()
    solo = [make_ctx(d, "poisson", "nearest", "mixed") for d in ds]
    for c in solo:
        c.iterate()
    refs = [c.get_model() for c in solo]
    for c in solo:
        c.close()
    ctxs = [make_ctx(d, "poisson", "nearest", "mixed") for d in ds]
    try:
        for c in ctxs:
            c.set_tuning(1, 2, 1, 1)
        with E.Batch(ctxs) as b:
            b.iterate()
            b.synchronize()
            for c, m in zip(ctxs, refs):
                assert rel(c.get_model(), m) < 1e-5, rel(c.get_model(), m)
    finally:
        for c in ctxs:
            c.close()


def test_single_dataset_iteration_as_a_graph():
    """The iteration of one dataset captured as one CUDA graph (a batch of
    one context) and replayed three times, against three eager iterations;
    both compress from responsibility lists, the graph's with their count
    read on the device."""
    import emc_b200 as E
    from emc_b200 import workloads as W
    d = W.make("small32")
    with make_ctx(d, "poisson", "nearest", "mixed") as c:
        for _ in range(3):
            c.iterate()
        ref_m, ref_s = c.get_model(), c.get_scaling()
    with make_ctx(d, "poisson", "nearest", "mixed") as c:
        with E.Batch([c]) as b:
            b.capture()
            b.launch(3)
            b.synchronize()
            assert rel(c.get_model(), ref_m) < 1e-5, rel(c.get_model(), ref_m)
            assert rel(c.get_scaling(), ref_s) < 1e-5
