"""CPU checks of the host-side helpers the GPU paths rely on: photon-list
packing, the grouping of fine rotations into coarse cells, and the seeded
pattern sequence that pattern shards cut (no GPU needed)."""
import numpy as np


def test_photon_lists_round_trip():
    import emc_b200 as E
    rng = np.random.default_rng(3)
    K = rng.poisson(0.05, (7, 9 * 9)).astype(np.float32)
    K[2] = 0.0  # a pattern without photons
    K[5, :] = 0.0
    K[5, -1] = 4.0  # one photon pixel at the last column
    row_ptr, pix, cnt = E.photon_lists(K)
    assert row_ptr.dtype == np.int64 and pix.dtype == np.int32 and cnt.dtype == np.float32
    assert row_ptr[0] == 0 and row_ptr[-1] == len(pix) == len(cnt) == np.count_nonzero(K)
    assert row_ptr[3] == row_ptr[2]  # the empty row
    back = np.zeros_like(K)
    for p in range(K.shape[0]):
        s, e = row_ptr[p], row_ptr[p + 1]
        assert np.all(np.diff(pix[s:e]) > 0)  # ascending, no repeats
        back[p, pix[s:e]] = cnt[s:e]
    np.testing.assert_array_equal(back, K)


def test_sorted_rotations_group_each_rotation_with_its_nearest_cell():
    import emc_b200 as E
    from emc_b200.proposal import sorted_rotations
    q, w = E.generate_rotations(4)
    qc, _ = E.generate_rotations(2)
    qs, ws, cell, n_cells = sorted_rotations(q, w, coarse_n=2)
    assert n_cells == len(qc) and len(qs) == len(q)
    assert np.all(np.diff(cell) >= 0)  # sorted by cell
    # every rotation's cell is its nearest coarse rotation (q and -q alike)
    dots = np.abs(qs.astype(np.float64) @ qc.astype(np.float64).T)
    np.testing.assert_array_equal(dots[np.arange(len(qs)), cell], dots.max(1))
    # a permutation of the input, each weight staying with its rotation
    order = np.lexsort(q.T[::-1])
    order_s = np.lexsort(qs.T[::-1])
    np.testing.assert_array_equal(q[order], qs[order_s])
    np.testing.assert_array_equal(w[order], ws[order_s])


def test_pattern_shards_cut_one_seeded_sequence():
    """Pattern-sharded ranks build their slice with first_pattern: the
    slices of one seeded dataset are the rows of the whole one, and the
    model, mask and rotations do not depend on the slice."""
    from emc_b200 import workloads as W
    w = W.Workload("shard16", 16, 2, 12, 400.0, 0.3, 1.5, 1, seed=9)
    whole = W.make(w, n_patterns=12)
    a = W.make(w, n_patterns=5, first_pattern=0)
    b = W.make(w, n_patterns=7, first_pattern=5)
    np.testing.assert_array_equal(np.concatenate([a["counts"], b["counts"]]), whole["counts"])
    for k in ("mask", "q", "w", "model0", "true_model"):
        np.testing.assert_array_equal(a[k], whole[k])
        np.testing.assert_array_equal(b[k], whole[k])


def test_metrics_log_appends_one_record_per_iteration(tmp_path):
    import json

    from emc_b200.diagnostics import MetricsLog

    class FakeContext:  # what MetricsLog reads of a context
        N, R = 4, 10

        def get_scaling(self):
            return np.array([0.5, 1.0, 1.5, 2.0], np.float32)

    log = MetricsLog(str(tmp_path))
    stats = {"sum_plogp": -12.5, "total_loglik": -1.25e4, "model_max": 3.0, "total_resp": 4.0}
    log.record(1, FakeContext(), stats, seconds=0.5, stages_ms=[1, 2, 3, 4, 5],
               errors={"model_rel_err": 1e-5})
    log.record(2, FakeContext(), stats)
    lines = open(tmp_path / "metrics.jsonl").read().splitlines()
    assert len(lines) == 2
    a, b = (json.loads(x) for x in lines)
    assert a["iteration"] == 1 and b["iteration"] == 2
    assert a["total_loglik"] == -1.25e4 and a["sum_plogp"] == -12.5
    assert a["scaling"] == {"mean": 1.25, "min": 0.5, "max": 2.0}
    assert a["evals_per_s"] == 80.0 and a["stages_ms"] == [1, 2, 3, 4, 5]
    assert a["errors"] == {"model_rel_err": 1e-5}
    assert "evals_per_s" not in b and "stages_ms" not in b
