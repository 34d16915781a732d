"""Pattern-sharded iteration (emc_b200.parallel) on 2 gloo ranks on CPU.

Each rank runs the FP64 oracle's stages on its half of the patterns through
ShardedIteration, whose all-reduce of the insertion accumulators is the only
exchange; the sharded model must equal the single-process oracle iteration
over all patterns (FP64, only the summation order differs)."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import oracle as O


class OracleShard:
    """Stage-by-stage stand-in of emc_b200.Context backed by the FP64 oracle."""

    def __init__(self, d, counts, scaling):
        w = d["workload"]
        self.d, self.K, self.scaling = d, counts, scaling.astype(np.float64)
        self.cfg = O.make_config(w.side, counts.shape[0], d["q"].shape[0])
        self.model = d["model0"].astype(np.float64)
        self.M = w.side ** 3

    def expand(self):
        d = self.d
        self.S = O.expand(self.cfg, self.model, d["q"], d["x"], d["y"], d["z"])

    def maximize(self):
        LL = O.loglik(self.cfg, self.S, self.K, self.d["mask"], self.scaling)
        self.P, lse, self.plogp = O.softmax(LL)
        self.loglik = float(lse.sum())
        self.scaling = O.update_scaling(self.cfg, self.S, self.K, self.d["mask"], self.P,
                                        self.scaling)
        self.T_all = torch.from_numpy(self.P.sum(axis=1))

    def total_resp_all_tensor(self):
        return self.T_all

    def compress_insert(self):
        d = self.d
        U, T = O.slice_average(self.cfg, self.P, self.K, d["mask"], self.scaling)
        acc_m, acc_w = O.insert(self.cfg, U, T, d["mask"], d["q"], d["w"], d["x"], d["y"], d["z"],
                                all_T=self.T_all.numpy())
        self.acc = torch.from_numpy(np.concatenate([acc_m, acc_w]))

    def accumulator_tensor(self):
        return self.acc

    def synchronize(self):
        pass

    def normalize(self):
        a = self.acc.numpy()
        self.model = O.normalize_model(a[: self.M], a[self.M:])

    def partial_stats(self):
        return self.plogp, self.loglik


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from emc_b200 import workloads as W
    from emc_b200.parallel import ShardedIteration, shard_range
    d = W.make("tiny16")
    first, n = shard_range(d["counts"].shape[0], rank, world)
    shard = OracleShard(d, d["counts"][first:first + n], d["scaling0"][first:first + n])
    it = ShardedIteration(shard)
    for _ in range(2):
        it()
    st = it.stats()
    if rank == 0:
        np.save(out, np.concatenate([shard.model, [st["sum_plogp"], st["total_loglik"]]]))
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_range_covers_everything():
    from emc_b200.parallel import shard_range
    for n, world in ((64, 2), (10, 3), (7, 8)):
        spans = [shard_range(n, r, world) for r in range(world)]
        assert sum(c for _, c in spans) == n
        assert all(spans[i][0] + spans[i][1] == spans[i + 1][0] for i in range(world - 1))


def test_sharded_iteration_equals_single_process(tmp_path):
    from emc_b200 import workloads as W
    out = str(tmp_path / "model.npy")
    mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    got = np.load(out)
    d = W.make("tiny16")
    cfg = O.make_config(d["workload"].side, d["counts"].shape[0], d["q"].shape[0])
    m, s = d["model0"].astype(np.float64), d["scaling0"].astype(np.float64)
    for _ in range(2):
        m, s, _, st = O.iterate(cfg, d["counts"], d["mask"], d["q"], d["w"], d["x"], d["y"], d["z"],
                                m, s)
    M = d["workload"].side ** 3
    np.testing.assert_allclose(got[:M], m, rtol=1e-12, atol=1e-12)
    assert abs(got[M] - st["sum_plogp"]) < 1e-9 * max(1.0, abs(st["sum_plogp"]))
    assert abs(got[M + 1] - st["total_loglik"]) < 1e-9 * max(1.0, abs(st["total_loglik"]))


class FailingShard(OracleShard):
    """A shard whose maximize raises: a rank that fails between collectives."""

    def maximize(self):
        raise RuntimeError("shard failed before the exchange")


def _failing_worker(rank, world, port, out_dir):
    import datetime
    import time
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=10))
    from emc_b200 import workloads as W
    from emc_b200.parallel import ShardedIteration, shard_range
    d = W.make("tiny16")
    first, n = shard_range(d["counts"].shape[0], rank, world)
    cls = FailingShard if rank == 1 else OracleShard
    it = ShardedIteration(cls(d, d["counts"][first:first + n], d["scaling0"][first:first + n]))
    t0 = time.monotonic()
    try:
        it()
        status = "completed"
    except Exception as e:  # noqa: BLE001 - the failure is what is recorded
        status = type(e).__name__
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
        f.write(f"{status} {time.monotonic() - t0:.2f}")
    # the failed rank leaves without joining any further collective
    os._exit(0)


def test_failed_rank_ends_the_others_collective_with_an_error(tmp_path):
    """Rank 1 raises before the responsibility-total all-reduce and leaves;
    rank 0's all-reduce must end with an error (the peer's exit or the
    10 s process-group timeout), not wait for ever."""
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_failing_worker, args=(r, 2, port, str(tmp_path)))
             for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive, "a rank did not finish"
    st0, t0 = open(tmp_path / "rank0.txt").read().split()
    st1, _ = open(tmp_path / "rank1.txt").read().split()
    assert st1 == "RuntimeError"
    assert st0 != "completed", st0
    assert float(t0) < 60.0
