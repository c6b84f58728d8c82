"""Multi-rank MLMC on CPU: two gloo ranks, each sampling its shard of every level call with the
CPU oracle as the local sampler (the GPU sampler has the same set_shard / sample interface), the
level results all-reduced (nmlmc.distributed.sharded_mlmc_run).  Both ranks must take exactly the
decisions of a single-process run and end with the same estimate and level sums."""
import os
import socket
import sys
from datetime import timedelta

import numpy as np

from conftest import PKG, ROOT

CFG = dict(N0=32, beta=2, r=1.5, seed=3, tol=4e-3, M0=256)


class OracleShardSampler:
    """CPU oracle on the OUTER layout, behind the nmlmc.Sampler interface used by the driver."""

    def __init__(self):
        import oracle as O
        self.s = O.Sampler(O.PREC_FP64, O.STREAMS_OUTER, 1, CFG["N0"], CFG["beta"], CFG["r"],
                           True, False, CFG["seed"])
        self.s.set_model(O.MODEL_SHIFT, 0.0, 1.0)

    def set_shard(self, rank, world):
        self.s.set_shard(rank, world)

    def sample(self, ell, M):
        r = self.s.sample(ell, M)
        return dict(fsums=r["fsums"], diffsums=r["diffsums"], work=r["work"], seconds=0.0)

    def sample_levels(self, ells, Ms):
        self.batches = getattr(self, "batches", 0) + 1
        return [self.sample(e, m) for e, m in zip(ells, Ms)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q, batched=False):
    for p in (ROOT, PKG, os.path.join(ROOT, "oracle")):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    from nmlmc.distributed import sharded_mlmc_run
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        smp = OracleShardSampler()
        out = sharded_mlmc_run(smp, targetTOL=CFG["tol"], M0=CFG["M0"], batched=batched)
        q.put((rank, [int(x) for x in out["level_M"]], out["Eg"], out["level_fsums"].tolist(),
               out["level_diffsums"].tolist(), out["calls"], getattr(smp, "batches", 0)))
    finally:
        dist.destroy_process_group()


import pytest


@pytest.mark.parametrize("world,batched", [(2, False), (2, True), (3, True)])
def test_gloo_ranks_reproduce_single_process(nm, world, batched):
    """Per-level calls, or one submission and one all_reduce per MLMC round (batched); three
    ranks split most calls unevenly."""
    import multiprocessing as mp
    single = nm.mlmc_run_cb(OracleShardSampler().sample, targetTOL=CFG["tol"], M0=CFG["M0"])
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, batched)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    for rank, level_M, Eg, fs, ds, calls, batches in res:
        assert (batches > 0) == batched
        assert level_M == [int(x) for x in single["level_M"]]
        assert Eg == single["Eg"]
        np.testing.assert_array_equal(np.array(fs), single["level_fsums"])
        np.testing.assert_array_equal(np.array(ds), single["level_diffsums"])
        assert calls == single["calls"]


class FailingShardSampler(OracleShardSampler):
    """Raises on its n-th level call: a rank whose sampler fails between collectives."""

    def __init__(self, fail_at=None):
        super().__init__()
        self.calls = 0
        self.fail_at = fail_at

    def sample(self, ell, M):
        self.calls += 1
        if self.fail_at is not None and self.calls == self.fail_at:
            raise RuntimeError("injected sampler failure")
        return super().sample(ell, M)


def _failing_worker(rank, world, port, q):
    for p in (ROOT, PKG, os.path.join(ROOT, "oracle")):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    from nmlmc.distributed import sharded_mlmc_run
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=20))
    try:
        smp = FailingShardSampler(fail_at=3 if rank == 1 else None)
        sharded_mlmc_run(smp, targetTOL=CFG["tol"], M0=CFG["M0"])
        q.put((rank, "finished"))
    except Exception as e:                      # noqa: BLE001 - reported to the parent
        q.put((rank, f"{type(e).__name__}: {e}"[:300]))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:                       # noqa: BLE001
            pass


def test_failing_rank_ends_the_other_ranks_with_an_error():
    """A rank whose sampler raises leaves the run between collectives; the other rank's next
    all_reduce ends with an error (peer gone, or the process group's 20 s timeout) instead of
    waiting for good, and both processes exit."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_failing_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode is not None
    assert "injected sampler failure" in res[1]
    assert res[0] != "finished", res[0]
