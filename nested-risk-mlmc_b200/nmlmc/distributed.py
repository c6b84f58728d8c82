"""Multi-GPU MLMC: one process per GPU, outer samples sharded, level results all-reduced.

Every outer sample owns its random stream (OUTER layout), so rank r of W evaluates a contiguous
share of each sample_level(ell, M) call (nmlmc_set_shard: floor(M/W) outer samples, one more on
the first M mod W ranks) and the 16-double level
results are summed over ranks with one all_reduce per call (NCCL on GPUs, gloo on CPU).  All ranks
then hold the single-device result, run the same host driver and take the same decisions; no
data-path collective exists.  The sampler is any object with set_shard(rank, world) and
sample(ell, M) -> dict (fsums, diffsums, work, seconds) — nmlmc.Sampler on GPUs.  With `batched`
and a sampler that has sample_levels(ells, Ms), every MLMC round is one submission per rank (one
CUDA graph on GPUs) and one all_reduce of all its levels.
"""
from __future__ import annotations

from . import mlmc_run_cb


def sharded_mlmc_run(sampler, group=None, device=None, *, targetTOL=1e-3, M0=100,
                     batched=False, **kw) -> dict:
    import torch
    import torch.distributed as dist
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    sampler.set_shard(rank, world)
    dev = device if device is not None else torch.device("cpu")

    def reduce(results):
        t = torch.tensor([[*r["fsums"], *r["diffsums"], r["work"]] for r in results],
                         dtype=torch.float64, device=dev)
        dist.all_reduce(t, group=group)
        rows = t.cpu().numpy()
        # sums over ranks; the device time stays this rank's own
        return [dict(fsums=row[0:4], diffsums=row[4:8], work=float(row[8]),
                     seconds=float(r.get("seconds", 0.0))) for row, r in zip(rows, results)]

    def one(ell, M):
        return reduce([sampler.sample(ell, M)])[0]

    def many(ells, Ms):
        return reduce(sampler.sample_levels(ells, Ms))

    levels_fn = many if batched and hasattr(sampler, "sample_levels") else None
    out = mlmc_run_cb(one, levels_fn, targetTOL=targetTOL, M0=M0, batched=batched, **kw)
    sampler.set_shard(0, 1)
    return out


def max_over_ranks(value: float, group=None, device=None) -> float:
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64,
                     device=device if device is not None else torch.device("cpu"))
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


__all__ = ["sharded_mlmc_run", "max_over_ranks"]
