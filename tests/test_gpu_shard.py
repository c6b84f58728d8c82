"""Outer-sample sharding on the GPU (nmlmc_set_shard), the data path of a multi-GPU run.

Rank r of W evaluates its static share of every level call: floor(M / W) outer samples, one more on
the first M mod W ranks, with the stream indices one device would use.  Emulated here on one GPU
with W contexts evaluated one after another (each a separate call; no kernel waits for another):
the ranks' traces, laid end to end, equal the unsharded call's trace record for record, and the
ranks' level sums added together equal the unsharded sums exactly (the moments are sums of phi
powers with power-of-two denominators, exact in double at these sizes), for per-level calls and
for the batched submission of several levels (nmlmc_sample_levels, one CUDA graph per call).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sampler(nm, prec, seed=9):
    s = nm.Sampler(0, N0=32, beta=2, adaptive_r=1.5, precision=prec, streams=nm.STREAMS_OUTER, seed=seed)
    s.set_model(nm.MODEL_SHIFT, 0.0, 1.0)
    s.set_autotune(0)
    return s


def _share(M, W, r):
    q, rem = divmod(M, W)
    return q + (1 if r < rem else 0)


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("prec_name", ["fp32", "fp64"])
def test_shards_add_up_to_the_unsharded_call(nm, world, prec_name):
    prec = nm.PREC_FP32 if prec_name == "fp32" else nm.PREC_FP64
    full = _sampler(nm, prec)
    ranks = [_sampler(nm, prec) for _ in range(world)]
    for r, s in enumerate(ranks):
        s.set_shard(r, world)
    for ell, M in ((0, 10001), (3, 7000), (6, 4003), (3, 5000)):   # level 3 twice: the next indices
        ref = full.sample(ell, M, trace=True)
        parts = [s.sample(ell, M, trace=True) for s in ranks]
        tr = np.concatenate([p["trace"][:_share(M, world, r)] for r, p in enumerate(parts)])
        np.testing.assert_array_equal(tr, ref["trace"])
        for key in ("fsums", "diffsums"):
            np.testing.assert_array_equal(sum(p[key] for p in parts), ref[key])
        assert sum(p["work"] for p in parts) == ref["work"]
        assert sum(int(p["stats"][0]) for p in parts) == int(ref["stats"][0])


@pytest.mark.parametrize("world", [2, 3])
def test_shards_of_a_batched_round(nm, world):
    """nmlmc_sample_levels (all levels of a round in one graph) sharded the same way."""
    full = _sampler(nm, nm.PREC_FP32, seed=10)
    ranks = [_sampler(nm, nm.PREC_FP32, seed=10) for _ in range(world)]
    for r, s in enumerate(ranks):
        s.set_shard(r, world)
    for ells, Ms in (([0, 1, 2, 4], [20000, 9001, 5000, 2000]), ([0, 2, 4, 5], [3000, 3001, 1500, 999])):
        ref = full.sample_levels(ells, Ms)
        parts = [s.sample_levels(ells, Ms) for s in ranks]
        for i in range(len(ells)):
            for key in ("fsums", "diffsums"):
                np.testing.assert_array_equal(sum(p[i][key] for p in parts), ref[i][key])
            assert sum(p[i]["work"] for p in parts) == ref[i]["work"]
