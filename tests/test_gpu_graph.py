"""nmlmc_sample_levels on the OUTER layout: one CUDA-graph submission per round.

The graph path must give bit-identical level results to consecutive nmlmc_sample calls on the
same streams, and rounds with the same topology must update the cached executable graph in
place instead of instantiating a new one.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pair(nm, precision, adaptive_r=1.5, seed=4):
    kw = dict(N0=32, beta=2, adaptive_r=adaptive_r, precision=precision, streams=nm.STREAMS_OUTER, seed=seed)
    a, b = nm.Sampler(**kw), nm.Sampler(**kw)
    for s in (a, b):
        s.set_model(nm.MODEL_SHIFT, 0.0, 1.0)
    return a, b


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_levels_submission_equals_per_level_calls(nm, prec):
    precision = nm.PREC_FP32 if prec == "fp32" else nm.PREC_FP64
    a, b = _pair(nm, precision)
    rounds = [([0, 1, 2, 3], [20000, 6000, 3000, 1500]),
              ([0, 1, 2, 3], [9000, 4000, 2500, 700]),
              ([0, 2, 4, 0], [5000, 800, 300, 1000])]   # a level twice in one round
    for ells, Ms in rounds:
        ra = a.sample_levels(ells, Ms)
        rb = [b.sample(e, m) for e, m in zip(ells, Ms)]
        for x, y in zip(ra, rb):
            np.testing.assert_array_equal(x["fsums"], y["fsums"])
            np.testing.assert_array_equal(x["diffsums"], y["diffsums"])
            np.testing.assert_array_equal(x["stats"], y["stats"])
            assert x["work"] == y["work"] and x["M"] == y["M"]
            assert x["seconds"] > 0
    st = a.graph_stats()
    assert st["launches"] == len(rounds)
    assert st["updates"] >= 1                 # round 2 repeats round 1's topology
    assert st["instantiations"] + st["updates"] == len(rounds)


def test_levels_submission_portfolio(nm):
    import oracle as O
    pf = O.synthetic_portfolio(4, 100, 3, prob="w")
    kw = dict(N0=32, beta=2, adaptive_r=1.5, precision=nm.PREC_FP32, streams=nm.STREAMS_OUTER, seed=2)
    a, b = nm.Sampler(**kw), nm.Sampler(**kw)
    for s in (a, b):
        s.set_portfolio(pf, rho=0.2, max_loss=0.5, subsample=nm.SUB_RANDOM, use_delta_cv=True)
    ra = a.sample_levels([0, 1, 2], [4000, 2000, 1000])
    rb = [b.sample(e, m) for e, m in ((0, 4000), (1, 2000), (2, 1000))]
    for x, y in zip(ra, rb):
        np.testing.assert_array_equal(x["fsums"], y["fsums"])
        np.testing.assert_array_equal(x["diffsums"], y["diffsums"])
