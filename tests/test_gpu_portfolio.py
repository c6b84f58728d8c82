"""GPU portfolio path: the FP32 SFU Black-Scholes against FP64 on the same streams, the loss
sweep, the seeded generator, and an end-to-end check of the C2 configuration (P(L > K) with K the
99 % loss quantile).

Tolerances (stated here, used below):
  * full-portfolio loss, FP32 vs FP64 on the same outer draws: |dL| <= 2e-6 * sum_i |w_i| (S0 + K_i)
    (per-option bound 1e-6 relative on each term of the regrouped BS value, nmlmc_bs.cuh);
  * FP32 vs FP64 level traces on the same streams: a phi may differ only where |inner mean| <
    2e-6 * P * mean_i |w_i| (S0 + K_i), an adaptive count only where the FP64 decision was within
    1e-4 of its threshold (|ln(new_count / cur)|, the oracle's margins); at most 0.5 % of outer
    samples; level sums differ only by what the differing outer samples explain;
  * the MLMC estimate of P(L > K) within 3 eps + 4 sigma of an independent full-evaluation
    Monte Carlo estimate over 2e6 outer samples.
"""
import numpy as np
import pytest

import oracle as O
from test_gpu_parity import MARGIN_FP32, MARGIN_FP64, assert_sums_explained, compare_traces

pytestmark = pytest.mark.gpu


def small_spec(nm, Q=20, P=2000):
    return dict(nm.PORTFOLIO_C2, Q=Q, P=P)


def sampler(nm, prec, pf, seed=0, **kw):
    s = nm.Sampler(0, N0=64, beta=2, adaptive_r=kw.pop("adaptive_r", 0.0), precision=prec,
                   streams=nm.STREAMS_OUTER, seed=seed)
    s.set_portfolio(pf, r=0.05, rho=kw.pop("rho", 0.0), max_loss=kw.pop("K", 0.0), tau=nm.TAU_WEEK,
                    subsample=nm.SUB_UNIFORM, use_delta_cv=kw.pop("cv", False),
                    discount=kw.pop("discount", False))
    return s


def test_fast_norm_cdf_bound(nm):
    """Phi of the FP32 Black-Scholes (rational erfc, SFU exponential and reciprocal) against the
    double-precision Phi over |x| <= 10: absolute error <= 2.5e-7; relative error <= 1e-5 where
    Phi >= 1e-20 (measured 2.0e-7 and 4.5e-6; the FP32 exponent limits the far tail)."""
    from math import erfc, sqrt
    x = np.concatenate([np.linspace(-10, 10, 200001), np.random.default_rng(1).uniform(-10, 10, 100000)])
    x = x.astype(np.float32)
    got = nm.norm_cdf_fast(x).astype(np.float64)
    ref = np.array([0.5 * erfc(-float(v) / sqrt(2.0)) for v in x])
    assert np.max(np.abs(got - ref)) <= 2.5e-7
    m = ref >= 1e-20
    rel = np.abs(got[m] - ref[m]) / ref[m]
    assert rel.max() <= 1e-5, (rel.max(), x[m][np.argmax(rel)])


def test_generator_deterministic(nm):
    a = nm.generate_portfolio(nm.PORTFOLIO_C2, 7)
    b = nm.generate_portfolio(nm.PORTFOLIO_C2, 7)
    c = nm.generate_portfolio(nm.PORTFOLIO_C2, 8)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])
    assert not np.array_equal(a["w"], c["w"])
    assert a["sigma"].min() >= 0.1 and a["sigma"].max() <= 0.4
    assert a["strike"].min() >= 80 and a["strike"].max() <= 120
    assert a["maturity"].min() >= 0.25 and a["maturity"].max() <= 2.0
    assert abs((a["type"] > 0).mean() - 0.5) < 0.02
    assert abs(a["w"].mean()) < 0.05 and abs(a["w"].std() - 1) < 0.05


def test_fp32_loss_sweep_against_fp64(nm):
    pf = nm.generate_portfolio(small_spec(nm), 3)
    s32 = sampler(nm, nm.PREC_FP32, pf)
    s64 = sampler(nm, nm.PREC_FP64, pf)
    L32 = s32.full_loss(5, 0, 4000)
    L64 = s64.full_loss(5, 0, 4000)
    scale = np.sum(np.abs(pf["w"]) * (100.0 + pf["strike"]))
    err = np.max(np.abs(L32 - L64))
    assert err <= 2e-6 * scale, (err, scale)
    # the FP64 sweep equals the CPU oracle's (reference arithmetic) on the same streams
    o = O.Sampler(O.PREC_FP64, O.STREAMS_OUTER, 1, 64, 2, 0.0, True, False, 0)
    o.set_portfolio(pf, r=0.05, rho=0.0, max_loss=0.0, tau=1 / 52, subsample=O.SUB_UNIFORM,
                    use_delta_cv=False, discount=False)
    np.testing.assert_allclose(L64[:200], o.full_loss(5, 0, 200), rtol=1e-11, atol=1e-8)


@pytest.mark.parametrize("cv", [False, True])
def test_fp32_level_traces_against_fp64(nm, cv):
    """FP32 against FP64 on the same streams; a count may differ only where the FP64 decision
    (the oracle's, on the same streams) was within MARGIN_FP32 of its threshold, and the level
    sums differ only by what the differing outer samples explain."""
    pf = nm.generate_portfolio(small_spec(nm, Q=8, P=500), 4)
    s64 = sampler(nm, nm.PREC_FP64, pf, adaptive_r=1.5, K=30.0, cv=cv)
    s32 = sampler(nm, nm.PREC_FP32, pf, adaptive_r=1.5, K=30.0, cv=cv)
    o = O.Sampler(O.PREC_FP64, O.STREAMS_OUTER, 1, 64, 2, 1.5, True, False, 0)
    o.set_portfolio(pf, r=0.05, rho=0.0, max_loss=30.0, tau=nm.TAU_WEEK, subsample=O.SUB_UNIFORM,
                    use_delta_cv=cv, discount=False)
    scale = 500 * np.mean(np.abs(pf["w"]) * (100.0 + pf["strike"]))
    for ell, M in ((0, 4000), (2, 2000), (5, 500)):
        g64 = s64.sample(ell, M, trace=True)
        g32 = s32.sample(ell, M, trace=True)
        go = o.sample(ell, M, trace=True, margins=True)
        compare_traces(g64["trace"], go["trace"], 1e-9 * scale, margins=go["margins"], margin_bound=MARGIN_FP64)
        compare_traces(g32["trace"], g64["trace"], 2e-6 * scale, max_frac=0.005, margins=go["margins"],
                       margin_bound=MARGIN_FP32)
        assert_sums_explained(g32, g64, f32=True)


def test_c2_end_to_end(nm):
    """C2: d = 20, P = 1e4, uniform sub-sampling, 64 * 2^ell inner samples, K = 99 % quantile of L
    over 1e5 full evaluations (seed 1); the MLMC estimate of P(L > K) agrees with a direct estimate
    from 2e6 full evaluations (sigma ~ 7e-5).  eps = 3e-4 (about 15 s on a B200): the
    configuration's relative 1e-2 (1e-4 absolute) takes the same sampler about 150 s, with the
    starting level at 11 and 3e13 inner samples (bench.py --case c2)."""
    pf = nm.generate_portfolio(nm.PORTFOLIO_C2, 1)
    q = sampler(nm, nm.PREC_FP32, pf, seed=1)
    K = nm.loss_quantile(q, 0.99, 100_000)
    # independent direct estimate of P(L > K) on other outer samples
    Ld = np.concatenate([q.full_loss(62, k * 500_000, 500_000) for k in range(4)])
    p_direct = float(np.mean(Ld > K))
    sd = np.sqrt(p_direct * (1 - p_direct) / len(Ld))
    s = sampler(nm, nm.PREC_FP32, pf, seed=5, K=K)
    eps = 3e-4
    out = s.mlmc_run(targetTOL=eps, M0=1024, batched=True)
    assert abs(out["Eg"] - p_direct) < 3 * eps + 4 * sd, (out["Eg"], p_direct, sd)
    assert 0.008 < p_direct < 0.012


def test_c3_end_to_end_at_its_eps(nm):
    """The large portfolio (d = 200, P = 1e6, importance sub-sampling prob ~ |w| with the delta
    control variate, adaptive r = 1.5) at the configuration's eps = 1e-4: the batched FP32 MLMC
    estimate of P(L > K) within 3 eps + 4 sigma of a direct estimate from 2e6 full evaluations of
    the loss (sigma ~ 7e-5), and P(L > K) near 0.01 by construction of K."""
    import bench
    pfw = bench.c3_portfolio(nm)
    q = bench.c3_sampler(nm, 0, pfw, 0.0, nm.PREC_FP32, nm.STREAMS_OUTER, seed=1)
    K = nm.loss_quantile(q, 0.99, 100_000)
    Ld = np.concatenate([q.full_loss(61, k * 500_000, 500_000) for k in range(4)])
    p_direct = float(np.mean(Ld > K))
    sd = float(np.sqrt(p_direct * (1 - p_direct) / len(Ld)))
    s = bench.c3_sampler(nm, 0, pfw, K, nm.PREC_FP32, nm.STREAMS_OUTER, seed=21)
    eps = 1e-4
    out = s.mlmc_run(targetTOL=eps, M0=1024, batched=True)
    assert abs(out["Eg"] - p_direct) < 3 * eps + 4 * sd, (out["Eg"], p_direct, sd)
    assert 0.008 < p_direct < 0.012
