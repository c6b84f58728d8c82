"""Path-simulated inner values (Exact and Unbiased options, portfolio_sampler.cpp:470-604;
gbm_approx.hpp:18-57) on the batched OUTER layout.

An Exact or Unbiased inner sample draws a variable number of normals (the Unbiased method a random
level L with h0 beta^L coupled fine / coarse Milstein or Euler steps); on the OUTER layout each
inner sample i of a phase has its own counter namespaces for them (normals: tag | (i + 1) << 16,
the level uniform: | 2^15), so any thread evaluates any inner sample.  Checks:
  * REF32 and FP64 against the oracle's OUTER restatement on the same streams: per-outer-sample
    counts equal except where the oracle's adaptive decision was within MARGIN of its threshold,
    phi equal except where |inner mean| < FLIP (libm ulps: the GPU's log / exp / sqrt against
    glibc's), level sums within what the differing samples explain;
  * FP32 (SFU Box-Muller normals, the same path arithmetic) against FP64 on the same streams:
    phi may differ only where |inner mean| < 1e-3 x the portfolio scale, counts only where the
    FP64 decision was within 1e-4 of its threshold, at most 2 % of outer samples;
  * the batch size of a call changes no result (addressability of the per-sample streams);
  * Subsampling::None is refused on the batched layout.
"""
import numpy as np
import pytest

import oracle as O
from test_gpu_parity import (FLIP_FP64, FLIP_REF32, MARGIN_FP32, MARGIN_FP64, MARGIN_REF32,
                             assert_sums_explained, compare_traces)

pytestmark = pytest.mark.gpu

# the golden mixed-method configurations (BS / Exact / Unbiased options, Milstein and Euler,
# antithetic risk and coarse delta CV on and off), sub-sampled modes only
CASES = [
    dict(name="J_cdf_cv", pf=dict(Q=3, P=24, seed=21, prob="w"), sub=O.SUB_RANDOM, cv=True, rho=0.2,
         max_loss=0.3, N0=32, beta=4, r=1.5, seed=6, anti_risk=True, milstein=True, coarse_cv=False,
         methods=[0, 2, 0, 0, 0, 0, 2, 2, 2, 2, 0, 0, 1, 1, 2, 0, 1, 2, 0, 1, 2, 2, 1, 0],
         calls=[(0, 400), (1, 300), (3, 120)]),
    dict(name="K_uniform_euler", pf=dict(Q=2, P=12, seed=22, prob="uniform"), sub=O.SUB_UNIFORM, cv=True,
         rho=0.0, max_loss=0.2, N0=32, beta=2, r=1.5, seed=8, anti_risk=False, milstein=False, coarse_cv=True,
         methods=[2, 0, 1, 1, 2, 0, 0, 1, 0, 2, 1, 2], calls=[(0, 300), (2, 200), (4, 80)]),
    # deep Unbiased levels (P(L) ~ 2^(-1.1 L), h0 = 1: about 2 % of the samples at L >= 5, which
    # the FP32 kernel evaluates warp-wide)
    dict(name="L_deep_levels", pf=dict(Q=3, P=24, seed=23, prob="w"), sub=O.SUB_RANDOM, cv=True, rho=0.1,
         max_loss=0.3, N0=32, beta=2, r=1.5, seed=9, anti_risk=True, milstein=True, coarse_cv=True,
         methods=[2, 2, 2, 0, 2, 2, 1, 2, 2, 2, 2, 2, 2, 0, 2, 2, 2, 2, 1, 2, 2, 2, 2, 2],
         dt=dict(dt_h0inv=1, dt_beta=2, dt_prob_expo=-1.1), calls=[(0, 300), (2, 200), (3, 120)]),
]


def pair(nm, case, o_prec, g_prec):
    import nmlmc
    pf = O.synthetic_portfolio(**case["pf"])
    kw = dict(r=0.05, rho=case["rho"], max_loss=case["max_loss"], tau=1 / 52, subsample=case["sub"],
              use_delta_cv=case["cv"])
    flags = dict(use_coarse_delta_cv=case["coarse_cv"], use_antithetic_risk=case["anti_risk"],
                 use_milstein=case["milstein"])
    o = O.Sampler(o_prec, O.STREAMS_OUTER, 1, case["N0"], case["beta"], case["r"], True, False, case["seed"])
    dt = case.get("dt", {})
    o.set_portfolio_methods(pf, case["methods"], **kw, **flags, **dt)
    g = nmlmc.Sampler(N0=case["N0"], beta=case["beta"], adaptive_r=case["r"], precision=g_prec,
                      streams=nmlmc.STREAMS_OUTER, seed=case["seed"])
    g.set_portfolio(pf, **kw, methods=dict(method=case["methods"], **flags, **dt))
    return o, g


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
@pytest.mark.parametrize("prec_name", ["ref32", "fp64"])
def test_outer_paths_match_the_oracle(nm, case, prec_name):
    o_prec = O.PREC_REF32 if prec_name == "ref32" else O.PREC_FP64
    g_prec = nm.PREC_REF32 if prec_name == "ref32" else nm.PREC_FP64
    flip, margin = (FLIP_REF32, MARGIN_REF32) if prec_name == "ref32" else (FLIP_FP64, MARGIN_FP64)
    o, g = pair(nm, case, o_prec, g_prec)
    for ell, M in case["calls"]:
        ro = o.sample(ell, M, trace=True, margins=True)
        rg = g.sample(ell, M, trace=True)
        compare_traces(rg["trace"], ro["trace"], flip, max_frac=0.01, margins=ro["margins"], margin_bound=margin)
        assert_sums_explained(rg, ro, f32=prec_name == "ref32")
        assert rg["work"] == pytest.approx(ro["work"], rel=1e-12)


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_outer_paths_fp32_against_fp64(nm, case):
    o, g64 = pair(nm, case, O.PREC_FP64, nm.PREC_FP64)
    _, g32 = pair(nm, case, O.PREC_FP64, nm.PREC_FP32)
    for ell, M in case["calls"]:
        ro = o.sample(ell, M, trace=True, margins=True)
        r64 = g64.sample(ell, M, trace=True)
        r32 = g32.sample(ell, M, trace=True)
        compare_traces(r64["trace"], ro["trace"], FLIP_FP64, max_frac=0.01, margins=ro["margins"],
                       margin_bound=MARGIN_FP64)
        compare_traces(r32["trace"], r64["trace"], 1e-3, max_frac=0.02, margins=ro["margins"],
                       margin_bound=MARGIN_FP32)
        assert_sums_explained(r32, r64, f32=True)


def test_outer_paths_batch_split_is_invisible(nm):
    import nmlmc
    case = CASES[0]
    pf = O.synthetic_portfolio(**case["pf"])
    out = []
    for batch in (1 << 16, 37):
        g = nmlmc.Sampler(N0=case["N0"], beta=case["beta"], adaptive_r=case["r"], precision=nm.PREC_FP32,
                          streams=nmlmc.STREAMS_OUTER, seed=4, batch=batch)
        g.set_portfolio(pf, r=0.05, rho=case["rho"], max_loss=case["max_loss"], tau=1 / 52,
                        subsample=case["sub"], use_delta_cv=case["cv"],
                        methods=dict(method=case["methods"], use_milstein=True))
        out.append(g.sample(2, 300, trace=True))
    np.testing.assert_array_equal(out[0]["trace"], out[1]["trace"])
    np.testing.assert_array_equal(out[0]["fsums"], out[1]["fsums"])


def test_outer_layout_refuses_no_subsampling(nm):
    import nmlmc
    pf = O.synthetic_portfolio(2, 6, 3)
    for methods in (None, dict(method=[0, 1, 2, 0, 1, 2])):
        s = nmlmc.Sampler(precision=nm.PREC_FP64, streams=nmlmc.STREAMS_OUTER, N0=32, beta=4, adaptive_r=1.5)
        s.set_portfolio(pf, subsample=nmlmc.SUB_NONE, methods=methods)
        with pytest.raises(nm.NmlmcError):
            s.sample(1, 10)


@pytest.mark.parametrize("prec_name", ["fp32", "fp64"])
def test_outer_paths_beyond_the_step_limit_fail(nm, prec_name):
    """An Unbiased inner sample whose h0 beta^L steps exceed NMLMC_MAX_PATH_STEPS fails the call
    with ERR_LIMIT before any path is stepped: with 1 / h0 = 2^24 + 1 every level does."""
    import nmlmc
    case = CASES[0]
    pf = O.synthetic_portfolio(**case["pf"])
    s = nmlmc.Sampler(N0=case["N0"], beta=case["beta"], adaptive_r=case["r"],
                      precision=nm.PREC_FP32 if prec_name == "fp32" else nm.PREC_FP64,
                      streams=nmlmc.STREAMS_OUTER, seed=4)
    s.set_portfolio(pf, r=0.05, rho=case["rho"], max_loss=case["max_loss"], tau=1 / 52, subsample=case["sub"],
                    use_delta_cv=case["cv"],
                    methods=dict(method=[2] * len(pf["w"]), dt_h0inv=(1 << 24) + 1, use_milstein=True))
    with pytest.raises(nm.NmlmcError) as err:
        s.sample(1, 64)
    assert err.value.status == nm.ERR_LIMIT
