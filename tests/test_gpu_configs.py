"""The benchmark configurations at their own sizes, checked through properties that do not need
an oracle run of the same size:

* C0 (model problem, plain FP64, non-adaptive, eps = 1e-3) and C1 (adaptive, batched FP32 with
  FP64 moments, eps = 1e-4): the estimate of P(E[X|Y] > 1) lands within 2 eps of the closed form
  1 - Phi(1) (eps is the target RMSE; the tolerance is two RMSEs);
* C1's FP32 estimate equals the all-FP64 estimate on the same streams to 1e-6;
* C3 (large portfolio, eps = 1e-3): within 3 eps + 4 sigma of an independent direct estimate from
  2e5 full evaluations (sigma its binomial standard error).
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EXACT = 0.5 * math.erfc(1 / math.sqrt(2))


def _model(nm, prec, streams, r, seed, cores=2048):
    s = nm.Sampler(cores=cores, N0=32, beta=2, adaptive_r=r, precision=prec, streams=streams, seed=seed)
    s.set_model(nm.MODEL_SHIFT, 0.0, 1.0)
    return s


def test_c0_plain_fp64_within_eps(nm):
    eps = 1e-3
    out = _model(nm, nm.PREC_FP64, nm.STREAMS_CORE, 0.0, 0).mlmc_run(targetTOL=eps, M0=1024)
    assert out["complete"]
    assert abs(out["Eg"] - EXACT) < 2 * eps, (out["Eg"], EXACT)


def test_c1_batched_fp32_within_eps_and_equal_to_fp64(nm):
    eps = 1e-4
    o32 = _model(nm, nm.PREC_FP32, nm.STREAMS_OUTER, 1.5, 0).mlmc_run(targetTOL=eps, M0=1024, batched=True)
    o64 = _model(nm, nm.PREC_FP64, nm.STREAMS_OUTER, 1.5, 0).mlmc_run(targetTOL=eps, M0=1024, batched=True)
    assert abs(o32["Eg"] - EXACT) < 2 * eps, (o32["Eg"], EXACT)
    assert abs(o32["Eg"] - o64["Eg"]) < 1e-6
    # about 4e8 outer samples on level 0, levels up to 7 or more
    assert o32["level_M"][0] > 1e8 and o32["nlevels"] >= 6


def test_c3_large_portfolio_against_direct_estimate(nm):
    pf = nm.generate_portfolio(nm.PORTFOLIO_C3, 1)
    order = np.argsort(-np.abs(pf["w"]), kind="stable")
    for k in ("strike", "maturity", "w", "stock_ind", "type"):
        pf[k] = pf[k][order]
    pf = dict(pf, prob=np.abs(pf["w"]))

    def sampler(K, seed):
        s = nm.Sampler(N0=64, beta=2, adaptive_r=1.5, precision=nm.PREC_FP32, streams=nm.STREAMS_OUTER,
                       seed=seed)
        s.set_portfolio(pf, r=0.05, rho=0.0, max_loss=K, tau=nm.TAU_WEEK, subsample=nm.SUB_RANDOM,
                        use_delta_cv=True, discount=False)
        return s

    q = sampler(0.0, 1)
    K = nm.loss_quantile(q, 0.99, 100_000)
    Ld = q.full_loss(62, 0, 200_000)
    p = float(np.mean(Ld > K))
    sd = math.sqrt(p * (1 - p) / len(Ld))
    eps = 1e-3
    out = sampler(K, 5).mlmc_run(targetTOL=eps, M0=1024, batched=True)
    assert 0.007 < p < 0.013
    assert abs(out["Eg"] - p) < 3 * eps + 4 * sd, (out["Eg"], p, sd)
