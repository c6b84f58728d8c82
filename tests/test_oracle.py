"""The CPU oracle (oracle/nmlmc_oracle.c) against the golden fixtures produced by the unmodified
reference (tests/golden/make_golden.py): bit-exact Threefry, random_state draws, Box-Muller,
norm_cdf_inv, option start values, and per-call event logs, level sums and inner_stats of the
nested sampler engine."""
import numpy as np
import pytest

import oracle as O


def test_threefry_golden(golden):
    _, A = golden
    out = O.threefry(A["threefry/ctr"], A["threefry/key"])
    np.testing.assert_array_equal(out, A["threefry/out"])
    # the value recorded when the reference was first run here
    assert int(out[0, 0]) == 0xC2B6E3A8C2C69865 and int(out[0, 1]) == 0x6F81ED42F350084D


@pytest.mark.parametrize("variant,prec", [("f32", O.PREC_REF32), ("f64", O.PREC_FP64)])
def test_stream_draws_golden(golden, variant, prec):
    meta, A = golden
    ops = meta["stream_ops"]
    for (s, c) in [(0, 0), (7, 3), (2**63 + 5, 2**32 + 1)]:
        real, u64 = O.stream_draws(prec, s, c, ops)
        np.testing.assert_array_equal(u64, A[f"stream/{variant}/{s}/{c}/u64"])
        np.testing.assert_array_equal(real, A[f"stream/{variant}/{s}/{c}/real"])


def test_boxmuller_golden(golden):
    _, A = golden
    x, y = O.boxmuller(A["bm/u0"], A["bm/u1"])
    np.testing.assert_array_equal(x, A["bm/x"])
    np.testing.assert_array_equal(y, A["bm/y"])


def test_norm_cdf_inv_golden(golden):
    _, A = golden
    got32 = np.array([O.norm_cdf_inv(p, O.PREC_REF32) for p in A["ncdfinv/p"]])
    got64 = np.array([O.norm_cdf_inv(p, O.PREC_FP64) for p in A["ncdfinv/p"]])
    np.testing.assert_array_equal(got32, A["ncdfinv/f32"])
    np.testing.assert_array_equal(got64, A["ncdfinv/f64"])


def _events(A, key):
    return (bytes(A[key + "/kinds"]).decode(), A[key + "/values"], A[key + "/aux"])


def make_oracle_case(case, prec, streams=O.STREAMS_CORE, cores=None):
    s = O.Sampler(prec, streams, cores or case["cores"], case["N0"], case["beta"], case["r"],
                  case["anti"], False, case["seed"])
    start = delta = None
    if case["kind"] == "model":
        s.set_model(case["model"], case["tau"], case["max_loss"])
    else:
        pf = O.synthetic_portfolio(**case["pf"])
        if "methods" in case:
            s.set_portfolio_methods(pf, case["methods"], r=0.05, rho=case["rho"],
                                    max_loss=case["max_loss"], tau=1 / 52, subsample=case["sub"],
                                    use_delta_cv=case["cv"], use_coarse_delta_cv=case["coarse_cv"],
                                    use_antithetic_risk=case["anti_risk"],
                                    use_milstein=case["milstein"])
            return s, None, None
        start, delta = s.set_portfolio(pf, r=0.05, rho=case["rho"], max_loss=case["max_loss"],
                                       tau=1 / 52, subsample=case["sub"], use_delta_cv=case["cv"])
    return s, start, delta


def engine_case_ids(meta):
    return [c["name"] for c in meta["engine"]]


@pytest.mark.parametrize("prec_name,prec", [("f32", O.PREC_REF32), ("f64", O.PREC_FP64)])
def test_engine_golden(golden, prec_name, prec):
    meta, A = golden
    for case in meta["engine"]:
        res = case["results"][prec_name]
        s, start, delta = make_oracle_case(case, prec)
        if start is not None:
            np.testing.assert_array_equal(start, A[f"{case['name']}/{res['variant']}/start"])
            np.testing.assert_array_equal(delta, A[f"{case['name']}/{res['variant']}/delta_est"])
        for i, call in enumerate(res["calls"]):
            got = s.sample(call["ell"], call["M"], events_cap=2_000_000)
            key = f"{case['name']}/{res['variant']}/{i}"
            k_ref, v_ref, a_ref = _events(A, key)
            k, v, a = got["events"]
            assert k == k_ref, (case["name"], i)
            np.testing.assert_array_equal(v, v_ref, err_msg=f"{case['name']} call {i}")
            np.testing.assert_array_equal(a, a_ref)
            np.testing.assert_array_equal(got["fsums"], call["fsums"])
            np.testing.assert_array_equal(got["diffsums"], call["diffsums"])
            assert got["work"] == call["work"]
            np.testing.assert_array_equal(got["stats"].astype(np.int64), call["stats"])


def test_trace_consistent_with_events(golden):
    """Per-outer-sample records agree with the event log of the same run."""
    meta, _ = golden
    case = meta["engine"][0]
    s, _, _ = make_oracle_case(case, O.PREC_REF32)
    got = s.sample(2, 30, trace=True, events_cap=200000)
    kinds, vals, aux = got["events"]
    tr = got["trace"]
    # one 'O' per outer sample; the last 'P' of each outer sample is the big-count mean
    outer_starts = [i for i, k in enumerate(kinds) if k == "O"] + [len(kinds)]
    for m in range(30):
        seg = range(outer_starts[m], outer_starts[m + 1])
        last_p = [i for i in seg if kinds[i] == "P"][-1]
        assert vals[last_p] == tr["mean_big"][m]
    assert tr["phi_f"].sum() == got["fsums"][0]
    assert (tr["phi_f"] - tr["phi_c"]).sum() == got["diffsums"][0]


def test_outer_layout_order_independent():
    """OUTER layout: splitting a call into pieces gives the same per-outer-sample results."""
    a = O.Sampler(O.PREC_FP64, O.STREAMS_OUTER, 1, 32, 2, 1.5, True, False, 9)
    a.set_model(O.MODEL_SHIFT, 0.0, 1.0)
    b = O.Sampler(O.PREC_FP64, O.STREAMS_OUTER, 1, 32, 2, 1.5, True, False, 9)
    b.set_model(O.MODEL_SHIFT, 0.0, 1.0)
    whole = a.sample(4, 40, trace=True)["trace"]
    p1 = b.sample(4, 15, trace=True)["trace"]
    p2 = b.sample(4, 25, trace=True)["trace"]
    np.testing.assert_array_equal(whole, np.concatenate([p1, p2]))


@pytest.mark.skipif(not O.ref_available("f32_lzcnt"), reason="oracle/_ref not built on this host")
def test_live_reference_random_case():
    """Where the reference is compiled here: a fresh random configuration, oracle vs reference."""
    rng = np.random.default_rng(77)
    cores = int(rng.integers(1, 6))
    ref = O.Reference("f32_lzcnt")
    ref.init(cores, 32, 2, 1.5, True)
    ref.model_init(1, 0.0, 0.7, 123, traced=True)
    s = O.Sampler(O.PREC_REF32, O.STREAMS_CORE, cores, 32, 2, 1.5, True, False, 123)
    s.set_model(O.MODEL_SHIFT, 0.0, 0.7)
    for ell in (0, 3, 5, 2):
        a = ref.sample(ell, 33, events_cap=500000)
        b = s.sample(ell, 33, events_cap=500000)
        assert a["events"][0] == b["events"][0]
        np.testing.assert_array_equal(a["events"][1], b["events"][1])
        np.testing.assert_array_equal(a["fsums"], b["fsums"])
        np.testing.assert_array_equal(a["diffsums"], b["diffsums"])


def test_outer_path_methods_need_subsampling():
    """On the OUTER layout every inner sample draws one option (and path-simulated options draw
    from the inner sample's own counter namespaces): path methods need a sub-sampled mode."""
    pf = O.synthetic_portfolio(2, 4, 1)
    s = O.Sampler(O.PREC_FP64, O.STREAMS_OUTER, 1, 32, 4, 1.5, True, False, 1)
    with pytest.raises(ValueError):
        s.set_portfolio_methods(pf, [0, 1, 2, 0], subsample=O.SUB_NONE)
    s2 = O.Sampler(O.PREC_FP64, O.STREAMS_OUTER, 1, 32, 4, 1.5, True, False, 1)
    s2.set_portfolio_methods(pf, [0, 1, 2, 0], subsample=O.SUB_RANDOM)
    s2.sample(1, 20)


def test_outer_exact_paths_average_to_black_scholes():
    """The OUTER layout's per-inner-sample path streams give unbiased option values: with every
    option priced by exact GBM paths (sample_inner_exact, portfolio_sampler.cpp:470-519) the inner
    mean of each outer sample agrees with the Black-Scholes one (same outer draws, the same option
    drawn by each inner sample) within 4 standard errors of their differences."""
    pf = O.synthetic_portfolio(2, 8, 5, "uniform")
    M, ell = 24, 4                                   # 32 * 4^4 = 8192 inner samples per outer sample
    kw = dict(r=0.05, rho=0.0, max_loss=0.0, tau=1 / 52, subsample=O.SUB_UNIFORM, use_delta_cv=False)
    bs = O.Sampler(O.PREC_FP64, O.STREAMS_OUTER, 1, 32, 4, 0.0, True, False, 3)
    bs.set_portfolio(pf, **kw, discount=True)
    ex = O.Sampler(O.PREC_FP64, O.STREAMS_OUTER, 1, 32, 4, 0.0, True, False, 3)
    ex.set_portfolio_methods(pf, [1] * 8, **kw)
    a = bs.sample(ell, M, trace=True)["trace"]["mean_big"]
    b = ex.sample(ell, M, trace=True)["trace"]["mean_big"]
    d = b - a
    assert np.all(np.isfinite(d)) and np.std(d) > 0
    assert abs(d.mean()) < 4 * d.std(ddof=1) / np.sqrt(M), (d.mean(), d.std(ddof=1))


@pytest.mark.skipif(not O.ref_available("f64_lzcnt"), reason="oracle/_ref not built on this host")
def test_live_reference_methods_case():
    """Where the reference is compiled here: a random mixed-method portfolio, oracle vs reference."""
    rng = np.random.default_rng(78)
    pf = O.synthetic_portfolio(3, 15, 31, prob="w")
    meth = rng.integers(0, 3, 15).astype(np.int32)
    ref = O.Reference("f64_lzcnt")
    ref.init(2, 32, 2, 1.5, True)
    ref.portfolio_init_methods(pf, meth, rho=0.1, max_loss=0.2, use_delta_cv=True, seed=44)
    s = O.Sampler(O.PREC_FP64, O.STREAMS_CORE, 2, 32, 2, 1.5, True, False, 44)
    s.set_portfolio_methods(pf, meth, rho=0.1, max_loss=0.2, use_delta_cv=True)
    for ell in (0, 2, 1):
        a = ref.sample(ell, 10, events_cap=500000)
        b = s.sample(ell, 10, events_cap=500000)
        assert a["events"][0] == b["events"][0]
        np.testing.assert_array_equal(a["events"][1], b["events"][1])
        np.testing.assert_array_equal(a["fsums"], b["fsums"])
        assert a["work"] == b["work"]


def test_adj_oracle_risk_neutral_mean():
    """Path-simulated loss oracle: with mu = r the discounted inner value is a martingale, so E[L]
    vanishes up to the time-step bias and the sampling error."""
    g = np.random.default_rng(3)
    Q, P = 2, 10
    S0 = np.array([100.0, 95.0])
    si = g.integers(0, Q, P).astype(np.uint32)
    b = dict(stock_off=np.array([0, Q], np.uint32), option_off=np.array([0, P], np.uint32),
             S0=S0, mu=np.full(Q, 0.05), sigma=np.array([0.2, 0.3]), stock_ind=si,
             type=np.where(g.random(P) < 0.5, 1, -1).astype(np.int32),
             maturity=0.5 + g.random(P), w=g.standard_normal(P), r=0.05, rho=0.3, tau=1 / 52)
    b["strike"] = S0[si] * (0.9 + 0.2 * g.random(P))
    L = O.adj_loss(b, 4, 32, 400, 7, True)[0]
    se = L.std() / np.sqrt(L.size)
    assert abs(L.mean()) < 4 * se + 5e-3 * np.abs(b["w"]).sum(), (L.mean(), se)


@pytest.mark.parametrize("P", [1, 2, 7, 1000, 4096])
def test_alias_table_exact_masses(P):
    """Every option's mass in the alias table equals W_j = phat_j P 2^32 exactly, the masses sum
    to P 2^32, and phat is within one mass unit of the requested probabilities."""
    g = np.random.default_rng(P)
    p = np.abs(g.standard_normal(P)) ** 3
    p[: max(1, P // 10)] *= 1e-9                       # some nearly-zero masses
    thr, al, ph = O.build_alias(p)
    unit = 1 << 32
    mass = np.zeros(P, dtype=object)
    for j in range(P):
        mass[j] += int(thr[j])
        mass[int(al[j])] += unit - int(thr[j])
    W = [int(round(x * P * unit)) for x in ph]
    assert list(mass) == W
    assert sum(W) == P * unit
    # rounding: half a unit per option, the summed residue (at most P/2 units) on the largest
    np.testing.assert_allclose(ph, p / p.sum(), rtol=0, atol=(P / 2 + 1) / (P * unit) + 1e-16)


def test_alias_draw_distribution():
    """The OUTER draw (column floor(v P / 2^64), coin (v P mod 2^64) >> 32) reproduces phat."""
    g = np.random.default_rng(1)
    p = np.array([5.0, 1.0, 0.25, 3.0, 0.75])
    thr, al, ph = O.build_alias(p)
    P = len(p)
    n = 200_000
    idx = np.empty(n, np.int64)
    for t, v in enumerate(int(x) for x in g.integers(0, 2**64, n, dtype=np.uint64, endpoint=False)):
        col = (v * P) >> 64
        coin = ((v * P) & (2**64 - 1)) >> 32
        idx[t] = col if coin < int(thr[col]) else int(al[col])
    freq = np.bincount(idx, minlength=P) / n
    assert np.all(np.abs(freq - ph) <= 4 * np.sqrt(ph * (1 - ph) / n)), (freq, ph)


# cores, N0, beta, adaptive r, antithetic, model kind, tau, K, levels, M per call: the sampler's
# parameters and edge sizes (M = 1, M below the core count so some cores get no outer sample,
# non-adaptive r = 0, r close to 2, beta = 4, odd core counts, no antithetic estimator)
LIVE_GRID = [
    (1, 32, 2, 0.0, True, O.MODEL_SHIFT, 0.0, 1.0, (0, 2, 4), 17),
    (3, 16, 2, 1.5, False, O.MODEL_SHIFT, 0.0, 0.7, (0, 1, 3), 11),
    (4, 32, 4, 1.5, True, O.MODEL_REFERENCE, 0.02, 0.09, (0, 1, 2), 9),
    (5, 64, 2, 1.9, True, O.MODEL_SHIFT, 0.0, 0.0, (0, 5), 3),
    (2, 32, 2, 1.5, True, O.MODEL_SHIFT, 0.0, 1.0, (6, 1), 1),
    (7, 32, 2, 1.5, True, O.MODEL_REFERENCE, 0.1, 0.2, (3, 0, 3), 20),
    (6, 32, 2, 1.5, True, O.MODEL_SHIFT, 0.0, 0.3, (2, 4), 300),
]


@pytest.mark.parametrize("variant,prec", [("f32_lzcnt", O.PREC_REF32), ("f64_lzcnt", O.PREC_FP64)])
@pytest.mark.parametrize("case", range(len(LIVE_GRID)))
def test_live_reference_parameter_grid(variant, prec, case):
    """Where the reference is compiled here: every event, level sum and inner statistic of the
    oracle equals the reference's over a grid of sampler parameters, including calls that leave
    cores without outer samples and repeated levels (streams persist across calls)."""
    if not O.ref_available(variant):
        pytest.skip("oracle/_ref not built on this host")
    cores, N0, beta, r, anti, kind, tau, K, ells, M = LIVE_GRID[case]
    seed = 1000 + case
    ref = O.Reference(variant)
    ref.init(cores, N0, beta, r, anti)
    ref.model_init(kind, tau, K, seed, traced=True)
    s = O.Sampler(prec, O.STREAMS_CORE, cores, N0, beta, r, anti, False, seed)
    s.set_model(kind, tau, K)
    for ell in ells:
        a = ref.sample(ell, M, events_cap=2_000_000)
        b = s.sample(ell, M, events_cap=2_000_000)
        assert a["events"][0] == b["events"][0], (case, ell)
        np.testing.assert_array_equal(a["events"][1], b["events"][1])
        np.testing.assert_array_equal(a["fsums"], b["fsums"])
        np.testing.assert_array_equal(a["diffsums"], b["diffsums"])
        np.testing.assert_array_equal(a["stats"], b["stats"])
        assert a["work"] == b["work"]


# portfolio (BS options): Q stocks, P options, generator seed, option weights, sub-sampling, delta
# CV, correlation, K, cores, N0, beta, r, levels, M per call
LIVE_PF_GRID = [
    (1, 7, 31, "uniform", O.SUB_UNIFORM, False, 0.0, 0.05, 2, 32, 2, 1.5, (0, 3, 1), 5),
    (6, 90, 32, "w", O.SUB_RANDOM, True, 0.5, 0.2, 5, 32, 4, 1.5, (0, 2), 3),
    (2, 9, 33, "w", O.SUB_NONE, True, 0.9, 0.3, 3, 16, 2, 0.0, (1, 2), 8),
    (3, 40, 34, "uniform", O.SUB_RANDOM, False, 0.1, 0.15, 4, 64, 2, 1.9, (0, 1, 2, 1), 13),
]


@pytest.mark.parametrize("variant,prec", [("f32_lzcnt", O.PREC_REF32), ("f64_lzcnt", O.PREC_FP64)])
@pytest.mark.parametrize("case", range(len(LIVE_PF_GRID)))
def test_live_reference_portfolio_grid(variant, prec, case):
    """Where the reference is compiled here: option start values, delta estimates and every
    event and level sum of the portfolio sampler equal the reference's over a grid of portfolio
    shapes, sub-sampling modes, delta CV, correlations and call sizes."""
    if not O.ref_available(variant):
        pytest.skip("oracle/_ref not built on this host")
    Q, P, g, prob, sub, cv, rho, K, cores, N0, beta, r, ells, M = LIVE_PF_GRID[case]
    pf = O.synthetic_portfolio(Q, P, g, prob=prob)
    seed = 2000 + case
    ref = O.Reference(variant)
    ref.init(cores, N0, beta, r, True)
    st_r, de_r = ref.portfolio_init(pf, r=0.05, rho=rho, max_loss=K, tau=1 / 52, subsample=sub,
                                    use_delta_cv=cv, seed=seed, traced=True)
    s = O.Sampler(prec, O.STREAMS_CORE, cores, N0, beta, r, True, False, seed)
    st_o, de_o = s.set_portfolio(pf, r=0.05, rho=rho, max_loss=K, tau=1 / 52, subsample=sub,
                                 use_delta_cv=cv)
    np.testing.assert_array_equal(st_o, st_r)
    np.testing.assert_array_equal(de_o, de_r)
    for ell in ells:
        a = ref.sample(ell, M, events_cap=2_000_000)
        b = s.sample(ell, M, events_cap=2_000_000)
        assert a["events"][0] == b["events"][0], (case, ell)
        np.testing.assert_array_equal(a["events"][1], b["events"][1])
        np.testing.assert_array_equal(a["events"][2], b["events"][2])
        np.testing.assert_array_equal(a["fsums"], b["fsums"])
        np.testing.assert_array_equal(a["diffsums"], b["diffsums"])
        np.testing.assert_array_equal(a["stats"], b["stats"])


# path-simulated inner values: Q, P, generator seed, sub-sampling, delta CV, coarse CV,
# antithetic risk, Milstein, h0 = 1/dt_h0inv, dt_beta, dt_prob_expo, cores, N0, beta, levels, M
LIVE_METHODS_GRID = [
    (2, 8, 41, O.SUB_NONE, False, False, True, True, 4, 2, -1.5, 2, 32, 2, (0, 1), 6),
    (3, 12, 42, O.SUB_UNIFORM, True, True, False, False, 8, 4, -1.2, 3, 32, 4, (0, 2), 5),
    (2, 10, 43, O.SUB_RANDOM, True, False, True, True, 16, 2, -2.0, 1, 16, 2, (1, 0, 1), 4),
    (4, 9, 44, O.SUB_RANDOM, False, True, True, False, 8, 3, -1.5, 4, 32, 2, (2,), 8),
]


@pytest.mark.parametrize("variant,prec", [("f32_lzcnt", O.PREC_REF32), ("f64_lzcnt", O.PREC_FP64)])
@pytest.mark.parametrize("case", range(len(LIVE_METHODS_GRID)))
def test_live_reference_methods_grid(variant, prec, case):
    """Where the reference is compiled here: mixed BS / Exact / Unbiased portfolios over the
    path-simulation parameters (step sizes, level distribution, Milstein or Euler, antithetic
    risk, coarse delta CV, sub-sampling modes): every event and level sum of the oracle equals
    the reference's."""
    if not O.ref_available(variant):
        pytest.skip("oracle/_ref not built on this host")
    (Q, P, g, sub, cv, ccv, arisk, mil, h0inv, dtb, expo, cores, N0, beta, ells, M) = LIVE_METHODS_GRID[case]
    rng = np.random.default_rng(100 + case)
    pf = O.synthetic_portfolio(Q, P, g, prob="w")
    meth = rng.integers(0, 3, P).astype(np.int32)
    meth[:3] = [0, 1, 2]                                    # every method present
    kw = dict(rho=0.15, max_loss=0.25, subsample=sub, use_delta_cv=cv, use_coarse_delta_cv=ccv,
              use_antithetic_risk=arisk, use_milstein=mil, dt_h0inv=h0inv, dt_beta=dtb,
              dt_prob_expo=expo)
    seed = 3000 + case
    ref = O.Reference(variant)
    ref.init(cores, N0, beta, 1.5, True)
    ref.portfolio_init_methods(pf, meth, seed=seed, **kw)
    s = O.Sampler(prec, O.STREAMS_CORE, cores, N0, beta, 1.5, True, False, seed)
    s.set_portfolio_methods(pf, meth, **kw)
    for ell in ells:
        a = ref.sample(ell, M, events_cap=2_000_000)
        b = s.sample(ell, M, events_cap=2_000_000)
        assert a["events"][0] == b["events"][0], (case, ell)
        np.testing.assert_array_equal(a["events"][1], b["events"][1])
        np.testing.assert_array_equal(a["events"][2], b["events"][2])
        np.testing.assert_array_equal(a["fsums"], b["fsums"])
        np.testing.assert_array_equal(a["diffsums"], b["diffsums"])
        np.testing.assert_array_equal(a["stats"], b["stats"])
        assert a["work"] == b["work"]


def test_alias_table_exact_masses_large_portfolio():
    """The alias table at the large portfolio's size (P = 1e6, prob ~ |w|): integer masses per
    option equal phat_j P 2^32 and sum exactly to P 2^32 (vectorised form of the check above)."""
    P = 1_000_000
    g = np.random.default_rng(7)
    p = np.abs(g.standard_normal(P))
    thr, al, ph = O.build_alias(p)
    unit = np.uint64(1 << 32)
    mass = thr.astype(np.uint64)
    np.add.at(mass, al.astype(np.int64), unit - thr.astype(np.uint64))
    assert int(mass.sum(dtype=np.uint64)) == P * (1 << 32)
    W = np.rint(ph * (P * float(1 << 32))).astype(np.uint64)
    np.testing.assert_array_equal(mass, W)
    np.testing.assert_allclose(ph, p / p.sum(), rtol=0, atol=(P / 2 + 1) / (P * 2.0 ** 32) + 1e-16)
