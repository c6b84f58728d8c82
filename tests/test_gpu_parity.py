"""GPU parity: the CUDA level sampler (through the C ABI) against the CPU oracle and the golden
fixtures of the unmodified reference.

Tolerances (stated here, used below):
  * Threefry2x64-20 blocks: bit-exact.
  * CORE layout (the reference's streams), REF32 and FP64: per-outer-sample inner counts equal
    except where the oracle's adaptive decision (new_count <= cur, get_samples_count) was within
    MARGIN_REF32 = 1e-5 / MARGIN_FP64 = 1e-10 of its threshold in |ln(new_count / cur)|; phi equal
    except where |inner mean| < 1e-5 (REF32) / 1e-12 (FP64) — the GPU's libm and sum order differ
    from glibc's by a few ulp.
  * OUTER layout FP64 / REF32 vs the oracle on the same streams: same rules.
  * OUTER layout FP32 (SFU Box-Muller, Kahan sums) vs FP64 on the same streams: a phi may
    flip only where |inner mean| < FLIP_FP32 = 2e-5 (model) and an adaptive count may differ only
    where the FP64 decision is within MARGIN_FP32 = 1e-4 of its threshold; at most 0.5% of outer
    samples.
  * Level sums: the GPU's and the oracle's moment sums differ by at most what their differing
    outer samples explain (sum over those samples of |phi_gpu^k - phi_oracle^k|, plus 1e-12 per
    outer sample for the order of the double sums); equal traces give equal sums.
"""
import math

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

FLIP_REF32 = 1e-5
FLIP_FP64 = 1e-12
FLIP_FP32 = 2e-5
MARGIN_REF32 = 1e-5
MARGIN_FP64 = 1e-10
MARGIN_FP32 = 1e-4


def nm_prec(o_prec):
    import nmlmc
    return nmlmc.PREC_REF32 if o_prec == O.PREC_REF32 else nmlmc.PREC_FP64


def compare_traces(gpu, ora, bound, per_core=False, max_frac=0.0, margins=None, margin_bound=0.0):
    """Counts equal and phi equal except explained differences: a count may differ only where the
    oracle's adaptive decision was within margin_bound of its threshold (`margins`: the oracle's
    per-outer-sample decision margins; without them a count difference is an error), a phi only
    where its inner mean was within `bound` of the threshold.  In the CORE layout a count
    difference shifts that core's later draws, so comparison of a core stops at its first
    difference."""
    assert len(gpu) == len(ora)
    bad = 0
    stopped = set()
    for m in range(len(gpu)):
        g, o = gpu[m], ora[m]
        core = int(o["core"])
        if per_core and core in stopped:
            continue
        if g["count_f"] != o["count_f"] or g["count_c"] != o["count_c"]:
            assert margins is not None and margins[m] < margin_bound, \
                (m, g, o, None if margins is None else margins[m])
            bad += 1
            if per_core:
                stopped.add(core)
            continue
        assert g["pilots"] == o["pilots"], (m, g, o)    # equal counts: the same pilot rounds
        if g["phi_f"] != o["phi_f"] or g["phi_c"] != o["phi_c"]:
            near = min(abs(o["mean_big"]), o["min_abs_small"])
            assert near < bound, (m, g, o)
            bad += 1
    assert bad <= max_frac * len(gpu) + (2 if max_frac == 0 else 0), bad
    return bad


def assert_sums_explained(gres, ores, f32=False):
    """The GPU's level sums against the oracle's: differences bounded by the outer samples whose
    phi differ (sum of |phi_gpu^k - phi_oracle^k| over them, the powers taken in the sampler's
    real type), plus 1e-12 per outer sample for the order of the double sums."""
    gt, ot = gres["trace"], ores["trace"]
    rt = np.float32 if f32 else np.float64
    M = len(gt)

    def powers(x):
        x = x.astype(rt)
        p, out = np.ones_like(x), []
        for _ in range(4):
            p = (p * x).astype(rt)
            out.append(p.astype(np.float64))
        return out

    for key, gv, ov in (("fsums", gt["phi_f"], ot["phi_f"]),
                        ("diffsums", gt["phi_f"] - gt["phi_c"], ot["phi_f"] - ot["phi_c"])):
        pg, po = powers(gv), powers(ov)
        for k in range(4):
            B = float(np.sum(np.abs(pg[k] - po[k])))
            d = abs(float(gres[key][k]) - float(ores[key][k]))
            assert d <= B + 1e-12 * M, (key, k, d, B)


def make_pair(case, o_prec, streams_o, streams_n, cores=None, seed=None):
    import nmlmc
    cores = cores or case["cores"]
    seed = case["seed"] if seed is None else seed
    s_o = O.Sampler(o_prec, streams_o, cores, case["N0"], case["beta"], case["r"], case["anti"],
                    case.get("incl", False), seed)
    s_g = nmlmc.Sampler(cores=cores, N0=case["N0"], beta=case["beta"], adaptive_r=case["r"],
                        antithetic=case["anti"], adaptive_incl_r2=case.get("incl", False),
                        precision=case.get("gpu_prec", nm_prec(o_prec)), streams=streams_n, seed=seed)
    if case["kind"] == "model":
        s_o.set_model(case["model"], case["tau"], case["max_loss"])
        s_g.set_model(case["model"], case["tau"], case["max_loss"])
    else:
        pf = O.synthetic_portfolio(**case["pf"])
        kw = dict(r=0.05, rho=case["rho"], max_loss=case["max_loss"], tau=1 / 52,
                  subsample=case["sub"], use_delta_cv=case["cv"])
        if "methods" in case:
            flags = dict(use_coarse_delta_cv=case["coarse_cv"], use_antithetic_risk=case["anti_risk"],
                         use_milstein=case["milstein"])
            s_o.set_portfolio_methods(pf, case["methods"], **kw, **flags)
            s_g.set_portfolio(pf, **kw, methods=dict(method=case["methods"], **flags))
            return s_o, s_g
        st_o, de_o = s_o.set_portfolio(pf, **kw)
        st_g, de_g = s_g.set_portfolio(pf, **kw)
        if case.get("gpu_prec", nm_prec(o_prec)) == nm_prec(o_prec):
            np.testing.assert_array_equal(st_g, st_o)  # host set-up: same libm as the reference
            np.testing.assert_array_equal(de_g, de_o)
    return s_o, s_g


def test_threefry_bit_exact(nm, golden):
    _, A = golden
    out = nm.threefry_blocks(A["threefry/ctr"], A["threefry/key"])
    np.testing.assert_array_equal(out, A["threefry/out"])
    rng = np.random.default_rng(5)
    ctr = rng.integers(0, 2**64, (20000, 2), dtype=np.uint64, endpoint=False)
    key = rng.integers(0, 2**64, (20000, 2), dtype=np.uint64, endpoint=False)
    np.testing.assert_array_equal(nm.threefry_blocks(ctr, key), O.threefry(ctr, key))


def test_outer_normals_fp64_and_fp32_bound(nm):
    """OUTER-layout normals: FP64 equals the oracle's to a few ulp; the SFU FP32 Box-Muller stays
    within 4e-6 of FP64."""
    o = O.Sampler(O.PREC_FP64, O.STREAMS_OUTER, 1, 32, 2, 0.0, True, False, 3)
    o.set_model(O.MODEL_SHIFT, 0.0, 1.0)
    n = 1 << 16
    g64 = nm.outer_normals(nm.PREC_FP64, 3, (1 << 56) | 7, 128, n)
    g32 = nm.outer_normals(nm.PREC_FP32, 3, (1 << 56) | 7, 128, n)
    # oracle: the same phase via the word/pair definition (Box-Muller on 32-bit words)
    blocks = O.threefry(np.stack([np.arange(n // 4, dtype=np.uint64), np.full(n // 4, 128, np.uint64)], 1),
                        np.tile(np.array([3, (1 << 56) | 7], np.uint64), (n // 4, 1)))
    words = np.stack([blocks[:, 0] & 0xFFFFFFFF, blocks[:, 0] >> 32,
                      blocks[:, 1] & 0xFFFFFFFF, blocks[:, 1] >> 32], 1).reshape(-1).astype(np.float64)
    u0 = words[0::2]
    u1 = words[1::2]
    a = np.where(u0 >= 2**31, u0 - 2**32, u0) * 2.0**-31 + 2.0**-32
    rr = np.sqrt(-2 * np.log(u1 * 2.0**-32 + 2.0**-33))
    ref = np.stack([np.sin(np.pi * a) * rr, np.cos(np.pi * a) * rr], 1).reshape(-1)
    assert np.max(np.abs(g64 - ref)) < 1e-13
    assert np.max(np.abs(g32 - g64)) < 4e-6


@pytest.mark.parametrize("prec_name,o_prec", [("f32", O.PREC_REF32), ("f64", O.PREC_FP64)])
def test_core_layout_matches_reference(nm, golden, prec_name, o_prec):
    """CORE layout at the golden cases: level sums/stats of the reference, per-outer traces of the
    oracle."""
    meta, _ = golden
    bound = FLIP_REF32 if o_prec == O.PREC_REF32 else FLIP_FP64
    for case in meta["engine"]:
        res = case["results"][prec_name]
        s_o, s_g = make_pair(case, o_prec, O.STREAMS_CORE, nm.STREAMS_CORE)
        margin = MARGIN_REF32 if o_prec == O.PREC_REF32 else MARGIN_FP64
        for call in res["calls"]:
            go = s_o.sample(call["ell"], call["M"], trace=True, margins=True)
            gg = s_g.sample(call["ell"], call["M"], trace=True)
            bad = compare_traces(gg["trace"], go["trace"], bound, per_core=True, margins=go["margins"],
                                 margin_bound=margin)
            assert_sums_explained(gg, go, f32=o_prec == O.PREC_REF32)
            if bad == 0:
                np.testing.assert_array_equal(gg["fsums"], call["fsums"], err_msg=case["name"])
                np.testing.assert_array_equal(gg["diffsums"], call["diffsums"], err_msg=case["name"])
                np.testing.assert_array_equal(gg["stats"].astype(np.int64), call["stats"], err_msg=case["name"])
                assert gg["work"] == call["work"], case["name"]


def test_reference_named_surface(nm, golden):
    """init_nestedmc_sampler / model_init / model_sample reproduce golden case A (float build)."""
    meta, _ = golden
    case = meta["engine"][0]
    res = case["results"]["f32"]
    p = nm.NestedSamplerParams(case["N0"], case["beta"], case["anti"], 4, 4, case["r"])
    nm.init_nestedmc_sampler(case["cores"], p)
    tau = np.float32(case["tau"])
    md = nm.ModelData(float(np.sqrt(tau)), float(np.sqrt(np.float32(1) - tau)), case["max_loss"], 0)
    nm.model_init(md, case["seed"])
    try:
        for call in res["calls"]:
            out = nm.model_sample(call["ell"], call["M"])
            assert out["M"] == call["M"]
            np.testing.assert_array_equal(out["fsums"], call["fsums"])
            np.testing.assert_array_equal(out["diffsums"], call["diffsums"])
            np.testing.assert_array_equal(out["stats"].astype(np.int64), call["stats"])
    finally:
        nm.cleanup_nestedmc_sampler()


def test_reference_named_portfolio_surface(nm, golden):
    meta, _ = golden
    case = meta["engine"][5]
    assert case["name"] == "F_pf_uniform"
    res = case["results"]["f32"]
    pf = O.synthetic_portfolio(**case["pf"])
    p = nm.NestedSamplerParams(case["N0"], case["beta"], case["anti"], 4, 4, case["r"])
    nm.init_nestedmc_sampler(case["cores"], p)
    d, keep = nm.make_portfolio_data(pf, r=0.05, rho=case["rho"], max_loss=case["max_loss"],
                                     tau=1 / 52, subsample=case["sub"], use_delta_cv=case["cv"])
    nm.portfolio_comp_params(d)
    nm.portfolio_init(d, case["seed"])
    try:
        for call in res["calls"]:
            out = nm.portfolio_sample(call["ell"], 0, call["M"])
            np.testing.assert_array_equal(out["fsums"], call["fsums"])
            np.testing.assert_array_equal(out["diffsums"], call["diffsums"])
    finally:
        nm.portfolio_cleanup()
        nm.cleanup_nestedmc_sampler()


def test_reference_named_portfolio_surface_methods(nm, golden):
    """portfolio_init with options[1] (Exact) and options[2] (Unbiased): golden case J."""
    meta, _ = golden
    case = next(c for c in meta["engine"] if c["name"] == "J_pf_methods_cdf_cv")
    res = case["results"]["f32"]
    pf = O.synthetic_portfolio(**case["pf"])
    p = nm.NestedSamplerParams(case["N0"], case["beta"], case["anti"], 4, 4, case["r"])
    nm.init_nestedmc_sampler(case["cores"], p)
    d, keep = nm.make_portfolio_data(pf, r=0.05, rho=case["rho"], max_loss=case["max_loss"],
                                     tau=1 / 52, subsample=case["sub"], use_delta_cv=case["cv"],
                                     method=case["methods"], use_coarse_delta_cv=case["coarse_cv"],
                                     use_antithetic_risk=case["anti_risk"], use_milstein=case["milstein"])
    nm.portfolio_comp_params(d)
    nm.portfolio_init(d, case["seed"])
    try:
        for call in res["calls"]:
            out = nm.portfolio_sample(call["ell"], 0, call["M"])
            np.testing.assert_array_equal(out["fsums"], call["fsums"])
            np.testing.assert_array_equal(out["diffsums"], call["diffsums"])
            assert out["work"] == call["work"]
    finally:
        nm.portfolio_cleanup()
        nm.cleanup_nestedmc_sampler()


OUTER_CASES = [
    dict(name="shift_r15", kind="model", model=1, tau=0.0, max_loss=1.0, cores=1, N0=32, beta=2,
         r=1.5, anti=True, seed=3, calls=[(0, 3000), (1, 2000), (3, 2000), (6, 1500), (9, 600)]),
    dict(name="shift_r2", kind="model", model=1, tau=0.0, max_loss=1.0, cores=1, N0=32, beta=2,
         r=2.0, incl=True, anti=True, seed=4, calls=[(2, 2000), (5, 1500), (10, 500)]),
    dict(name="refmodel_b4", kind="model", model=0, tau=0.02, max_loss=0.09, cores=1, N0=32, beta=4,
         r=1.5, anti=True, seed=5, calls=[(0, 2000), (1, 1000), (3, 400), (5, 100)]),
    dict(name="shift_nonadapt", kind="model", model=1, tau=0.0, max_loss=1.0, cores=1, N0=32, beta=2,
         r=0.0, anti=True, seed=6, calls=[(0, 5000), (4, 1000), (8, 200)]),
    dict(name="pf_uniform", kind="portfolio", pf=dict(Q=6, P=300, seed=3, prob="uniform"),
         sub=O.SUB_UNIFORM, cv=False, rho=0.0, max_loss=2.0, cores=1, N0=64, beta=2, r=1.5, anti=True,
         seed=7, calls=[(0, 1000), (2, 800), (5, 300)]),
    dict(name="pf_cdf_cv", kind="portfolio", pf=dict(Q=4, P=200, seed=4, prob="w"),
         sub=O.SUB_RANDOM, cv=True, rho=0.3, max_loss=1.0, cores=1, N0=32, beta=4, r=1.5, anti=True,
         seed=8, calls=[(0, 800), (1, 500), (3, 100)]),
]


@pytest.mark.parametrize("case", OUTER_CASES, ids=[c["name"] for c in OUTER_CASES])
@pytest.mark.parametrize("o_prec", [O.PREC_FP64, O.PREC_REF32], ids=["fp64", "ref32"])
def test_outer_layout_matches_oracle(nm, case, o_prec):
    bound = FLIP_REF32 if o_prec == O.PREC_REF32 else FLIP_FP64
    s_o, s_g = make_pair(case, o_prec, O.STREAMS_OUTER, nm.STREAMS_OUTER)
    margin = MARGIN_REF32 if o_prec == O.PREC_REF32 else MARGIN_FP64
    for ell, M in case["calls"]:
        go = s_o.sample(ell, M, trace=True, margins=True)
        gg = s_g.sample(ell, M, trace=True)
        bad = compare_traces(gg["trace"], go["trace"], bound, max_frac=0.001, margins=go["margins"],
                             margin_bound=margin)
        assert_sums_explained(gg, go, f32=o_prec == O.PREC_REF32)
        if bad == 0:
            np.testing.assert_array_equal(gg["fsums"], go["fsums"])
            np.testing.assert_array_equal(gg["diffsums"], go["diffsums"])
            assert gg["stats"][0] == go["stats"][0]


@pytest.mark.parametrize("case", OUTER_CASES, ids=[c["name"] for c in OUTER_CASES])
def test_fp32_against_fp64_same_streams(nm, case):
    """Batched FP32 (SFU Box-Muller, Kahan sums) against all-FP64 on the same OUTER streams."""
    c32 = dict(case, gpu_prec=nm.PREC_FP32)
    _, s32 = make_pair(c32, O.PREC_FP64, O.STREAMS_OUTER, nm.STREAMS_OUTER)
    s_o = O.Sampler(O.PREC_FP64, O.STREAMS_OUTER, 1, case["N0"], case["beta"], case["r"], case["anti"],
                    case.get("incl", False), case["seed"])
    if case["kind"] == "model":
        s_o.set_model(case["model"], case["tau"], case["max_loss"])
    else:
        s_o.set_portfolio(O.synthetic_portfolio(**case["pf"]), r=0.05, rho=case["rho"],
                          max_loss=case["max_loss"], tau=1 / 52, subsample=case["sub"],
                          use_delta_cv=case["cv"])
    scale = 1.0 if case["kind"] == "model" else 1e3
    for ell, M in case["calls"]:
        go = s_o.sample(ell, M, trace=True, margins=True)
        gg = s32.sample(ell, M, trace=True)
        compare_traces(gg["trace"], go["trace"], FLIP_FP32 * scale, max_frac=0.005, margins=go["margins"],
                       margin_bound=MARGIN_FP32)
        assert_sums_explained(gg, go, f32=True)


def test_edge_cases(nm):
    s = nm.Sampler(precision=nm.PREC_FP32, streams=nm.STREAMS_OUTER, N0=32, beta=2, adaptive_r=1.5)
    s.set_model(nm.MODEL_SHIFT, 0.0, 1.0)
    r0 = s.sample(3, 0)
    assert r0["M"] == 0 and not np.any(r0["fsums"])
    r1 = s.sample(0, 1)
    assert r1["M"] == 1 and r1["stats"][0] == 32
    # CORE layout with fewer outer samples than cores: idle cores contribute nothing
    c = nm.Sampler(precision=nm.PREC_REF32, streams=nm.STREAMS_CORE, cores=64, N0=32, beta=2)
    c.set_model(nm.MODEL_SHIFT, 0.0, 1.0)
    rc = c.sample(2, 5)
    assert rc["stats"][1] == 5
    # invalid configurations are errors, not silent fallbacks
    with pytest.raises(nm.NmlmcError):
        nm.Sampler(precision=nm.PREC_FP32, streams=nm.STREAMS_CORE)
    with pytest.raises(nm.NmlmcError):
        nm.Sampler(streams=nm.STREAMS_OUTER, antithetic=False)
    with pytest.raises(nm.NmlmcError):
        s.sample(40, 10)            # counts beyond 32-bit per-item counters
    with pytest.raises(nm.NmlmcError):
        s.set_portfolio(dict(S0=[100.0], mu=[0.05], sigma=[0.2], strike=[100.0], maturity=[1.0],
                             w=[1.0], prob=[1.0], stock_ind=[3], type=[1]))


def test_batch_split_is_invisible(nm):
    """OUTER layout: the same outer samples give the same sums whatever the batch size."""
    a = nm.Sampler(precision=nm.PREC_FP32, N0=32, beta=2, adaptive_r=1.5, seed=2, batch=1 << 20)
    b = nm.Sampler(precision=nm.PREC_FP32, N0=32, beta=2, adaptive_r=1.5, seed=2, batch=777)
    for s in (a, b):
        s.set_model(nm.MODEL_SHIFT, 0.0, 1.0)
    ra = a.sample(5, 5000, trace=True)
    rb = b.sample(5, 5000, trace=True)
    np.testing.assert_array_equal(ra["trace"], rb["trace"])
    np.testing.assert_array_equal(ra["fsums"], rb["fsums"])


def test_full_loss_matches_oracle(nm):
    pf = O.synthetic_portfolio(8, 500, 11, "uniform")
    s_g = nm.Sampler(precision=nm.PREC_FP64, N0=64, beta=2, seed=1)
    s_g.set_portfolio(pf, rho=0.2, max_loss=1.0)
    s_o = O.Sampler(O.PREC_FP64, O.STREAMS_OUTER, 1, 64, 2, 0.0, True, False, 1)
    s_o.set_portfolio(pf, rho=0.2, max_loss=1.0)
    np.testing.assert_allclose(s_g.full_loss(0, 100, 300), s_o.full_loss(0, 100, 300), rtol=1e-12, atol=1e-9)


def test_model_problem_closed_form(nm):
    """MLMC on the X = Y + Z model lands within eps of 1 - Phi(1)."""
    eps = 2e-3
    s = nm.Sampler(precision=nm.PREC_FP32, N0=32, beta=2, adaptive_r=2.0, adaptive_incl_r2=True, seed=12)
    s.set_model(nm.MODEL_SHIFT, 0.0, 1.0)
    out = s.mlmc_run(targetTOL=eps, M0=1024, batched=True)
    exact = 0.5 * math.erfc(1 / math.sqrt(2))
    assert abs(out["Eg"] - exact) < 3 * eps, (out["Eg"], exact)
