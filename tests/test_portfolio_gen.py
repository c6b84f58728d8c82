"""The portfolio generators of libnmlmc.so (host code, no device needed):

* the reference demo main's (portfolio_gen_data / portfolio_free_data, portfolio_sampler.cpp:
  784-912): byte-identical to the compiled reference for the same arguments, and its argument
  checks;
* the benchmark's (nmlmc_portfolio_generate): every field recomputed from the oracle's Threefry."""
import ctypes
import os

import numpy as np
import pytest

import oracle as O

OPTION_FIELDS = ("strike", "maturity", "start", "w", "delta_est", "stock_ind", "type", "prob", "W_est")
SCALARS = ("r", "rho", "s1_rho2", "max_loss", "tau", "dt_h0inv", "dt_beta", "dt_prob_expo",
           "phi_type", "_phi_size", "subsample", "use_delta_cv", "use_coarse_delta_cv",
           "use_antithetic_risk", "use_milstein")


def _bind(nm, L):
    L.portfolio_gen_data.restype = nm.PortfolioData
    L.portfolio_gen_data.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64,
                                     ctypes.POINTER(ctypes.c_double), ctypes.c_bool, ctypes.c_bool]
    L.portfolio_free_data.restype = None
    L.portfolio_free_data.argtypes = [ctypes.POINTER(nm.PortfolioData)]
    return L


def _dump(d):
    """Scalars and every option / stock record as raw bytes (bit-exact comparison)."""
    out = {k: getattr(d, k) for k in SCALARS}
    for m in range(3):
        n = d.options[m].size
        out[f"options{m}"] = ctypes.string_at(d.options[m].data, n * ctypes.sizeof(d.options[m].data._type_)) if n else b""
        out[f"n{m}"] = n
    out["stocks"] = ctypes.string_at(d.stocks.data, d.stocks.size * 12)
    return out


CASES = [   # P, Q, seed, probs, uniform_weights, uniform_prob
    (100, 10, 0, (1.0, 0.0, 0.0), False, False),
    (1000, 20, 42, (0.3, 0.5, 0.2), False, False),     # the reference main's method fractions
    (64, 32, 7, (0.5, 0.25, 0.25), False, True),
    (500, 3, 2**40 + 5, (0.2, 0.2, 0.6), False, False),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_generator_matches_the_reference(nm, case):
    if not O.ref_available("f32"):
        pytest.skip("oracle/_ref not built on this host")
    P, Q, seed, probs, uw, up = CASES[case]
    pr = (ctypes.c_double * 3)(*probs)
    ours = _bind(nm, nm.lib())
    ref = _bind(nm, ctypes.CDLL(os.path.join(O.REF_DIR, "libref_f32.so")))
    a = ours.portfolio_gen_data(P, Q, seed, pr, uw, up)
    assert nm.lib().nmlmc_last_error() == nm.OK
    b = ref.portfolio_gen_data(P, Q, seed, pr, uw, up)
    da, db = _dump(a), _dump(b)
    for k in SCALARS:
        assert da[k] == db[k], k
    assert da["stocks"] == db["stocks"]
    for m in range(3):
        assert da[f"n{m}"] == db[f"n{m}"]
        assert da[f"options{m}"] == db[f"options{m}"], f"method {m}"
    w = np.array([a.options[m].data[j].w for m in range(3) for j in range(a.options[m].size)])
    assert np.isfinite(w).all() and abs(w.sum() - 1) < 1e-4
    ours.portfolio_free_data(ctypes.byref(a))
    ref.portfolio_free_data(ctypes.byref(b))
    assert not a.stocks.data and a.options[0].size == 0


def test_generator_arguments(nm):
    L = _bind(nm, nm.lib())
    pr = (ctypes.c_double * 3)(0.5, 0.5, 0.0)
    d = L.portfolio_gen_data(10, 6, 1, pr, False, False)        # P < 2Q
    assert nm.lib().nmlmc_last_error() == nm.ERR_ARG and not d.stocks.data
    d = L.portfolio_gen_data(10, 2, 1, (ctypes.c_double * 3)(0.3, 0.3, 0.3), False, False)   # 9 != 10
    assert nm.lib().nmlmc_last_error() == nm.ERR_ARG and not d.stocks.data
    d = L.portfolio_gen_data(10, 2, 1, None, False, False)
    assert nm.lib().nmlmc_last_error() == nm.ERR_ARG
    d = L.portfolio_gen_data(40, 4, 3, pr, True, False)          # weights start at 1
    assert nm.lib().nmlmc_last_error() == nm.OK
    w = np.array([d.options[m].data[j].w for m in range(3) for j in range(d.options[m].size)])
    assert np.isfinite(w).all() and abs(w.sum() - 1) < 1e-5
    L.portfolio_free_data(ctypes.byref(d))
    L.portfolio_free_data(None)
    assert nm.lib().nmlmc_last_error() == nm.ERR_ARG


def test_benchmark_generator_against_the_oracle_threefry(nm):
    """nmlmc_portfolio_generate (host code, no device): every field is the documented function of
    Threefry2x64-20 blocks, recomputed here with the oracle's Threefry (itself pinned to Random123):
    value(field f, index i) = Threefry(ctr = (i, f), key = (seed, 'PORTGEN'))."""
    spec = dict(nm.PORTFOLIO_C2, Q=7, P=300)
    seed = 11
    pf = nm.generate_portfolio(spec, seed)
    key = np.array([seed, 0x4E454754524F50], np.uint64)

    def blocks(field, n):
        ctr = np.stack([np.arange(n, dtype=np.uint64), np.full(n, field, np.uint64)], axis=1)
        return O.threefry(ctr, np.tile(key, (n, 1)))

    def u01(words):
        return ((words >> np.uint64(11)).astype(np.float64) + 0.5) * 2.0 ** -53

    Q, P = spec["Q"], spec["P"]
    sig = spec["sigma_lo"] + (spec["sigma_hi"] - spec["sigma_lo"]) * u01(blocks(1, Q)[:, 0])
    np.testing.assert_array_equal(pf["sigma"], sig)
    stock = np.array([(int(v) * Q) >> 64 for v in blocks(2, P)[:, 0]], np.uint32)
    np.testing.assert_array_equal(pf["stock_ind"], stock)
    typ = np.where(u01(blocks(3, P)[:, 0]) < spec["call_fraction"], 1, -1)
    np.testing.assert_array_equal(pf["type"], typ)
    strike = spec["S0"] * (spec["strike_lo"] + (spec["strike_hi"] - spec["strike_lo"]) * u01(blocks(4, P)[:, 0]))
    np.testing.assert_array_equal(pf["strike"], strike)
    mat = spec["maturity_lo"] + (spec["maturity_hi"] - spec["maturity_lo"]) * u01(blocks(5, P)[:, 0])
    np.testing.assert_array_equal(pf["maturity"], mat)
    wb = blocks(6, P)
    w = np.sqrt(-2.0 * np.log(u01(wb[:, 0]))) * np.cos(2.0 * np.pi * u01(wb[:, 1]))
    np.testing.assert_allclose(pf["w"], w, rtol=1e-13, atol=1e-15)
    np.testing.assert_array_equal(pf["S0"], np.full(Q, spec["S0"]))


def test_comp_params_and_layout_helpers(nm):
    """make_portfolio_data builds the reference's portfolio_data layout from SoA arrays (options
    grouped by method, in order); the exported portfolio_comp_params fills start / delta_est like
    the compiled reference's on the same struct; make_batch concatenates with offsets."""
    pf = O.synthetic_portfolio(5, 60, 17, prob="w")
    meth = np.array([0, 1, 2] * 20, np.int32)
    d, keep = nm.make_portfolio_data(pf, rho=0.2, max_loss=0.3, method=meth)
    assert [d.options[m].size for m in range(3)] == [20, 20, 20] and d.stocks.size == 5
    for m in range(3):
        for k, j in enumerate(np.flatnonzero(meth == m)):
            assert d.options[m].data[k].strike == np.float32(pf["strike"][j])
    L = nm.lib()
    L.portfolio_comp_params.argtypes = [ctypes.POINTER(nm.PortfolioData)]
    L.portfolio_comp_params(ctypes.byref(d))
    ours = b"".join(ctypes.string_at(d.options[m].data, ctypes.sizeof(nm.OptionParams) * d.options[m].size) for m in range(3))
    if O.ref_available("f32"):
        e, keep2 = nm.make_portfolio_data(pf, rho=0.2, max_loss=0.3, method=meth)
        R = ctypes.CDLL(os.path.join(O.REF_DIR, "libref_f32.so"))
        R.portfolio_comp_params.argtypes = [ctypes.POINTER(nm.PortfolioData)]
        R.portfolio_comp_params(ctypes.byref(e))
        theirs = b"".join(ctypes.string_at(e.options[m].data, ctypes.sizeof(nm.OptionParams) * e.options[m].size) for m in range(3))
        assert ours == theirs
    starts = [d.options[m].data[k].start for m in range(3) for k in range(d.options[m].size)]
    assert np.all(np.isfinite(starts)) and np.all(np.array(starts) >= 0)
    b = nm.make_batch([pf, O.synthetic_portfolio(2, 7, 18)], [1.0, 2.0])
    assert list(b["stock_off"]) == [0, 5, 7] and list(b["option_off"]) == [0, 60, 67]
    assert len(b["strike"]) == 67 and list(b["K"]) == [1.0, 2.0]
