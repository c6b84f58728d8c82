"""The host continuation-MLMC driver (nmlmc_mlmc_run_cb) against the reference's mlmc_t::run on
the same deterministic synthetic level sampler (golden fixtures): identical sequence of
sample_level(ell, M) calls, level sums, error split and the to_string() table text."""
import math

import numpy as np
import pytest


class Synthetic:
    """The synthetic level sampler of oracle/ref_harness.cpp (ref_mlmc_synthetic), restated."""

    def __init__(self, a, alpha, v, beta, w, gamma, seed):
        self.a, self.alpha, self.v, self.beta, self.w, self.gamma = a, alpha, v, beta, w, gamma
        self.state = seed
        self.calls = []

    def _next(self):
        M64 = (1 << 64) - 1
        self.state = (self.state + 0x9E3779B97F4A7C15) & M64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        z ^= z >> 31
        return float(z >> 11) * (1.0 / 9007199254740992.0)

    def __call__(self, ell, M):
        self.calls.append((ell, M))
        mf = self.a * math.pow(2.0, -self.alpha * ell) + 0.1
        md = 0.0 if ell == 0 else self.a * math.pow(2.0, -self.alpha * ell)
        sd_f = math.sqrt(self.v)
        sd_d = math.sqrt(self.v * math.pow(2.0, -self.beta * ell))
        n = M if M < 64 else 64
        f_s = [0.0] * 4
        d_s = [0.0] * 4
        for _ in range(n):
            u = (self._next() - 0.5) * math.sqrt(12.0)
            f = mf + sd_f * u
            d = md + sd_d * u
            pf = pd = 1.0
            for j in range(4):
                pf *= f
                pd *= d
                f_s[j] += pf * (float(M) / n)
                d_s[j] += (0.0 if ell == 0 else pd * (float(M) / n))
        return dict(fsums=f_s, diffsums=d_s, work=self.w * math.pow(2.0, self.gamma * ell) * M)


@pytest.mark.parametrize("idx", [0, 1, 2])
def test_driver_matches_reference(nm, golden, idx):
    meta, _ = golden
    g = meta["mlmc"][idx]
    tol, M0, a, alpha, v, beta, w, gamma, seed = g["args"]
    syn = Synthetic(a, alpha, v, beta, w, gamma, int(seed))
    out = nm.mlmc_run_cb(syn, targetTOL=tol, M0=int(M0), verbose=False)
    assert [c[0] for c in syn.calls] == g["calls_ell"]
    assert [c[1] for c in syn.calls] == g["calls_M"]
    lv = np.array(g["levels"])
    assert out["nlevels"] == len(lv)
    np.testing.assert_array_equal(out["level_fsums"], lv[:, 0:4])
    np.testing.assert_array_equal(out["level_diffsums"], lv[:, 4:8])
    np.testing.assert_array_equal(out["level_work"], lv[:, 8])
    np.testing.assert_array_equal(out["level_M"].astype(float), lv[:, 9])
    assert out["starting_level"] == g["misc"][0]
    assert out["bias_est"] == g["misc"][1]
    assert out["stat_error"] == g["misc"][2]
    assert out["TOL"] == g["misc"][3]
    assert out["table"] == g["table"]


def test_batched_driver_same_decisions(nm, golden):
    """Batched submissions (all levels of a round at once) take the same decisions when the
    sampler's results do not depend on call order."""
    meta, _ = golden
    tol, M0, a, alpha, v, beta, w, gamma, seed = meta["mlmc"][1]["args"]

    def det(ell, M):   # order-independent sampler: a pure function of (ell, M)
        mf = a * 2.0 ** (-alpha * ell) + 0.1
        md = 0.0 if ell == 0 else a * 2.0 ** (-alpha * ell)
        vf, vd = v, v * 2.0 ** (-beta * ell)
        f = [M * mf, M * (vf + mf * mf), M * mf ** 3, M * mf ** 4]
        d = [0.0] * 4 if ell == 0 else [M * md, M * (vd + md * md), M * md ** 3, M * md ** 4]
        return dict(fsums=f, diffsums=d, work=w * 2.0 ** (gamma * ell) * M)

    r1 = nm.mlmc_run_cb(det, targetTOL=tol, M0=int(M0), batched=False)
    r2 = nm.mlmc_run_cb(det, targetTOL=tol, M0=int(M0), batched=True)
    np.testing.assert_array_equal(r1["level_M"], r2["level_M"])
    assert r1["Eg"] == r2["Eg"]


# tol, M0, a, alpha, v, beta, w, gamma, seed: variance decay faster / slower than cost growth,
# tiny and large M0, loose and tight tolerances, added levels and a starting level that moves up
LIVE_DRIVER_GRID = [
    (5e-2, 10, 1.0, 1.0, 0.5, 2.0, 1.0, 1.0, 11),
    (2e-3, 1000, 0.4, 1.5, 0.2, 1.0, 1.0, 2.0, 12),
    (5e-3, 20, 2.0, 0.5, 1.0, 1.5, 0.5, 1.0, 13),
    (1e-3, 200, 0.2, 1.0, 0.01, 3.0, 2.0, 1.0, 14),
    (8e-3, 64, 0.6, 2.0, 0.3, 2.0, 1.0, 3.0, 15),
    (1e-2, 100, 0.5, 1.0, 0.3, 0.3, 1.0, 0.5, 17),     # slow variance decay: starting level 8
    (5e-3, 100, 0.8, 1.2, 0.2, 0.5, 1.0, 0.8, 18),     # starting level 3
]


@pytest.mark.parametrize("case", range(len(LIVE_DRIVER_GRID)))
def test_driver_matches_live_reference(nm, case):
    """Where the reference is compiled here: its mlmc_t<double, 4>::run and this driver take the
    same calls, sums, error split and print the same table over a grid of problems."""
    import oracle as O
    if not O.ref_available("f64"):
        pytest.skip("oracle/_ref not built on this host")
    tol, M0, a, alpha, v, beta, w, gamma, seed = LIVE_DRIVER_GRID[case]
    ref = O.Reference("f64").mlmc_synthetic(tol, M0, a, alpha, v, beta, w, gamma, seed)
    syn = Synthetic(a, alpha, v, beta, w, gamma, seed)
    out = nm.mlmc_run_cb(syn, targetTOL=tol, M0=M0, verbose=False)
    assert [c[0] for c in syn.calls] == ref["calls_ell"].tolist()
    assert [c[1] for c in syn.calls] == ref["calls_M"].tolist()
    lv = ref["levels"]
    assert out["nlevels"] == len(lv)
    np.testing.assert_array_equal(out["level_fsums"], lv[:, 0:4])
    np.testing.assert_array_equal(out["level_diffsums"], lv[:, 4:8])
    np.testing.assert_array_equal(out["level_M"].astype(float), lv[:, 9])
    assert [out["starting_level"], out["bias_est"], out["stat_error"], out["TOL"]] == list(ref["misc"][:4])
    assert out["table"] == ref["table"]


def test_level_cap(nm):
    """A bias that never decays (difference variance and mean constant over levels) would add
    levels for good: the driver stops with NMLMC_ERR_ARG at max_levels, or at the 64 levels the
    output and checkpoint arrays hold."""
    syn = Synthetic(0.5, 1.0, 0.5, 0.0, 1.0, 1.0, 16)
    with pytest.raises(nm.NmlmcError) as e:
        nm.mlmc_run_cb(syn, targetTOL=2e-2, M0=50, verbose=False, max_levels=5)
    assert e.value.status == nm.ERR_ARG and max(c[0] for c in syn.calls) == 4
    syn = Synthetic(0.5, 1.0, 0.5, 0.0, 1.0, 1.0, 16)
    with pytest.raises(nm.NmlmcError) as e:
        nm.mlmc_run_cb(syn, targetTOL=2e-2, M0=50, verbose=False)
    assert e.value.status == nm.ERR_ARG and max(c[0] for c in syn.calls) == 63


@pytest.mark.parametrize("bad", [dict(M0=0), dict(theta=0.0), dict(theta=1.0), dict(Ca=0.0),
                                 dict(startTOL=float("inf")), dict(targetTOL=float("nan")),
                                 dict(targetTOL=0.0), dict(startTOL=1e-4)])
def test_driver_rejects_inputs_it_cannot_finish(nm, bad):
    """theta = 0 or 1 asks for a zero statistical error or bias (the loop would never end), M0 = 0
    samples nothing, non-finite tolerances break the TOL sequence: NMLMC_ERR_ARG before any call."""
    syn = Synthetic(0.5, 1.0, 0.5, 1.5, 1.0, 1.0, 3)
    kw = dict(targetTOL=1e-2, M0=50, verbose=False)
    kw.update(bad)
    with pytest.raises(nm.NmlmcError) as e:
        nm.mlmc_run_cb(syn, **kw)
    assert e.value.status == nm.ERR_ARG and syn.calls == []


@pytest.mark.parametrize("key,level", [("diffsums", 1), ("fsums", 0), ("fsums", 2)])
def test_non_finite_level_results_stop_the_run(nm, key, level):
    """A sampler that returns a non-finite sum stops the run with NMLMC_ERR_STATE at that call,
    instead of turning into NaN sample counts (an absurd next request) or a silent NaN estimate."""
    syn = Synthetic(0.5, 1.0, 0.5, 1.5, 1.0, 1.0, 3)
    calls = []

    def bad(ell, M):
        calls.append((ell, M))
        assert M < 10**8, "absurd sample request"
        r = syn(ell, M)
        if ell == level:
            r[key][1] = float("nan")
        return r

    with pytest.raises(nm.NmlmcError) as e:
        nm.mlmc_run_cb(bad, targetTOL=1e-2, M0=50, verbose=False)
    assert e.value.status == nm.ERR_STATE and e.value.__cause__ is None
    assert calls[-1][0] == level


def test_sample_count_beyond_range_is_an_error(nm):
    """A tolerance no run can reach on this problem (over 2^62 samples on a level) is reported,
    not converted into a wrapped integer request."""
    syn = Synthetic(0.5, 1.0, 1e30, 1.5, 1.0, 1.0, 3)
    with pytest.raises(nm.NmlmcError) as e:
        nm.mlmc_run_cb(syn, targetTOL=1e-12, startTOL=1e-12, M0=50, verbose=False)
    assert e.value.status == nm.ERR_ARG


def test_tolerance_ratio_beyond_2_to_31(nm):
    """startTOL / targetTOL >= 2^31: the TOL sequence still starts near startTOL (the reference's
    targetTOL * (1 << k) is undefined from k = 31 on)."""
    syn = Synthetic(0.5, 1.0, 0.5, 1.5, 1.0, 1.0, 3)
    out = nm.mlmc_run_cb(syn, targetTOL=1e-11, startTOL=0.5, M0=50, verbose=False, max_iterations=1)
    assert out["iterations_done"] == 1 and not out["complete"]
    assert 0.5 / 2 ** 1.5 < out["TOL"] < 0.5
