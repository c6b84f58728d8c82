"""Phase-kernel autotuner of the batched FP32 path (nmlmc_set_autotune / nmlmc_autotune_level /
nmlmc_get_phase_config / nmlmc_set_phase_config).

* The register/occupancy variants (the portfolio's pipelined one included) run the same
  arithmetic: bit-identical level sums and per-outer-sample traces on the same streams.
* Tuning probes use stream indices far from the real ones: a tuned call returns exactly what the
  same configuration returns when pinned in a context that never tuned.
* Another chunk length regroups the FP32 compensated inner sums: results stay within the FP32
  bound of the all-FP64 run on the same streams.
"""
import numpy as np
import pytest

import oracle as O
from test_gpu_parity import FLIP_FP32, compare_traces

pytestmark = pytest.mark.gpu


def _model(nm, autotune=1, seed=3, N0=32):
    s = nm.Sampler(N0=N0, beta=2, adaptive_r=1.5, precision=nm.PREC_FP32, streams=nm.STREAMS_OUTER, seed=seed)
    s.set_model(nm.MODEL_SHIFT, 0.0, 1.0)
    s.set_autotune(autotune)
    return s


def _portfolio(nm, autotune=1, seed=5):
    s = nm.Sampler(N0=64, beta=2, adaptive_r=1.5, precision=nm.PREC_FP32, streams=nm.STREAMS_OUTER, seed=seed)
    s.set_portfolio(O.synthetic_portfolio(6, 400, 9, prob="w"), rho=0.2, max_loss=1.0,
                    subsample=nm.SUB_RANDOM, use_delta_cv=True)
    s.set_autotune(autotune)
    return s


def _same(a, b):
    np.testing.assert_array_equal(a["fsums"], b["fsums"])
    np.testing.assert_array_equal(a["diffsums"], b["diffsums"])
    np.testing.assert_array_equal(a["stats"], b["stats"])
    assert a["work"] == b["work"]


@pytest.mark.parametrize("kind", ["model", "portfolio"])
def test_variants_are_bit_identical(nm, kind):
    ell, M = (6, 6000) if kind == "model" else (4, 3000)
    ref = None
    for v in (0, 1, 2, 3):                      # 3: the portfolio's pipelined variant (variant 0 elsewhere)
        s = _model(nm, autotune=0) if kind == "model" else _portfolio(nm, autotune=0)
        s.set_phase_config(ell, variant=v)
        assert s.phase_config(ell)["state"] == nm.PHASE_PINNED and s.phase_config(ell)["variant"] == v
        r = s.sample(ell, M, trace=True)
        if ref is None:
            ref = r
        else:
            _same(r, ref)
            np.testing.assert_array_equal(r["trace"], ref["trace"])


def test_default_configuration(nm):
    m, p = _model(nm, autotune=0), _portfolio(nm, autotune=0)
    assert m.phase_config(3) == dict(variant=1, chunk=32, state=nm.PHASE_DEFAULT, probe_ms=0.0)
    assert p.phase_config(3)["variant"] == 2 and p.phase_config(3)["chunk"] == 32


def test_automatic_tuning_leaves_results_unchanged(nm):
    """A call large enough to time tunes its level first; the probe does not touch the result."""
    ell, M = 2, 1 << 17
    a = _model(nm, autotune=1)
    assert a.phase_config(ell)["state"] == nm.PHASE_DEFAULT
    ra = a.sample(ell, M)
    pc = a.phase_config(ell)
    assert pc["state"] == nm.PHASE_TUNED and pc["variant"] in (0, 1, 2) and pc["chunk"] == 32
    assert pc["probe_ms"] > 0
    b = _model(nm, autotune=0)
    b.set_phase_config(ell, variant=pc["variant"], chunk=pc["chunk"])
    _same(ra, b.sample(ell, M))
    # small calls do not tune
    assert a.sample(7, 100)["M"] == 100 and a.phase_config(7)["state"] == nm.PHASE_DEFAULT
    # a new seed keeps the tuned choice; another configuration drops it
    a.configure(seed=11)
    assert a.phase_config(ell) == pc
    a.configure(adaptive_r=1.25)
    assert a.phase_config(ell)["state"] == nm.PHASE_DEFAULT


def test_tuning_before_graph_capture(nm):
    """nmlmc_sample_levels tunes outside the capture; the graph result equals per-level calls."""
    a, b = _model(nm, autotune=1, seed=8), _model(nm, autotune=0, seed=8)
    ells, Ms = [0, 1, 3], [1 << 19, 1 << 17, 1 << 15]
    ra = a.sample_levels(ells, Ms)
    for e in ells:
        pc = a.phase_config(e)
        b.set_phase_config(e, variant=pc["variant"], chunk=pc["chunk"])
    rb = [b.sample(e, m) for e, m in zip(ells, Ms)]
    for x, y in zip(ra, rb):
        _same(x, y)
    assert a.phase_config(0)["state"] == nm.PHASE_TUNED


def test_explicit_tuning_and_chunk_bound(nm):
    """nmlmc_autotune_level also tries half / double chunks; any chunk stays within the FP32 bound
    of the all-FP64 run on the same streams."""
    ell, M = 5, 4000
    s = _model(nm, autotune=0, N0=64)
    pc = s.autotune_level(ell, 1 << 15)
    assert pc["state"] == nm.PHASE_TUNED and pc["chunk"] in (16, 32, 64)
    o = O.Sampler(O.PREC_FP64, O.STREAMS_OUTER, 1, 64, 2, 1.5, True, False, 3)
    o.set_model(O.MODEL_SHIFT, 0.0, 1.0)
    go = o.sample(ell, M, trace=True)
    for ch in (8, 16, 32, 64):
        g = _model(nm, autotune=0, N0=64)
        g.set_phase_config(ell, variant=1, chunk=ch)
        compare_traces(g.sample(ell, M, trace=True)["trace"], go["trace"], FLIP_FP32, max_frac=0.005)


def test_invalid_and_unpinned_configurations(nm):
    s = _model(nm, autotune=0)
    with pytest.raises(nm.NmlmcError):
        s.set_phase_config(2, variant=4)
    with pytest.raises(nm.NmlmcError):
        s.set_phase_config(2, chunk=24)          # not a power of two
    with pytest.raises(nm.NmlmcError):
        s.set_phase_config(2, chunk=128)         # above the largest chunk
    with pytest.raises(nm.NmlmcError):
        s.set_autotune(3)
    s.set_phase_config(2, variant=1, chunk=16)
    assert s.phase_config(2)["state"] == nm.PHASE_PINNED
    s.set_model(nm.MODEL_SHIFT, 0.0, 1.0)        # pinned choices survive a model change
    assert s.phase_config(2)["state"] == nm.PHASE_PINNED
    s.set_phase_config(2)
    assert s.phase_config(2)["state"] == nm.PHASE_DEFAULT
    f64 = nm.Sampler(precision=nm.PREC_FP64, streams=nm.STREAMS_OUTER)
    f64.set_model(nm.MODEL_SHIFT, 0.0, 1.0)
    with pytest.raises(nm.NmlmcError):
        f64.autotune_level(2, 1 << 15)           # tuning is for the FP32 path
