"""Failure handling of the library, made on the host (no GPU fault is provoked):

* a device allocation that fails (nmlmc_inject_alloc_failure) is reported as NMLMC_ERR_NOMEM
  by the call that needed it, and the same context works afterwards with identical results;
* non-finite or non-positive model and portfolio inputs are rejected with NMLMC_ERR_ARG instead
  of turning into phi = 0 inside the kernels.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _model(nm, **kw):
    s = nm.Sampler(N0=32, beta=2, adaptive_r=1.5, precision=nm.PREC_FP32, streams=nm.STREAMS_OUTER, seed=2, **kw)
    s.set_model(nm.MODEL_SHIFT, 0.0, 1.0)
    return s


@pytest.mark.parametrize("after", [0, 3, 8])
def test_allocation_failure_is_reported_and_recoverable(nm, after):
    ref = _model(nm).sample(4, 5000)
    s = _model(nm)
    lib = nm.lib()
    assert lib.nmlmc_inject_alloc_failure(after) == nm.OK
    try:
        with pytest.raises(nm.NmlmcError) as e:
            s.sample(4, 5000)
        assert e.value.status == nm.ERR_NOMEM
    finally:
        lib.nmlmc_inject_alloc_failure(-1)
    s.reset_streams()
    got = s.sample(4, 5000)                 # the context recovers: same streams, same sums
    np.testing.assert_array_equal(got["fsums"], ref["fsums"])
    np.testing.assert_array_equal(got["diffsums"], ref["diffsums"])


def test_allocation_failure_in_a_graph_round(nm):
    s = _model(nm)
    lib = nm.lib()
    lib.nmlmc_inject_alloc_failure(0)
    try:
        with pytest.raises(nm.NmlmcError):
            s.sample_levels([0, 2], [4000, 1000])
    finally:
        lib.nmlmc_inject_alloc_failure(-1)
    s.reset_streams()
    a = s.sample_levels([0, 2], [4000, 1000])
    b = _model(nm).sample_levels([0, 2], [4000, 1000])
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x["fsums"], y["fsums"])


def test_non_finite_inputs_are_rejected(nm):
    s = nm.Sampler(N0=32, beta=2, precision=nm.PREC_FP32, streams=nm.STREAMS_OUTER)
    for tau, K in ((0.0, float("nan")), (float("inf"), 1.0)):
        with pytest.raises(nm.NmlmcError):
            s.set_model(nm.MODEL_SHIFT, tau, K)
    with pytest.raises(nm.NmlmcError):
        s.set_model(nm.MODEL_REFERENCE, 1.5, 0.1)      # sqrt(1 - tau) undefined
    pf = O.synthetic_portfolio(4, 100, 3)
    for key, bad in (("strike", np.nan), ("w", np.inf), ("sigma", 0.0), ("S0", -1.0), ("maturity", np.nan)):
        p = {k: np.array(v, copy=True) for k, v in pf.items()}
        p[key][0] = bad
        with pytest.raises(nm.NmlmcError):
            s.set_portfolio(p, max_loss=1.0)
    with pytest.raises(nm.NmlmcError):
        s.set_portfolio(pf, max_loss=float("nan"))
    s.set_portfolio(pf, max_loss=1.0)                    # the valid portfolio is accepted
    assert s.sample(1, 100)["M"] == 100
