"""The allocation-free level call (nmlmc_sample_level_noalloc) against the regular entry point.

Who it is for: callers that may not allocate device memory — code running while a framework
owns the device memory pool, latency-critical code that cannot afford cudaMalloc's implicit
device-wide synchronisation, hosts that reserve all device memory up front.  It keeps its scratch
in one fixed device array, so this test calls it through the C ABI twice in a row (the second
call must not see the first call's leftovers) and compares each result with nmlmc_sample on the
same outer samples (same streams, so the sums are equal; the tolerance is exact equality, the
same rule as the other same-stream tests).  The cases cover both models, level 0 (fine only) and
an adaptive level, the non-adaptive rule, and M at the scratch limit (NMLMC_NOALLOC_MAX_OUTER,
where the carved buffers are used in full).

This file is collected last (test_zz_*), so a run that stops at the first failure has already
run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_OUTER = 65536          # NMLMC_NOALLOC_MAX_OUTER


def _device_buffer(n_doubles):
    import torch
    return torch.zeros(n_doubles, dtype=torch.float64, device="cuda:0")


@pytest.mark.parametrize("prec_name", ["fp32", "fp64"])
@pytest.mark.parametrize("kind_name", ["shift", "reference"])
@pytest.mark.parametrize("ell,r,M", [(6, 1.5, 20000), (0, 1.5, 20000), (6, 0.0, 20000), (5, 1.5, MAX_OUTER)])
def test_noalloc_matches_regular_entry_point(nm, prec_name, kind_name, ell, r, M):
    import torch
    prec = nm.PREC_FP32 if prec_name == "fp32" else nm.PREC_FP64
    kind, tau, max_loss = ((nm.MODEL_SHIFT, 0.0, 1.0) if kind_name == "shift"
                           else (nm.MODEL_REFERENCE, 0.02, 0.09))
    N0, beta, seed = 32, 2, 21
    s = nm.Sampler(0, N0=N0, beta=beta, adaptive_r=r, precision=prec, streams=nm.STREAMS_OUTER, seed=seed)
    s.set_model(kind, tau, max_loss)
    s.set_autotune(0)
    regular = [s.sample(ell, M), s.sample(ell, M)]     # outer samples [0, M) then [M, 2M)

    lib = nm.lib()
    out = _device_buffer(16)
    for call, first in enumerate((0, M)):
        rc = lib.nmlmc_sample_level_noalloc(kind, tau, max_loss, N0, beta, r, 0, prec, seed,
                                            ell, first, M, ctypes.c_void_p(out.data_ptr()), None)
        assert rc == nm.OK, nm.error_string(rc)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        ref = regular[call]
        np.testing.assert_array_equal(got[0:4], ref["fsums"])
        np.testing.assert_array_equal(got[4:8], ref["diffsums"])
        assert got[8] == ref["work"]
        assert got[9] == ref["stats"][0]
        assert got[10] == ref["stats"][2] and got[11] == ref["stats"][3]


def test_noalloc_rejects_sizes_beyond_its_scratch(nm):
    out = _device_buffer(16)
    lib = nm.lib()
    rc = lib.nmlmc_sample_level_noalloc(nm.MODEL_SHIFT, 0.0, 1.0, 32, 2, 1.5, 0, nm.PREC_FP32, 1,
                                        3, 0, MAX_OUTER + 1, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == nm.ERR_ARG
    assert lib.nmlmc_last_error() == nm.ERR_ARG
