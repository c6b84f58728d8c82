"""Checkpoint / resume of the GPU MLMC driver (nmlmc_mlmc_run_ckpt) and the context's sampler
state (nmlmc_get_sampler_state / nmlmc_set_sampler_state).

A run stopped after a few TOL iterations and resumed in a fresh context from its checkpoint
continues the same streams (OUTER: the next outer index per level; CORE: every virtual core's
stream state) and ends with the level sums, estimate and decisions of the uninterrupted run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sampler(nm, layout):
    if layout == "outer_fp32":
        s = nm.Sampler(N0=32, beta=2, adaptive_r=1.5, precision=nm.PREC_FP32, streams=nm.STREAMS_OUTER, seed=7)
    else:
        s = nm.Sampler(cores=64, N0=32, beta=2, adaptive_r=1.5, precision=nm.PREC_REF32,
                       streams=nm.STREAMS_CORE, seed=7)
    s.set_model(nm.MODEL_SHIFT, 0.0, 1.0)
    return s


def _same(a, b):
    for k in ("nlevels", "starting_level", "bias_est", "stat_error", "TOL", "Eg", "calls", "iterations_done"):
        assert a[k] == b[k], k
    for k in ("level_M", "level_fsums", "level_diffsums", "level_work"):
        np.testing.assert_array_equal(a[k], b[k])


@pytest.mark.parametrize("layout", ["outer_fp32", "core_ref32"])
def test_resume_in_a_fresh_context(nm, tmp_path, layout):
    tol = 2e-3 if layout == "outer_fp32" else 1e-2
    batched = layout == "outer_fp32"
    full = _sampler(nm, layout).mlmc_run(targetTOL=tol, M0=1024, batched=batched)
    path = str(tmp_path / f"{layout}.ckpt")
    part = _sampler(nm, layout).mlmc_run(targetTOL=tol, M0=1024, batched=batched, checkpoint=path,
                                         max_iterations=3)
    assert not part["complete"] and part["iterations_done"] == 3
    ck = nm.checkpoint.read_checkpoint(path)
    assert ck["itr_next"] == 3 and len(ck["sampler_state"]) > 0
    res = _sampler(nm, layout).mlmc_run(targetTOL=tol, M0=1024, batched=batched, checkpoint=path, resume=True)
    assert res["complete"]
    _same(res, full)
    np.testing.assert_array_equal(nm.checkpoint.read_checkpoint(path)["level_fsums"], full["level_fsums"])


@pytest.mark.parametrize("layout", ["outer_fp32", "core_ref32"])
def test_sampler_state_round_trip(nm, layout):
    s = _sampler(nm, layout)
    s.sample(2, 3000)
    st = s.sampler_state()
    a = s.sample(2, 3000)
    s.set_sampler_state(st)                 # rewind the streams
    b = s.sample(2, 3000)
    np.testing.assert_array_equal(a["fsums"], b["fsums"])
    np.testing.assert_array_equal(a["diffsums"], b["diffsums"])
    other = nm.Sampler(N0=32, beta=2, adaptive_r=1.5, precision=nm.PREC_FP32, streams=nm.STREAMS_OUTER, seed=8)
    other.set_model(nm.MODEL_SHIFT, 0.0, 1.0)
    with pytest.raises(nm.NmlmcError):      # another seed's streams
        other.set_sampler_state(_sampler(nm, "outer_fp32").sampler_state())
