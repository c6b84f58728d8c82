"""Checkpoint / resume of the host MLMC driver (nmlmc_mlmc_run_cb_ckpt) and the readers of its
checkpoint file and printed reports.

The synthetic level sampler of the driver tests is deterministic and stateful (a counter-based
generator), so a run interrupted by a failing sampler and resumed from its last checkpoint, with
the sampler's state restored from the same file, must reproduce the uninterrupted run exactly:
the same sample_level calls, FP64 level sums, error split and report text.
"""
import json
import os

import numpy as np
import pytest

from test_mlmc_driver import Synthetic


def _args(golden, idx=1):
    meta, _ = golden
    tol, M0, a, alpha, v, beta, w, gamma, seed = meta["mlmc"][idx]["args"]
    return dict(tol=tol, M0=int(M0)), (a, alpha, v, beta, w, gamma, int(seed))


class Failing(Synthetic):
    """The synthetic sampler that raises on its `fail_at`-th call (a crashed job)."""

    def __init__(self, *a, fail_at=None):
        super().__init__(*a)
        self.fail_at = fail_at

    def __call__(self, ell, M):
        if self.fail_at is not None and len(self.calls) == self.fail_at:
            raise RuntimeError("sampler lost")
        return super().__call__(ell, M)


def _state(s):
    """(save, load) of a synthetic sampler: its generator state and call count."""
    def save():
        return json.dumps([s.state, len(s.calls)]).encode()

    def load(b):
        st, n = json.loads(b.decode())
        s.state = st
        s.restored_calls = n
    return save, load


def _same_run(a, b):
    for k in ("nlevels", "starting_level", "bias_est", "stat_error", "TOL", "Eg", "calls", "table"):
        assert a[k] == b[k], k
    for k in ("level_M", "level_fsums", "level_diffsums", "level_work"):
        np.testing.assert_array_equal(a[k], b[k])


def test_resume_after_a_crash_equals_the_uninterrupted_run(nm, golden, tmp_path):
    kw, sa = _args(golden)
    full_s = Synthetic(*sa)
    full = nm.mlmc_run_cb(full_s, targetTOL=kw["tol"], M0=kw["M0"], verbose=False)
    assert full["complete"] and full["iterations_done"] > 4
    path = str(tmp_path / "run.ckpt")
    fail_at = len(full_s.calls) * 2 // 3
    s1 = Failing(*sa, fail_at=fail_at)
    with pytest.raises(nm.NmlmcError, match="sampler lost") as e:
        nm.mlmc_run_cb(s1, targetTOL=kw["tol"], M0=kw["M0"], checkpoint=path, state=_state(s1))
    assert isinstance(e.value.__cause__, RuntimeError)      # the sampler's own exception
    ck = nm.checkpoint.read_checkpoint(path)
    assert 0 < ck["itr_next"] < ck["total_itrs"] + 1 and ck["calls"] <= fail_at
    s2 = Synthetic(*sa)
    res = nm.mlmc_run_cb(s2, targetTOL=kw["tol"], M0=kw["M0"], checkpoint=path, resume=True,
                         state=_state(s2))
    _same_run(res, full)
    assert res["complete"] and res["iterations_done"] == full["iterations_done"]
    # the resumed sampler made exactly the calls the uninterrupted one made after the checkpoint
    assert s2.calls == full_s.calls[s2.restored_calls:]
    # the final checkpoint holds the run's FP64 level sums
    ck = nm.checkpoint.read_checkpoint(path)
    np.testing.assert_array_equal(ck["level_fsums"], res["level_fsums"])
    np.testing.assert_array_equal(ck["level_diffsums"], res["level_diffsums"])
    np.testing.assert_array_equal(ck["level_M"], res["level_M"])
    assert ck["itr_next"] == ck["total_itrs"] + 1 and ck["TOL"] == res["TOL"]


@pytest.mark.parametrize("batched", [False, True])
def test_max_iterations_then_resume(nm, golden, tmp_path, batched):
    kw, sa = _args(golden, 2)
    full = nm.mlmc_run_cb(Synthetic(*sa), targetTOL=kw["tol"], M0=kw["M0"], batched=batched)
    path = str(tmp_path / "slices.ckpt")
    s = Synthetic(*sa)
    done = 0
    for k in range(100):                       # time slices of 3 iterations each
        res = nm.mlmc_run_cb(s, targetTOL=kw["tol"], M0=kw["M0"], batched=batched, checkpoint=path,
                             resume=k > 0, state=_state(s), max_iterations=3)
        assert res["iterations_done"] == min(done + 3, full["iterations_done"])
        done = res["iterations_done"]
        if res["complete"]:
            break
        assert nm.checkpoint.read_checkpoint(path)["itr_next"] == done
    _same_run(res, full)


def test_warm_start_from_another_tolerance(nm, golden, tmp_path):
    """Other input parameters: the saved level sums seed a fresh schedule (no sample is lost)."""
    kw, sa = _args(golden)
    path = str(tmp_path / "warm.ckpt")
    s = Synthetic(*sa)
    first = nm.mlmc_run_cb(s, targetTOL=4 * kw["tol"], M0=kw["M0"], checkpoint=path, state=_state(s))
    n_first = len(s.calls)
    tight = nm.mlmc_run_cb(s, targetTOL=kw["tol"], M0=kw["M0"], checkpoint=path, resume=True, state=_state(s))
    assert tight["complete"] and tight["TOL"] < first["TOL"]
    M_first = first["level_M"]
    assert np.all(tight["level_M"][:len(M_first)] >= M_first)
    assert len(s.calls) > n_first
    ck = nm.checkpoint.read_checkpoint(path)
    assert ck["targetTOL"] == kw["tol"]


def test_resume_without_a_file_starts_fresh_and_bad_files_are_errors(nm, golden, tmp_path):
    kw, sa = _args(golden)
    path = str(tmp_path / "none.ckpt")
    a = nm.mlmc_run_cb(Synthetic(*sa), targetTOL=kw["tol"], M0=kw["M0"], checkpoint=path, resume=True)
    b = nm.mlmc_run_cb(Synthetic(*sa), targetTOL=kw["tol"], M0=kw["M0"])
    _same_run(a, b)
    bad = str(tmp_path / "bad.ckpt")
    with open(bad, "wb") as f:
        f.write(b"NMLMCCK1" + b"\0" * 20)
    with pytest.raises(nm.NmlmcError):
        nm.mlmc_run_cb(Synthetic(*sa), targetTOL=kw["tol"], M0=kw["M0"], checkpoint=bad, resume=True)
    with pytest.raises(ValueError):
        nm.checkpoint.read_checkpoint(bad)
    assert not os.path.exists(path + ".tmp")


def test_failing_state_hook_stops_the_run(nm, golden, tmp_path):
    """A sampler whose state cannot be saved must not leave a checkpoint without it."""
    kw, sa = _args(golden)

    def bad_save():
        raise RuntimeError("state unavailable")

    with pytest.raises(nm.NmlmcError, match="state unavailable") as e:
        nm.mlmc_run_cb(Synthetic(*sa), targetTOL=kw["tol"], M0=kw["M0"], checkpoint=str(tmp_path / "x.ckpt"),
                       state=(bad_save, lambda b: None))
    assert e.value.status == nm.ERR_STATE and isinstance(e.value.__cause__, RuntimeError)
    assert not os.path.exists(str(tmp_path / "x.ckpt"))


def test_report_reader(nm, golden):
    """The reports' text (identical to the reference's to_string) read back: the final report
    of each golden run against the driver's numbers."""
    meta, _ = golden
    for g in meta["mlmc"]:
        tol, M0, *sa = g["args"]
        out = nm.mlmc_run_cb(Synthetic(*sa[:6], int(sa[6])), targetTOL=tol, M0=int(M0))
        reps = nm.tables.parse_reports(g["table"])
        assert len(reps) == 1
        r = reps[0]
        assert r["starting_level"] == out["starting_level"]
        np.testing.assert_array_equal(nm.tables.column(r, "M"), out["level_M"].astype(float))
        np.testing.assert_allclose(r["Eg"], out["Eg"], rtol=1e-5)
        np.testing.assert_allclose(r["TOL"], out["TOL"], rtol=1e-5)
        np.testing.assert_allclose(nm.tables.column(r, "Wl"), out["level_work"] / out["level_M"], rtol=1e-4)


def test_report_reader_on_the_driver_stdout(nm, golden, capfd):
    """The driver's verbose stdout (the reference's "# Sampling" lines and one report per TOL
    iteration) read back: one report per completed iteration, TOL shrinking by sqrt(2), the last
    report equal to the returned table."""
    kw, sa = _args(golden)
    out = nm.mlmc_run_cb(Synthetic(*sa), targetTOL=kw["tol"], M0=kw["M0"], verbose=True)
    text = capfd.readouterr().out
    assert "# Sampling" in text
    reps = nm.tables.parse_reports(text)
    assert len(reps) == out["iterations_done"]
    tols = [r["TOL"] for r in reps]
    np.testing.assert_allclose(np.array(tols[1:]) / np.array(tols[:-1]), 2 ** -0.5, rtol=1e-4)
    last = nm.tables.parse_reports(out["table"])[0]
    np.testing.assert_array_equal(last["data"], reps[-1]["data"])
    assert last["starting_level"] == reps[-1]["starting_level"] == out["starting_level"]


def test_report_reader_starred_levels(nm):
    text = """TOL: 0.001
RMS: 0.0009 (0.0004, 0.0008)
Eg: 0.25 --- [0.249,0.251]
Discarded Work: 10
Discarded Time: 0
Total Work: 100
Total Time: 0
| ell |    dEl     |    fEl     |   M   |
+-----+------------+------------+-------+
|  *0 | 0.0000e+00 | 5.0000e-01 |   100 |
|  *1 | 1.0000e-01 | 4.0000e-01 |    50 |
|   2 | 2.0000e-02 | 3.0000e-01 |    25 |
+-----+------------+------------+-------+
"""
    r = nm.tables.parse_reports(text)[0]
    assert r["starting_level"] == 2 and r["Discarded Work"] == 10
    np.testing.assert_array_equal(nm.tables.column(r, "M"), [100, 50, 25])


class Bounded(Synthetic):
    """The synthetic sampler, refusing absurd sample counts (a damaged file must not turn into a
    run that never ends)."""

    def __call__(self, ell, M):
        if M > 10**6:
            raise RuntimeError("sample count out of range")
        return super().__call__(ell, M)


def test_damaged_checkpoints_are_errors_not_crashes(nm, golden, tmp_path):
    """Every truncation of a checkpoint is rejected; a flipped bit gives an error or a normal
    (bounded) run, never a crash, a hang or a NaN-sized request."""
    import collections
    kw, sa = _args(golden, 2)
    path = str(tmp_path / "good.ckpt")
    s = Synthetic(*sa)
    nm.mlmc_run_cb(s, targetTOL=kw["tol"], M0=kw["M0"], checkpoint=path, state=_state(s), max_iterations=3)
    good = open(path, "rb").read()
    bad = str(tmp_path / "bad.ckpt")

    def attempt(blob):
        with open(bad, "wb") as f:
            f.write(blob)
        s2 = Bounded(*sa)
        try:
            nm.mlmc_run_cb(s2, targetTOL=kw["tol"], M0=kw["M0"], checkpoint=bad, resume=True,
                           state=_state(s2), max_iterations=2)
            return "ran"
        except nm.NmlmcError:
            return "error"

    for n in range(0, len(good), max(1, len(good) // 97)):
        assert attempt(good[:n]) == "error", n
        with pytest.raises(ValueError):           # the Python reader agrees
            nm.checkpoint.read_checkpoint(bad)
    assert attempt(good) == "ran"
    rng = np.random.default_rng(5)
    seen = collections.Counter()
    for _ in range(300):
        b = bytearray(good)
        b[int(rng.integers(len(b)))] ^= 1 << int(rng.integers(8))
        seen[attempt(bytes(b))] += 1
    assert seen["error"] > 0 and seen["ran"] > 0, seen
    # a level sum made non-finite (level 0's first fine sum: after the 120-byte header and the
    # level's M) is rejected by the reader
    import struct
    b = bytearray(good)
    b[128:136] = struct.pack("<d", float("nan"))
    assert attempt(bytes(b)) == "error"
    b[128:136] = struct.pack("<d", float("inf"))
    assert attempt(bytes(b)) == "error"


def test_unwritable_checkpoint_stops_the_run(nm, golden, tmp_path):
    """A checkpoint that cannot be written (its directory is missing) stops the run with
    NMLMC_ERR_STATE at the first save instead of running on unprotected."""
    kw, sa = _args(golden)
    s = Synthetic(*sa)
    with pytest.raises(nm.NmlmcError) as e:
        nm.mlmc_run_cb(s, targetTOL=kw["tol"], M0=kw["M0"], checkpoint=str(tmp_path / "missing" / "x.ckpt"))
    assert e.value.status == nm.ERR_STATE and len(s.calls) > 0
