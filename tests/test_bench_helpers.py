"""Host logic of bench.py, without a GPU: the clock / throttle-reason parsing that decides whether
a run's clocks are valid, the per-level extrapolation of the FP64 drop-in's time, and the report
of the autotuner's per-level choices, and the reference arm's line."""
import os

import bench
from conftest import ROOT


def test_clock_samples_median_and_reasons():
    rows = "\n".join([
        "0, 1965, 1965, 820.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 990.7, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1965, 1965, 1001.2, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "garbage line",
    ])
    c = bench.parse_clock_samples(rows)
    assert c["sm_mhz"] == 1965.0 and c["sm_max_mhz"] == 1965.0 and c["samples"] == 3
    assert c["reasons"] == ["sw_power_cap"]
    hot = bench.parse_clock_samples("0, 1200, 1965, 700, 0x40, Not Active, Active, Not Active, Not Active")
    assert hot["reasons"] == ["hw_thermal_slowdown"] and hot["sm_mhz"] == 1200.0
    assert bench.parse_clock_samples("")["sm_mhz"] is None


class FakeSampler:
    """Device time linear in the outer samples of a call: cost[ell] seconds per outer sample."""

    def __init__(self, cost):
        self.cost = cost
        self.calls = []

    def sample(self, ell, M):
        self.calls.append((ell, M))
        return {"seconds": self.cost[ell] * M}


def test_dropin_extrapolation_is_cost_per_outer_sample_times_counts():
    cost = [1e-7, 3e-6, 1e-4]
    level_M = [10_000_000, 500_000, 40_000]
    s = FakeSampler(cost)
    out = bench.dropin_extrapolated(s, level_M, budget_s=3.0)
    expect = sum(c * m for c, m in zip(cost, level_M))
    assert abs(out["value"] - expect) <= 1e-9 * expect
    assert out["extrapolated"] and out["e2e"] is None
    # every level is sampled on at least one call per virtual core and never beyond its count
    for ell, m in s.calls:
        assert 2048 <= m <= max(level_M[ell], 2048)


def test_phase_choices_report():
    class S:
        def phase_config(self, ell):
            return dict(variant=ell % 3, chunk=32, state=1 if ell < 2 else 0, probe_ms=1.0)
    assert bench.phase_choices(S(), 3) == {"0": [0, 32, True], "1": [1, 32, True], "2": [2, 32, False]}


def test_reference_arm_line(tmp_path):
    """`bench.py --impl reference` runs the reference's CPU level sampler (no GPU) and prints one
    JSON line with the contract's keys; under torchrun only rank 0 prints."""
    import json
    import subprocess
    import sys
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
           "--warmup", "3", "--ref-budget", "1"]
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is False
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    env1 = dict(env, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    out1 = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env1)
    assert out1.returncode == 0 and not out1.stdout.strip()


def test_reference_model_main_on_the_cpu(golden):
    """The CPU leg of `--case ref-model`: the reference's sampler of its model main under the host
    driver (a loose tolerance here); the model's exact answer is eta = 0.025, and the library's
    max_loss of the main equals the compiled reference's."""
    import nmlmc as nm
    meta, _ = golden
    assert bench.ref_main_max_loss(nm.norm_cdf_inv) == meta["model_max_loss_f32"]
    r = bench.ref_main_cpu(threads=2, tol=1e-2)
    if "unavailable" in r:
        import pytest
        pytest.skip(r["unavailable"])
    assert r["threads"] == 2 and r["levels"] >= 2 and r["total_work"] > 0
    assert abs(r["Eg"] - bench.REF_MAIN["eta"]) < 3e-2
