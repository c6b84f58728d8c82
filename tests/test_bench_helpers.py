"""Host logic of bench.py, without a GPU: the clock / throttle-reason parsing that decides whether
a run's clocks are valid, the per-level extrapolation of the FP64 drop-in's time, the report of the
autotuner's per-level choices, the reference arm's lines (model problem and large portfolio) and
the assembly of both workloads' lines from fake samplers."""
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
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--case", "c1",
           "--steps", "1", "--warmup", "3", "--ref-budget", "1"]
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


class _FakeSampler:
    """Stands in for nmlmc.Sampler in the bench's default path: fixed level results, so the
    JSON line's assembly runs without a GPU."""

    def __init__(self, device=0, **kw):
        self.kw = kw

    def set_model(self, *a):
        pass

    def set_autotune(self, mode):
        pass

    def configure(self, **kw):
        pass

    def set_profiling(self, on):
        pass

    def phase_kernel_time(self):
        return 40, 0.1

    def phase_config(self, ell):
        return dict(variant=1, chunk=32, state=1, probe_ms=20.0)

    def mlmc_run(self, targetTOL, M0, batched=False):
        import numpy as np
        n = 4
        return dict(level_time=np.full(n, 0.03), total_work=2.0e9, calls=12, nlevels=n,
                    level_M=np.array([1000, 500, 200, 100], np.uint64), Eg=0.1587)


def test_default_line_with_a_fake_sampler(monkeypatch, capsys):
    """bench.py's default run assembles a line with every key of the contract (value, e2e with
    its byte counts, roofline, clocks, gpu_launches, config) from the sampler's results."""
    import json
    import sys
    import types
    fake = types.ModuleType("nmlmc")
    fake.Sampler = _FakeSampler
    fake.PREC_FP32, fake.PREC_FP64, fake.PREC_REF32 = 2, 1, 0
    fake.STREAMS_OUTER, fake.STREAMS_CORE, fake.MODEL_SHIFT = 1, 0, 1
    fake.kernel_launches = lambda: 0
    monkeypatch.setitem(sys.modules, "nmlmc", fake)
    monkeypatch.setattr(sys, "argv", ["bench.py", "--case", "c1", "--steps", "2", "--warmup", "3", "--no-compare",
                                      "--no-cpu"])
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    bench.main()
    line = json.loads([l for l in capsys.readouterr().out.splitlines() if l.startswith("{")][-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "e2e", "roofline", "clocks",
                "gpu_launches"):
        assert key in line, key
    assert line["value"] == 0.12 and line["steps"] == 2 and line["warmup"] == 3
    assert line["e2e"]["d2h_bytes_per_step"] == 12 * 144 and line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["config"]["workload"] and line["phase_config"]["0"] == [1, 32, True]
    assert 0 < line["roofline"]["frac"] and line["roofline"]["unit"] == "Gop/s"


def test_cpu_baseline_falls_back_to_the_port(monkeypatch):
    """Without oracle/_ref the CPU baseline times the C restatement (kind "port", one thread) on
    the same bounded per-level samples."""
    import oracle as O
    monkeypatch.setattr(O, "ref_available", lambda variant="f32": False)
    schedule = dict(levels=[0, 1], M=[4000, 1000])
    v, kind, cores, desc = bench.cpu_reference_time(schedule, budget_s=0.2)
    assert kind == "port" and cores == 1 and v > 0 and "C port" in desc


class _FakePortfolioSampler(_FakeSampler):
    """Stands in for nmlmc.Sampler on the large-portfolio line: a table set-up, a loss sweep and
    fixed MLMC results (levels 0-3, starting level 2)."""

    def set_portfolio(self, *a, **kw):
        pass

    def full_loss(self, ell, first, n):
        import numpy as np
        return np.linspace(0.0, 1.0, n)

    def set_phase_config(self, ell, variant=None, chunk=None):
        pass

    def sample(self, ell, M, trace=False):
        import numpy as np
        return dict(stats=np.array([64.0 * M, 0, 0, 0]), seconds=1e-3, fsums=np.zeros(4), diffsums=np.zeros(4))

    def close(self):
        pass

    def mlmc_run(self, targetTOL, M0, batched=False):
        d = super().mlmc_run(targetTOL, M0, batched)
        return dict(d, starting_level=2)


def test_large_portfolio_line_with_a_fake_sampler(monkeypatch, capsys):
    """The default line (large portfolio): the contract's keys, the table upload counted as host->
    device bytes of every step, the configuration dict shared with the reference arm."""
    import json
    import sys
    import types
    import numpy as np
    fake = types.ModuleType("nmlmc")
    fake.Sampler = _FakePortfolioSampler
    fake.PREC_FP32, fake.PREC_FP64, fake.PREC_REF32 = 2, 1, 0
    fake.STREAMS_OUTER, fake.STREAMS_CORE, fake.SUB_RANDOM, fake.TAU_WEEK = 1, 0, 1, 1 / 52
    fake.PORTFOLIO_C3 = dict(Q=3, P=10)
    fake.kernel_launches = lambda: 0
    fake.generate_portfolio = lambda spec, seed: dict(S0=np.full(3, 100.0), mu=np.full(3, 0.05),
                                                      sigma=np.full(3, 0.2), strike=np.full(10, 100.0),
                                                      maturity=np.ones(10), w=np.arange(10.0) - 4.5,
                                                      stock_ind=np.zeros(10, np.uint32),
                                                      type=np.ones(10, np.int32), prob=np.ones(10))
    fake.loss_quantile = lambda s, q, n: 0.99
    monkeypatch.setitem(sys.modules, "nmlmc", fake)
    monkeypatch.setattr(sys, "argv", ["bench.py", "--steps", "2", "--warmup", "3", "--no-compare", "--no-cpu"])
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    bench.main()
    line = json.loads([l for l in capsys.readouterr().out.splitlines() if l.startswith("{")][-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "e2e", "roofline", "clocks",
                "gpu_launches"):
        assert key in line, key
    assert line["metric"] == bench.METRIC and line["value"] == 0.12 and line["steps"] == 2
    assert line["config"] == bench.C3_CONFIG
    assert line["e2e"]["h2d_bytes_per_step"] == bench.c3_upload_bytes(10, 3)
    assert line["e2e"]["d2h_bytes_per_step"] == 12 * 144
    assert line["starting_level"] == 2 and line["roofline"]["frac"] > 0


def test_large_portfolio_reference_arm_line():
    """`bench.py --impl reference` (default: the large portfolio) times the reference's CPU
    sampler on the schedule recorded from the GPU run (with its K) and calibrates the
    extrapolation with one complete CPU run; its config is the GPU line's."""
    import json
    import subprocess
    import sys
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
           "--warmup", "3", "--ref-budget", "2"]
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=900, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    d = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])
    assert d["impl"] == "reference" and d["config"] == bench.C3_CONFIG and d["value"] > 0
    c = d["cpu_baseline"]
    assert c["kind"] in ("reference", "port") and c["value"] == d["value"]
    cal = c["calibration"]
    assert cal["measured_s"] > 0 and cal["extrapolated_s"] > 0 and cal["eps"] <= 1e-2
