"""Host logic of bench.py, without a GPU: the clock / throttle-reason parsing that decides whether
a run's clocks are valid, the per-level extrapolation of the FP64 drop-in's time, and the report
of the autotuner's per-level choices."""
import bench


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
