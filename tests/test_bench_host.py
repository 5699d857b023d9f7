"""Host-side arithmetic behind the bench line (no device): the time-to-error comparison of the
learned configurations, the error metric, the whole-job throughput, and the clock summary that
decides whether a run saw a throttle reason."""

from __future__ import annotations

import sys
from pathlib import Path

import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
import bench  # noqa: E402


def test_max_error_skips_the_initial_value():
    assert bench._max_error([5.0, 0.1, 0.3], [0.0, 0.15, 0.2]) == pytest.approx(0.1)


def test_time_to_error_takes_the_fastest_learned_run_at_or_below_each_plain_error():
    plain = {20: {"max_error": 0.05, "wall_s": 1.0}, 24: {"max_error": 0.001, "wall_s": 3.0}}
    learned = {16: {"max_error": 0.04, "wall_s": 0.5}, 18: {"max_error": 0.02, "wall_s": 0.6},
               20: {"max_error": 0.002, "wall_s": 0.9}}
    rows = bench._time_to_error(plain, learned)
    assert [r["plain_budget_log2"] for r in rows] == [20, 24]
    assert rows[0]["learned_budget_log2"] == 16 and rows[0]["ratio"] == pytest.approx(2.0)
    # no learned run reaches 0.001: no ratio is claimed
    assert rows[1]["learned_budget_log2"] is None and rows[1]["ratio"] is None


def test_replica_throughput_is_all_terms_over_the_slowest_rank():
    value, max_ms, terms = bench.replica_throughput(2.0e9, 100.0, 1)
    assert (max_ms, terms) == (100.0, 2.0e9)
    assert value == pytest.approx(2.0e10)


def test_clock_summary_from_nvml_samples_names_the_reasons():
    c = bench.ClockSampler(0)
    c.samples = [(1965.0, 1965.0, 0), (1900.0, 1965.0, 0x4), (1965.0, 1965.0, 0x40 | 0x4)]
    s = c.summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0 and s["samples"] == 3
    assert s["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"] and s["source"] == "nvml"


def test_clock_summary_from_nvidia_smi_lines():
    c = bench.ClockSampler(0)
    c.lines = ["0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Active",
               "0, 1800, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active"]
    s = c.summary()
    assert s["samples"] == 2 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"] and s["source"] == "nvidia-smi"


def test_clock_summary_without_samples():
    s = bench.ClockSampler(0).summary()
    assert s["sm_mhz"] is None and s["samples"] == 0
