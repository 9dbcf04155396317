"""bench.py's host logic, without a GPU: the clock summary of nvidia-smi samples (the median SM
clock over the samples under load, every throttle reason seen) and the CPU baseline's estimator
(the median of the differenced samples, as the reference arm takes it)."""

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def _sample(mhz: str, watts: str, power_cap: bool = False, thermal: bool = False) -> list[str]:
    active = "Active"
    idle = "Not Active"
    return ["0", mhz, "1965", watts, "0x0", idle, idle, active if thermal else idle, active if power_cap else idle]


def test_clock_summary_counts_the_samples_under_load():
    clocks = bench.Clocks(0)
    clocks.samples = [_sample("705", "85.2"), _sample("1605", "1001.4", power_cap=True),
                      _sample("1620", "998.0", power_cap=True), _sample("1650", "640.0"),
                      _sample("[N/A]", "[N/A]"), ["0", "1965"]]
    summary = clocks.summary()
    assert summary["sm_mhz"] == 1620.0  # 1605, 1620, 1650: at least half of 1001.4 W
    assert summary["samples_under_load"] == 3 and summary["samples"] == 6
    assert summary["sm_max_mhz"] == 1965.0 and summary["power_w_max"] == pytest.approx(1001.4)
    assert summary["reasons"] == ["sw_power_cap"]


def test_clock_summary_reports_every_reason_and_no_samples():
    clocks = bench.Clocks(0)
    clocks.samples = [_sample("1500", "900", thermal=True), _sample("1500", "900", power_cap=True)]
    assert clocks.summary()["reasons"] == ["sw_power_cap", "sw_thermal_slowdown"]
    empty = bench.Clocks(0).summary()
    assert empty["sm_mhz"] is None and empty["samples"] == 0 and empty["reasons"] == []


def test_cpu_baseline_takes_the_median_of_its_samples(monkeypatch):
    # Five differenced samples with every thread, three with one: the median of each, the best
    # beside; the whole solve timed once (stood in for here).
    calls = []

    def seconds(image, threads, sample, repeats):
        calls.append((threads, sample, repeats))
        if repeats == 1:
            return [1.0]
        return [0.2, 0.1, 0.4, 0.3, 0.25][:repeats] if threads > 1 else [2.0, 1.5, 3.0][:repeats]

    class Reference:
        @staticmethod
        def available():
            return True

        @staticmethod
        def solve(*args):
            return "whole"

    monkeypatch.setattr(bench, "_reference_seconds", seconds)
    monkeypatch.setitem(sys.modules, "oracle.reference", Reference)
    monkeypatch.setattr(bench, "_components", lambda image: [])
    import oracle

    monkeypatch.setattr(oracle, "reference", Reference, raising=False)

    class Image:
        height, width, color_space = 4, 4, 1

    baseline, whole = bench._cpu_baseline(Image())
    pixels = bench.HEIGHT * bench.WIDTH
    assert whole == "whole"
    assert baseline["value"] == pytest.approx(pixels * 2 / 0.25 / 1e6)
    assert baseline["best_of_samples"] == pytest.approx(pixels * 2 / 0.1 / 1e6)
    assert baseline["one_thread"]["value"] == pytest.approx(pixels * 2 / 2.0 / 1e6)
    assert [c[2] for c in calls] == [1, 5, 3]
