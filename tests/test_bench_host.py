"""Host logic of bench.py: the clock-sample window and the traffic figure."""

from __future__ import annotations

import datetime
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def _line(ts, sm, reasons=("Not Active",) * 4):
    # timestamp, index, clocks.sm, clocks.max.sm, power.draw, active mask, then the four reasons
    return f"{ts:%Y/%m/%d %H:%M:%S.%f}, 0, {sm}, 1965, 700.0, 0x0, " + ", ".join(reasons)


def test_clock_samples_are_kept_inside_the_timed_window():
    t = datetime.datetime(2026, 1, 1, 12, 0, 0)
    ms = datetime.timedelta(milliseconds=1)
    lines = [_line(t, 1200), _line(t + 100 * ms, 1965), _line(t + 150 * ms, 1955),
             _line(t + 300 * ms, 1100, ("Not Active", "Not Active", "Not Active", "Active"))]
    got = bench.ClockSampler.summarise(lines, t + 90 * ms, t + 200 * ms)
    assert got["samples"] == 2 and got["sm_mhz"] == 1960 and got["sm_max_mhz"] == 1965
    assert got["reasons"] == [] and got["sampled"] == "timed region"
    # the power-capped idle sample after the window does not count; inside, it does
    got = bench.ClockSampler.summarise(lines, t + 250 * ms, t + 350 * ms)
    assert got["reasons"] == ["sw_power_cap"] and got["samples"] == 1


def test_a_window_shorter_than_the_interval_keeps_the_nearest_sample():
    t = datetime.datetime(2026, 1, 1, 12, 0, 0)
    ms = datetime.timedelta(milliseconds=1)
    lines = [_line(t, 1500), _line(t + 50 * ms, 1965), _line(t + 100 * ms, 1700), "garbage line"]
    got = bench.ClockSampler.summarise(lines, t + 56 * ms, t + 60 * ms)
    assert got["samples"] == 1 and got["sm_mhz"] == 1965
    assert got["sampled"].startswith("nearest")


def test_tile_traffic_adds_the_cpml_passes():
    n, cpml = 256, 3932160
    d = bench._traffic("tile_step", n, cpml)
    assert d is not None and abs(d / n**3 - (99.97 + 203.7 * cpml / n**3)) < 1e-6
    assert abs(bench._traffic("update_E+update_H", n) / n**3 - 129.02) < 1e-9
