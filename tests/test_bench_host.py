"""CPU tests of bench.py's host-side pieces: the clock record taken during the timed region and
the roofline denominator."""
from __future__ import annotations

import json

import bench


def _sampler(lines):
    s = bench.ClockSampler(0)
    s.lines = list(lines)
    return s


def test_clock_summary_takes_the_median_and_the_active_reasons():
    lines = [
        "0, 1965, 1965, 700.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1800, 1965, 990.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1950, 1965, 820.5, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "garbage line",
        "0, [N/A], 1965, 0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ]
    d = _sampler(lines).summary()
    assert d == {"sm_mhz": 1950.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}


def test_clock_summary_flags_thermal_and_hardware_slowdowns():
    lines = ["0, 1400, 1965, 1000, 0x68, Active, Active, Active, Not Active"] * 4
    d = _sampler(lines).summary()
    assert d["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]
    assert d["sm_mhz"] == 1400.0


def test_clock_summary_without_samples():
    d = _sampler([]).summary()
    assert d == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}


def test_roofline_peak_comes_from_the_measured_file(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench._peaks() == (6650.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 7012.5}))
    assert bench._peaks() == (7012.5, "measured")
