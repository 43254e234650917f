"""Host-side pieces of bench.py (CPU): the clock summary the rejection rules
read (median SM clock under load, max clock, active throttle reasons) and
the HBM peak lookup with its fallback."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_clock_summary():
    c = bench.ClockSampler(0)
    c.rows = [["0", "1965", "1965", "700", "Not Active", "Not Active", "Not Active", "Active"],
              ["0", "1900", "1965", "710", "Not Active", "Not Active", "Not Active", "Not Active"],
              ["0", "1965", "1965", "690", "Not Active", "Active", "Not Active", "Not Active"],
              ["0", "[N/A]", "1965", "690", "x", "x", "x", "x"]]
    s = c.summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0 and s["samples"] == 4
    assert s["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]
    assert bench.ClockSampler(0).summary()["sm_mhz"] is None


def test_peak_lookup(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "HERE", str(tmp_path))
    assert bench.measured_peak_hbm() == (6650.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6438.5}))
    assert bench.measured_peak_hbm() == (6438.5, "measured")
