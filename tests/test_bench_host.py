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


def test_source_sets_and_error_check():
    import numpy as np
    from fmt2d_b200 import synth
    m = synth.config(1)
    one = bench.source_set(m, 0, 1)
    assert np.array_equal(one, m.obs_x)
    shards = [bench.source_set(m, r, 4) for r in range(4)]
    allx = np.concatenate(shards)
    assert allx.size == 120 and np.unique(np.round(allx, 6)).size == 120
    assert all(s.min() >= m.xpos[1] and s.max() <= m.xpos[-2] for s in shards)

    class FakeCtx:                      # device fields = checker + 0.2 ms, one node unreached
        def field(self, s, tf):
            T = checked[tf] + 2e-4
            T[0] = 1e20
            return T, None, None

    checked = {1: np.linspace(0.0, 5.0, 50), 4: np.linspace(0.0, 7.0, 40),
               5: np.linspace(1.0, 9.0, 40)}
    err, diff = bench.max_error_ms(FakeCtx(), checked, 0b101)
    assert abs(err - 0.2) < 1e-9 and diff == 3
