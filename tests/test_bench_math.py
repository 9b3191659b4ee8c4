"""bench.py's roofline and clock arithmetic on CPU: the issue-rate fraction from the
warp-instruction count, the peak's source, and the parsing of nvidia-smi clock samples
(median SM clock under load, throttle reasons seen in the region)."""

import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def test_issue_roofline_fraction():
    import bench
    r = bench.issue_roofline(9.87e9, {"sm_mhz": 1950.0})
    peak = 148 * 4 * 1950.0e6 / 1e9                 # G warp-instructions/s
    assert r["peak"] == pytest.approx(peak)
    assert r["achieved"] == pytest.approx(bench.WARP_INST_PER_UPDATE * 9.87)
    assert r["frac"] == pytest.approx(r["achieved"] / peak)
    assert 0.3 < r["frac"] < 0.5
    # without samples the max clock stands in
    assert bench.issue_roofline(1e9, None)["sm_mhz"] == 1965.0


def test_peak_source():
    import bench
    p = bench.peaks()
    if (ROOT / "MEASURED_PEAKS.json").exists():
        d = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        assert p == dict(hbm_gbs=float(d["hbm_gbs"]), source="measured")
    else:
        assert p == dict(hbm_gbs=bench.FALLBACK_HBM_GBS, source="fallback")


class _Done:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0


def test_clock_samples_parse(tmp_path):
    import bench
    rows = [
        "0, 1965, 1965, 120.5, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 900.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1935, 1965, 990.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1965, 1965, 800.0, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "garbage line",
    ]
    path = tmp_path / "clocks.csv"
    path.write_text("\n".join(rows) + "\n")
    s = bench.ClockSampler(0)
    s.proc, s.path, s.f = _Done(), str(path), open(tmp_path / "sink", "w")
    c = s.stop()
    assert c["samples"] == 4
    assert c["sm_mhz"] == 1950.0          # median of the samples above 250 W
    assert c["sm_max_mhz"] == 1965.0
    assert c["reasons"] == ["sw_power_cap"]
    assert c["power_w_max"] == 990.0
    assert not path.exists()


def test_clock_sampler_without_nvidia_smi_returns_none():
    import bench
    s = bench.ClockSampler(0)
    assert s.stop() is None
