"""Host-side logic of bench.py (no GPU needed): the clock-record parsing that
decides whether a bench line is kept, the peak-bandwidth fallback, and the
CPU baseline of the Taylor-Green config."""
import json
import os
import sys
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


class _Proc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0

    def kill(self):
        pass


def _clocks_from(lines):
    c = bench.Clocks(0)
    fd, c.path = tempfile.mkstemp(suffix=".csv")
    with os.fdopen(fd, "w") as f:
        f.write("\n".join(lines) + "\n")
    c.proc = _Proc()
    return c.stop()


def test_clock_record_median_and_reasons():
    rows = ["0, 1965, 1965, 700.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
            "0, 1905, 1965, 990.2, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
            "0, 1950, 1965, 950.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
            "garbage line",
            "0, [N/A], 1965, 1.0, 0x0, Not Active, Not Active, Not Active, Not Active"]
    ck = _clocks_from(rows)
    assert ck["samples"] == 3
    assert ck["sm_mhz"] == 1950 and ck["sm_max_mhz"] == 1965
    assert ck["reasons"] == ["sw_power_cap"]


def test_clock_record_flags_thermal_slowdown():
    rows = ["0, 1500, 1965, 990.0, 0x0000000000000040, Not Active, Active, Not Active, Active"]
    ck = _clocks_from(rows)
    assert ck["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]


def test_clock_record_without_samples_is_none():
    assert _clocks_from([]) is None
    assert bench.Clocks(0).stop() is None   # never started


def test_peak_bandwidth_source():
    v, kind = bench.peaks()
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        assert kind == "measured" and v == float(json.load(open(path))["hbm_gbs"])
    else:
        assert (v, kind) == (6650.0, "fallback")


def test_taylor_green_cpu_baseline_line():
    pytest.importorskip("restated")
    b = bench.cpu_baseline_tgv(1)
    assert b["kind"] == "port" and b["cores"] == 1 and b["unit"] == bench.METRIC
    assert b["value"] > 0 and b["seconds"] > 0 and "32^3" in b["sample"]
