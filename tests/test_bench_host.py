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
        with open(path) as f:
            assert kind == "measured" and v == float(json.load(f)["hbm_gbs"])
    else:
        assert (v, kind) == (6650.0, "fallback")


def test_taylor_green_cpu_baseline_line():
    pytest.importorskip("restated")
    b = bench.cpu_baseline_tgv(1)
    assert b["kind"] == "port" and b["cores"] == 1 and b["unit"] == bench.METRIC
    assert b["value"] > 0 and b["seconds"] > 0 and "32^3" in b["sample"]


def _state(u, p, n_extra_ghosts=0):
    from sph_b200 import layout
    import numpy as np
    n = len(u) + n_extra_ghosts
    S = np.zeros(n, dtype=layout.PART1)
    S["i_type"] = 1
    S["p_type"] = 1
    S["ux"][:len(u)], S["uy"][:len(u)], S["uz"][:len(u)] = np.asarray(u, np.float32).T
    S["pres"][:len(p)] = p
    S["buffer_type"][len(u):] = layout.BUFFER_PERIODIC_GHOST
    S["ux"][len(u):] = 99.0
    return S


def test_form_error_counts_u_limit_decisions_apart():
    import numpy as np
    u_ref = [[1.0, 0.0, 0.0]] * 8 + [[1.0, -0.59, 0.0]]
    u_new = [[1.0 + 1e-6, 0.0, 0.0]] * 8 + [[0.62, 19.97, 0.0]]   # one particle accepted at the limit
    p = np.linspace(1.0, 2.0, 9)
    B, A = _state(u_ref, p, n_extra_ghosts=3), _state(u_new, p, n_extra_ghosts=3)
    e = bench.form_error(A, B, 20.0)
    assert e["particles"] == 9                       # ghosts excluded
    assert e["u_limit_decided_differently"] == 1
    assert e["u_rel_l2"] > 1.0
    assert abs(e["u_rel_l2_other_particles"] - 1e-6) < 1e-7
    assert e["p_rel_l2"] == 0.0 and e["p_rel_max"] == 0.0


def test_form_error_of_equal_states_is_zero():
    import numpy as np
    u = np.random.default_rng(1).normal(size=(50, 3))
    S = _state(u, np.ones(50))
    e = bench.form_error(S, S.copy(), 20.0)
    assert e["u_rel_l2"] == 0.0 and e["u_limit_decided_differently"] == 0 and e["u_rel_l2_other_particles"] == 0.0
