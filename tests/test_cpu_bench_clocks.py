"""bench.py's clock record on CPU: the summary of nvidia-smi samples (median
SM clock, throttle reasons that reject a run) and the untimed fill that gives
timed regions shorter than the sampling period their readings."""
import time

import bench


class _FakeProc:
    pass


def _sampler(tmp_path, lines=None):
    c = bench.ClockSampler(0)
    c.path = str(tmp_path / "clocks.csv")
    if lines is not None:
        with open(c.path, "w") as f:
            f.write("\n".join(lines) + "\n")
    c.proc = _FakeProc()
    return c


def test_summary_median_and_reasons(tmp_path):
    # index, clocks.sm, clocks.max.sm, power, active mask, hw_slowdown,
    # hw_thermal_slowdown, sw_thermal_slowdown, sw_power_cap
    rows = ["0, 1965, 1965, 700.5, 0x0, Not Active, Not Active, Not Active, Not Active",
            "0, 1900, 1965, 980.0, 0x4, Not Active, Not Active, Not Active, Active",
            "0, 1965, 1965, 720.0, 0x0, Not Active, Not Active, Not Active, Not Active",
            "garbage line"]
    s = _sampler(tmp_path, rows).summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["samples"] == 3
    assert s["reasons"] == ["sw_power_cap"]
    rows.append("0, 1200, 1965, 500.0, 0x40, Not Active, Active, Not Active, Not Active")
    assert "hw_thermal_slowdown" in _sampler(tmp_path, rows).summary()["reasons"]


def test_summary_without_sampler():
    c = bench.ClockSampler(0)
    assert c.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}


def test_fill_runs_only_for_short_regions(tmp_path):
    c = _sampler(tmp_path)
    calls = []
    t0 = time.perf_counter()
    assert c.fill(lambda: calls.append(1), t0, min_s=0.05)
    assert calls and time.perf_counter() - t0 >= 0.05
    calls.clear()
    # a region already longer than min_s: nothing runs
    assert not c.fill(lambda: calls.append(1), time.perf_counter() - 1.0, min_s=0.05)
    assert not calls
    # no sampler process: nothing runs
    c.proc = None
    assert not c.fill(lambda: calls.append(1), time.perf_counter(), min_s=0.05)
    assert not calls
