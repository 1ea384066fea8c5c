"""bench.py's host-side helpers on CPU: the clock record taken from
nvidia-smi during the timed region, and the roofline denominator."""
from __future__ import annotations

import bench


class _FakeProc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0

    def kill(self):
        pass


def _sampler(lines):
    s = bench.ClockSampler(0)
    s.proc = _FakeProc()
    s.lines = list(lines)
    return s


def test_clock_record_median_max_and_reasons():
    # index, clocks.sm, clocks.max.sm, power, active, hw_slowdown, hw_thermal, sw_thermal, sw_power_cap
    lines = [
        "0, 1965, 1965, 800.1, 0x0, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 910.4, 0x4, Not Active, Not Active, Not Active, Active",
        "0, 1965, 1965, 905.0, 0x0, Not Active, Not Active, Not Active, Not Active",
        "garbage line",
        "0, [N/A], 1965, 0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ]
    rec = _sampler(lines).stop()
    assert rec["sm_mhz"] == 1965.0
    assert rec["sm_max_mhz"] == 1965.0
    assert rec["samples"] == 3
    assert rec["reasons"] == ["sw_power_cap"]


def test_clock_record_flags_thermal_slowdown():
    lines = ["0, 1500, 1965, 990, 0x40, Not Active, Active, Not Active, Not Active"]
    rec = _sampler(lines).stop()
    assert rec["reasons"] == ["hw_thermal_slowdown"]


def test_clock_record_without_nvidia_smi():
    s = bench.ClockSampler(0)
    rec = s.stop()
    assert rec["sm_mhz"] is None and rec["reasons"] == ["nvidia-smi unavailable"]


def test_measured_peak_is_read_from_the_driver_file():
    peak, kind = bench.measured_peaks()
    assert peak > 1000.0
    assert kind in ("measured", "fallback")
