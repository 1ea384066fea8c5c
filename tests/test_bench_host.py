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


def test_reference_arm_line_at_small_sizes():
    """--impl reference on the host cores (no GPU): one JSON line with the
    measured calibration run, the bounded samples and the CPU-runnable
    configurations at one and all threads."""
    import json
    import os
    import subprocess
    import sys

    import pytest

    from oracle.ffi import REF_PI, REF_SO
    if not (os.path.exists(REF_PI) and os.path.exists(REF_SO)):
        pytest.skip("oracle/_ref not built (the reference sources are not in this checkout)")
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, os.path.join(bench.ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "1", "--digits", "1000000", "--ref-sample", "10000",
                        "--ref-calibration", "100000"], capture_output=True, text=True, env=env, timeout=600,
                       check=True)
    line = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][-1])
    assert line["impl"] == "reference" and line["unit"] == "s" and line["higher_is_better"] is False
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    small = line["cpu_runnable_configs"]
    assert "error" not in small, small
    assert small["pi_1e6_s"]["1"] > 0
    assert set(small["isolated_products_s"]) == {"12", "16", "20"}
