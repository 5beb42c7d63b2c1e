"""Host-side pieces of bench.py that decide what a bench line reports, on CPU:
the clock summary (median SM clock, max clock, throttle reasons seen during
the timed region) from NVML samples and from nvidia-smi lines."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_clock_summary_from_nvml_samples():
    c = bench.ClockSampler(0)
    B = bench.ClockSampler.BITS
    c.samples = [(1965.0, 1965.0, 0), (1800.0, 1965.0, B["sw_power_cap"]), (1900.0, 1965.0, 0x1),
                 (1950.0, 1965.0, B["hw_slowdown"] | B["sw_power_cap"])]
    s = c.summary()
    assert s["sm_mhz"] == pytest.approx(1925.0)
    assert s["sm_max_mhz"] == 1965.0
    # bit 0x1 (GPU idle) is not a throttle reason the bench reports
    assert s["reasons"] == ["hw_slowdown", "sw_power_cap"]
    assert s["samples"] == 4 and s["source"] == "nvml"


def test_clock_summary_from_nvidia_smi_lines():
    c = bench.ClockSampler(0)
    c.lines = [
        "0, 1965, 1965, 612.30, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1312, 1965, 999.80, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1500, 1965, 800.00, 0x0000000000000020, Not Active, Not Active, Active, Not Active",
        "0, [N/A], 1965, 800.00, 0x0, Not Active, Not Active, Not Active, Not Active",
        "garbage line",
    ]
    s = c.summary()
    assert s["sm_mhz"] == 1500.0
    assert s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap", "sw_thermal_slowdown"]
    assert s["samples"] == 3 and s["source"] == "nvidia-smi"


def test_clock_summary_without_samples():
    s = bench.ClockSampler(0).summary()
    assert s["sm_mhz"] is None and s["sm_max_mhz"] is None and s["reasons"] == [] and s["samples"] == 0
