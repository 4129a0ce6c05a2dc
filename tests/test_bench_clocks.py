"""bench.py's clock record on CPU: the sampler's summary of NVML reason bits
and of the nvidia-smi text fallback, and that it degrades to an empty record
(no exception) on a host without a GPU."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [ROOT, os.path.join(ROOT, "del-splat_b200")]

import bench  # noqa: E402


def test_nvml_samples_and_reason_bits():
    c = bench.ClockSampler(0)
    c.samples = [(1965, 1965, 0x0), (1950, 1965, 0x4), (1965, 1965, 0x4 | 0x40)]
    s = c.summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0 and s["samples"] == 3
    assert s["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]


def test_nvidia_smi_lines():
    c = bench.ClockSampler(0)
    c.lines = ["0, 1965, 1965, 700.5, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
               "0, 1800, 1965, 990.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
               "garbled"]
    s = c.summary()
    assert s["samples"] == 2 and s["sm_mhz"] == (1965 + 1800) / 2 and s["reasons"] == ["sw_power_cap"]


def test_sampler_without_gpu_records_nothing():
    with bench.ClockSampler(0, period_s=0.001) as c:
        pass
    s = c.summary()
    assert s["samples"] == len(c.samples) + sum(1 for _ in c.lines if _.count(",") >= 8)
