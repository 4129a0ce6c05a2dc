"""bench.py on CPU: the clock sampler's summary of NVML reason bits and of
the nvidia-smi text fallback, that it degrades to an empty record (no
exception) on a host without a GPU, and the reference arm's JSON line."""
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


def test_reference_arm_line(tmp_path):
    """`bench.py --impl reference` prints one JSON line with the arm's keys
    (a tiny scene; each step is one view's CPU fwd+bwd)."""
    import json
    import subprocess
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "4096",
                        "--steps", "2", "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=tmp_path)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][-1])
    assert line["impl"] == "reference" and line["unit"] == "views/s" and line["value"] > 0
    assert line["steps"] == 2 and line["warmup"] == 1 and line["higher_is_better"] is True
    assert line["metric"] == bench.METRIC
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "views/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
