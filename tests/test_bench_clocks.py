"""Clock record of bench.py on CPU: which samples count, and how clock-event reasons are read.

No GPU and no NVML here: the sampler is fed the samples its NVML poll and its nvidia-smi reader
would have collected, and stop() is checked on them."""
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402

# NVML clock-event reason bits (nvmlClocksEventReason*): sw power cap 0x4, hw slowdown 0x8,
# sw thermal 0x20, hw thermal 0x40
BITS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}


class _DoneProc:
    """Stands in for the nvidia-smi process after it printed its lines."""

    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0

    def kill(self):
        pass


def _sampler():
    c = bench.ClockSampler(0)
    c.bits = BITS
    c.max_mhz = 1965.0
    return c


def test_only_samples_inside_the_timed_windows_count():
    c = _sampler()
    c.windows = [(10.0, 11.0), (20.0, 21.0)]
    # idle samples before, between and after the windows run at a low clock with a reason set
    c.polled = [(9.5, 345.0, 0x8), (10.2, 1965.0, 0), (10.8, 1950.0, 0), (15.0, 345.0, 0x40),
                (20.5, 1965.0, 0x4), (22.0, 345.0, 0x20)]
    got = c.stop()
    assert got["samples"] == 3
    assert got["sm_mhz"] == 1965.0
    assert got["sm_max_mhz"] == 1965.0
    assert got["reasons"] == ["sw_power_cap"]
    assert got["source"].startswith("NVML")


def test_throttle_reasons_inside_a_window_are_reported():
    c = _sampler()
    c.windows = [(0.0, 1.0)]
    c.polled = [(0.1, 1200.0, 0x8 | 0x40), (0.2, 1300.0, 0x20), (0.3, 1965.0, 0)]
    got = c.stop()
    assert got["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]
    assert got["sm_mhz"] == 1300.0


def test_nvidia_smi_record_when_no_nvml_sample_is_inside():
    c = _sampler()
    c.windows = [(0.0, 1.0)]
    c.polled = [(5.0, 1965.0, 0)]
    c.proc = _DoneProc()
    # index, clocks.sm, clocks.max.sm, power.draw, active, hw_slowdown, hw_thermal, sw_thermal, sw_power_cap
    c.lines = ["0, 1965, 1965, 700.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
               "0, 1950, 1965, 990.5, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
               "0, 1965, 1965, 980.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
               "garbage line"]
    got = c.stop()
    assert got["source"] == "nvidia-smi -lms 200"
    assert got["samples"] == 3
    assert got["sm_mhz"] == 1965.0
    assert got["sm_max_mhz"] == 1965.0
    assert got["reasons"] == ["sw_power_cap"]


def test_no_record_at_all():
    c = _sampler()
    got = c.stop()
    assert got["sm_mhz"] is None
    assert got["reasons"] == ["nvidia-smi unavailable"]


def test_window_context_records_its_span():
    c = _sampler()
    with c.window():
        pass
    assert len(c.windows) == 1
    a, b = c.windows[0]
    assert a <= b
