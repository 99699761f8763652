"""The bench's clock record (bench.ClockSampler) from nvidia-smi's CSV lines: the median SM clock under
load, the highest maximum clock, and every throttle reason that any sample shows as Active; lines
that are not samples are skipped, and a run without nvidia-smi says so instead of inventing a clock."""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


class _Done:
    """A finished nvidia-smi process and its reader thread."""

    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0

    def join(self, timeout=None):
        pass


def _sampler(lines):
    c = bench.ClockSampler(0)
    c.proc = _Done()
    c.thread = _Done()
    c.lines = list(lines)
    return c


def test_median_clock_and_active_reasons():
    # index, clocks.sm, clocks.max.sm, power.draw, active mask, hw_slowdown, hw_thermal, sw_thermal, sw_power_cap
    lines = ["0, 1965, 1965, 812.4, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
             "0, 1950, 1965, 990.1, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
             "0, 1965, 1965, 870.0, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
             "garbage line",
             "0, [N/A], 1965, 870.0, 0x0, Not Active, Not Active, Not Active, Not Active"]
    out = _sampler(lines).stop()
    assert out["sm_mhz"] == 1965.0
    assert out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"]
    assert out["samples"] == 3


def test_thermal_reasons_are_reported():
    lines = ["0, 1400, 1965, 700.0, 0x48, Active, Not Active, Active, Not Active"]
    out = _sampler(lines).stop()
    assert out["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]


def test_no_samples_and_no_tool():
    assert _sampler([]).stop()["reasons"] == ["no samples"]
    c = bench.ClockSampler(0)
    c.proc = None
    assert c.stop() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
