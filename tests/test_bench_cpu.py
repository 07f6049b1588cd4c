"""Host-side pieces of bench.py that need no GPU: the clock sampler's
summary (against a stand-in for NVML that only answers reads) and the
profile values the bench line is built from."""
import sys
import time
import types

import bench


class FakeNvml(types.SimpleNamespace):
    """Answers the reads the sampler makes; every call is recorded."""

    def __init__(self, clocks, reasons):
        super().__init__()
        self.calls = []
        self.clocks, self.reasons, self.i = clocks, reasons, 0
        self.NVML_CLOCK_SM = 1
        self.nvmlClocksEventReasonHwSlowdown = 0x8
        self.nvmlClocksEventReasonHwThermalSlowdown = 0x40
        self.nvmlClocksEventReasonSwThermalSlowdown = 0x20
        self.nvmlClocksEventReasonSwPowerCap = 0x4

    def nvmlInit(self):
        self.calls.append("init")

    def nvmlDeviceGetHandleByIndex(self, i):
        return ("dev", i)

    def nvmlDeviceGetHandleByUUID(self, u):
        return ("dev", u)

    def nvmlDeviceGetMaxClockInfo(self, h, kind):
        return 1965

    def nvmlDeviceGetClockInfo(self, h, kind):
        v = self.clocks[min(self.i, len(self.clocks) - 1)]
        self.i += 1
        return v

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        return self.reasons


def test_clock_sampler_summary_from_nvml(monkeypatch):
    fake = FakeNvml([1965, 1965, 1950], 0x4)
    monkeypatch.setitem(sys.modules, "pynvml", fake)
    with bench.ClockSampler(0, period_s=0.001) as c:
        time.sleep(0.02)
    s = c.summary()
    assert s["samples"] >= 3 and s["sm_max_mhz"] == 1965.0
    assert s["sm_mhz"] in (1950.0, 1965.0)
    assert s["reasons"] == ["sw_power_cap"]
    # only reads: no call that changes a setting exists on the stand-in
    assert not any(n.startswith("nvmlDeviceSet") for n in dir(fake))


def test_clock_sampler_reports_throttle_reasons(monkeypatch):
    fake = FakeNvml([1200], 0x8 | 0x20)
    monkeypatch.setitem(sys.modules, "pynvml", fake)
    with bench.ClockSampler(0, period_s=0.001) as c:
        time.sleep(0.01)
    assert c.summary()["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]


def test_traffic_comes_from_the_committed_profile():
    t = bench.load_traffic()
    assert isinstance(t, int) and t > 0
