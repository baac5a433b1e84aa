"""Clock sampling around a timed region, against a fake NVML (no GPU)."""
import subprocess
import time

from fastwigner_b200.benchmarks import ClockSampler


class FakeNvml:
    NVML_CLOCK_SM = 1

    def __init__(self, reasons):
        self.reasons = reasons
        self.calls = 0

    def nvmlDeviceGetClockInfo(self, h, kind):
        self.calls += 1
        return 1800 + 10 * (self.calls % 3)

    def nvmlDeviceGetMaxClockInfo(self, h, kind):
        return 1965

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        return self.reasons

    def nvmlShutdown(self):
        pass


def _use(monkeypatch, fake):
    def handle(self):
        self._nvml = fake
        return object()

    monkeypatch.setattr(ClockSampler, "_nvml_handle", handle)


def test_samples_while_the_region_runs(monkeypatch):
    fake = FakeNvml(0x4)
    _use(monkeypatch, fake)
    with ClockSampler(device_index=0, interval=0.001) as clk:
        time.sleep(0.05)
    s = clk.summary()
    assert s["source"] == "nvml"
    assert s["samples"] >= 5
    assert s["sm_max_mhz"] == 1965
    assert 1800 <= s["sm_mhz"] <= 1820
    assert s["reasons"] == ["sw_power_cap"]
    n = fake.calls
    time.sleep(0.01)
    assert fake.calls == n  # the thread stops at exit


def test_reason_bits(monkeypatch):
    _use(monkeypatch, FakeNvml(0x8 | 0x40 | 0x20))
    with ClockSampler(device_index=0, interval=0.001) as clk:
        time.sleep(0.01)
    assert clk.summary()["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]


def test_unsampled_without_nvml_or_nvidia_smi(monkeypatch):
    def no_nvml(self):
        raise RuntimeError("NVML unavailable")

    def no_smi(*a, **k):
        raise OSError("nvidia-smi not found")

    monkeypatch.setattr(ClockSampler, "_nvml_handle", no_nvml)
    monkeypatch.setattr(subprocess, "Popen", no_smi)
    with ClockSampler(device_index=0) as clk:
        pass
    assert clk.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
