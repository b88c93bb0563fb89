"""Host logic of bench.py that needs no GPU: the clock sampler against a fake NVML."""

import sys
import time
import types

import pytest

import bench


def _fake_nvml(reason_bits, clocks=(1965, 1950, 1965)):
    """A stand-in for pynvml: fixed max clock, SM clocks cycling through ``clocks``,
    clock-event reasons ``reason_bits``; the UUID lookup fails (no CUDA device here)
    so the sampler falls back to the device index."""
    nv = types.ModuleType("pynvml")
    nv.NVML_CLOCK_SM = 1
    calls = {"init": 0, "by_index": [], "n": 0}

    class NVMLError(Exception):
        pass

    def init():
        calls["init"] += 1

    def by_uuid(u):
        raise NVMLError("no such device")

    def by_index(i):
        calls["by_index"].append(i)
        return ("handle", i)

    def max_clock(h, kind):
        assert kind == nv.NVML_CLOCK_SM
        return 1965

    def clock(h, kind):
        calls["n"] += 1
        return clocks[calls["n"] % len(clocks)]

    nv.NVMLError = NVMLError
    nv.nvmlInit = init
    nv.nvmlDeviceGetHandleByUUID = by_uuid
    nv.nvmlDeviceGetHandleByIndex = by_index
    nv.nvmlDeviceGetMaxClockInfo = max_clock
    nv.nvmlDeviceGetClockInfo = clock
    nv.nvmlDeviceGetCurrentClocksEventReasons = lambda h: reason_bits
    return nv, calls


@pytest.mark.parametrize("bits, names", [
    (0, []),
    (0x4, ["sw_power_cap"]),
    (0x8 | 0x40, ["hw_slowdown", "hw_thermal_slowdown"]),
    (0x20 | 0x80, ["hw_power_brake_slowdown", "sw_thermal_slowdown"]),
    (0x1 | 0x2, []),  # idle / application-clock bits are not slowdowns
])
def test_clock_sampler_nvml(monkeypatch, bits, names):
    nv, calls = _fake_nvml(bits)
    monkeypatch.setitem(sys.modules, "pynvml", nv)
    cs = bench.ClockSampler(3)
    cs.start()
    time.sleep(0.06)
    out = cs.stop()
    assert calls["init"] == 1 and calls["by_index"] == [3]
    assert out["source"].startswith("nvml")
    assert out["sm_max_mhz"] == 1965.0
    assert out["samples"] >= 2 and out["samples"] == calls["n"]
    assert out["sm_mhz"] in (1950.0, 1965.0)
    assert out["reasons"] == names


def test_clock_sampler_without_nvml_or_smi(monkeypatch):
    broken = types.ModuleType("pynvml")

    def fail():
        raise RuntimeError("driver not loaded")

    broken.nvmlInit = fail
    monkeypatch.setitem(sys.modules, "pynvml", broken)
    monkeypatch.setenv("PATH", "")
    cs = bench.ClockSampler(0)
    cs.start()
    out = cs.stop()
    assert out["sm_mhz"] is None and out["reasons"] == ["nvidia-smi unavailable"]
