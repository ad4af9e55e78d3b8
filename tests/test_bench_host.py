"""Host logic of bench.py that needs no GPU: the clock sampler's reading of NVML, against a fake
NVML module (read-only queries: current and maximum SM clock, active clock-event reasons)."""
import sys
import time
import types

import bench


def fake_nvml(clocks, reasons):
    m = types.ModuleType("pynvml")
    state = {"i": 0}
    m.NVML_CLOCK_SM = 1
    m.nvmlInit = lambda: None
    m.nvmlDeviceGetHandleByIndex = lambda i: ("gpu", i)
    m.nvmlDeviceGetHandleByUUID = lambda u: ("gpu", u)
    m.nvmlDeviceGetHandleByPciBusId = lambda b: ("gpu", b)

    def clock(h, kind):
        v = clocks[min(state["i"], len(clocks) - 1)]
        state["i"] += 1
        return v

    m.nvmlDeviceGetClockInfo = clock
    m.nvmlDeviceGetMaxClockInfo = lambda h, kind: 1965
    m.nvmlDeviceGetCurrentClocksEventReasons = lambda h: reasons
    return m


def test_sampler_reads_clocks_and_reasons(monkeypatch):
    monkeypatch.setitem(sys.modules, "pynvml", fake_nvml([1965, 1950, 1965, 1965, 1900], 0x4 | 0x40))
    with bench.ClockSampler(0) as clk:
        time.sleep(0.15)
    s = clk.summary()
    assert s["source"] == "nvml, 20 ms"
    assert s["samples"] >= 3
    assert s["sm_max_mhz"] == 1965
    assert 1900 <= s["sm_mhz"] <= 1965
    assert s["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]


def test_sampler_reports_no_reason_when_none_is_active(monkeypatch):
    monkeypatch.setitem(sys.modules, "pynvml", fake_nvml([1965], 0x1))  # GPU idle is not a slowdown
    with bench.ClockSampler(0) as clk:
        time.sleep(0.06)
    assert clk.summary()["reasons"] == []


def test_sampler_falls_back_without_nvml(monkeypatch):
    broken = types.ModuleType("pynvml")

    def fail():
        raise RuntimeError("no driver")

    broken.nvmlInit = fail
    monkeypatch.setitem(sys.modules, "pynvml", broken)
    with bench.ClockSampler(0) as clk:
        time.sleep(0.01)
    s = clk.summary()
    assert s.get("source") != "nvml, 20 ms"
    assert "reasons" in s
