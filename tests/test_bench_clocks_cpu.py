"""The bench's clock samplers on the CPU, against fakes of their sources.

The JSON line's `clocks` object (median SM clock under load, the maximum, and
which throttle reasons were seen active) is read either from an nvidia-smi
process's CSV lines or from NVML in the bench's own process. Both are checked
here with made-up readings: a fake NVML module and a fake nvidia-smi output.
"""
import os
import sys
import time
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def fake_nvml(readings):
    """A stand-in for pynvml returning `readings` (sm MHz, mW, reason bits) in turn."""
    m = types.ModuleType("pynvml")
    m.NVML_CLOCK_SM = 1
    m.nvmlClocksEventReasonSwPowerCap = 4
    m.nvmlClocksEventReasonHwSlowdown = 8
    m.nvmlClocksEventReasonSwThermalSlowdown = 32
    m.nvmlClocksEventReasonHwThermalSlowdown = 64
    state = {"i": 0, "bus": None, "shutdown": False}

    def cur():
        return readings[min(state["i"], len(readings) - 1)]

    def clock(h, kind):
        assert kind == m.NVML_CLOCK_SM
        return cur()[0]

    def power(h):
        return cur()[1]

    def reasons(h):
        r = cur()[2]
        state["i"] += 1
        return r

    def by_bus(bus):
        state["bus"] = bus
        return "handle"

    m.nvmlInit = lambda: None
    m.nvmlShutdown = lambda: state.__setitem__("shutdown", True)
    m.nvmlDeviceGetHandleByPciBusId = by_bus
    m.nvmlDeviceGetMaxClockInfo = lambda h, kind: 1965
    m.nvmlDeviceGetClockInfo = clock
    m.nvmlDeviceGetPowerUsage = power
    m.nvmlDeviceGetCurrentClocksEventReasons = reasons
    return m, state


class FakeProps:
    pci_domain_id = 0
    pci_bus_id = 0x1B
    pci_device_id = 0


def run_nvml_sampler(monkeypatch, readings):
    m, state = fake_nvml(readings)
    monkeypatch.setitem(sys.modules, "pynvml", m)
    import torch
    monkeypatch.setattr(torch.cuda, "get_device_properties", lambda d: FakeProps())
    s = bench.NvmlClockSampler(0)
    monkeypatch.setattr(s.halt, "wait", lambda t: time.sleep(0.001))
    s.start()
    deadline = time.time() + 5
    while state["i"] < len(readings) and time.time() < deadline:
        time.sleep(0.005)
    return s.stop(), state


def test_nvml_sampler_reports_median_max_and_the_reasons_seen(monkeypatch):
    readings = [(1965, 700_000, 0), (1950, 980_000, 4), (1965, 990_000, 4 | 1), (1965, 800_000, 0)]
    out, state = run_nvml_sampler(monkeypatch, readings)
    assert state["bus"] == "00000000:1b:00.0"
    assert state["shutdown"]
    assert out["sm_max_mhz"] == 1965
    assert out["reasons"] == ["sw_power_cap"]
    assert out["samples"] >= len(readings)
    assert out["sm_mhz"] == 1965
    assert out["source"] == "nvml"


def test_nvml_sampler_names_every_rejecting_reason(monkeypatch):
    out, _ = run_nvml_sampler(monkeypatch, [(1200, 500_000, 8), (1100, 500_000, 64 | 32)])
    assert out["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]
    assert out["sm_mhz"] <= 1200


def test_nvml_sampler_without_nvml_says_so(monkeypatch):
    m = types.ModuleType("pynvml")

    def fail():
        raise RuntimeError("no driver")
    m.nvmlInit = fail
    monkeypatch.setitem(sys.modules, "pynvml", m)
    s = bench.NvmlClockSampler(0)
    s.start()
    assert s.stop() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["NVML unavailable"]}


class FakeProc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0


def test_nvidia_smi_sampler_parses_its_csv_lines():
    s = bench.ClockSampler(0)
    s.proc = FakeProc()
    s.lines = [
        "0, 1965, 1965, 712.40, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 995.10, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1965, 1965, 990.00, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "garbage",
    ]
    out = s.stop()
    assert out == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"],
                   "samples": 3}


@pytest.mark.parametrize("col,name", [(5, "hw_slowdown"), (6, "hw_thermal_slowdown"),
                                      (7, "sw_thermal_slowdown")])
def test_nvidia_smi_sampler_flags_rejecting_reasons(col, name):
    parts = ["0", "1500", "1965", "600.0", "0x1"] + ["Not Active"] * 4
    parts[col] = "Active"
    s = bench.ClockSampler(0)
    s.proc = FakeProc()
    s.lines = [", ".join(parts)]
    assert s.stop()["reasons"] == [name]
