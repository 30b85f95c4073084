"""bench.py's clock sampler on the CPU, against a fake NVML and a fake nvidia-smi.

The sampler only reads (clocks, power, event reasons); these tests check that
the readings become the `clocks` record of the bench line: the median SM clock,
the maximum, and every throttle reason seen while sampling.
"""

import sys
import time
import types

import pytest


def _fake_nvml(reasons_seq, fail_after=None):
    calls = {"n": 0, "shutdown": 0, "by_bus": None}

    def reasons(h):
        calls["n"] += 1
        if fail_after is not None and calls["n"] > fail_after:
            raise RuntimeError("NVML read failed")
        return reasons_seq[min(calls["n"] - 1, len(reasons_seq) - 1)]

    nv = types.SimpleNamespace(
        NVML_CLOCK_SM=1,
        nvmlClocksEventReasonSwPowerCap=0x4,
        nvmlClocksEventReasonHwSlowdown=0x8,
        nvmlClocksEventReasonSwThermalSlowdown=0x20,
        nvmlClocksEventReasonHwThermalSlowdown=0x40,
        nvmlInit=lambda: None,
        nvmlShutdown=lambda: calls.__setitem__("shutdown", calls["shutdown"] + 1),
        nvmlDeviceGetHandleByIndex=lambda i: ("idx", i),
        nvmlDeviceGetHandleByPciBusId=lambda b: calls.__setitem__("by_bus", b) or ("bus", b),
        nvmlDeviceGetClockInfo=lambda h, c: 1965 if calls["n"] % 2 else 1800,
        nvmlDeviceGetMaxClockInfo=lambda h, c: 1965,
        nvmlDeviceGetPowerUsage=lambda h: 812345,
        nvmlDeviceGetCurrentClocksEventReasons=reasons,
    )
    return nv, calls


def _sample(bench, seconds=0.15):
    s = bench.ClockSampler(0, period_s=0.005)
    with s:
        time.sleep(seconds)
    return s


def test_nvml_samples_and_reasons(monkeypatch):
    import bench

    nv, calls = _fake_nvml([0x4, 0x4, 0x4 | 0x8, 0x0])
    monkeypatch.setitem(sys.modules, "pynvml", nv)
    s = _sample(bench)
    out = s.summary()
    assert out["source"] == "nvml" and out["samples"] >= 5
    assert out["sm_max_mhz"] == 1965.0 and out["sm_mhz"] in (1800.0, 1882.5, 1965.0)
    assert out["reasons"] == ["hw_slowdown", "sw_power_cap"]
    assert s.rows[0][3] == "812.35"
    assert calls["shutdown"] == 1


def test_nvml_uses_the_pci_bus_id(monkeypatch):
    import bench

    nv, calls = _fake_nvml([0])
    monkeypatch.setitem(sys.modules, "pynvml", nv)
    monkeypatch.setattr(bench, "_pci_bus_id", lambda i: "00000000:3b:00.0")
    s = _sample(bench, 0.03)
    assert calls["by_bus"] == "00000000:3b:00.0" and s.summary()["reasons"] == []


def test_falls_back_to_nvidia_smi(monkeypatch):
    import bench

    nv, calls = _fake_nvml([0], fail_after=2)           # NVML answers twice, then fails
    monkeypatch.setitem(sys.modules, "pynvml", nv)
    line = "0, 1965, 1965, 700.00, 0x0000000000000004, Not Active, Not Active, Active, Active\n"
    seen = []

    def fake_run(cmd, **kw):
        seen.append(cmd)
        return types.SimpleNamespace(stdout=line)

    monkeypatch.setattr(bench.subprocess, "run", fake_run)
    s = bench.ClockSampler(0, period_s=0.005)
    with s:
        time.sleep(0.5)
    out = s.summary()
    assert out["source"] == "nvidia-smi" and seen and seen[0][1] == "--id=0"
    assert out["reasons"] == ["sw_power_cap", "sw_thermal_slowdown"]
    assert out["samples"] >= 3


def test_no_nvml_module(monkeypatch):
    import bench

    monkeypatch.setitem(sys.modules, "pynvml", None)    # import fails
    monkeypatch.setattr(bench.subprocess, "run",
                        lambda cmd, **kw: types.SimpleNamespace(stdout=""))
    s = bench.ClockSampler(0)
    assert s.source == "nvidia-smi"
    with s:
        time.sleep(0.05)
    assert s.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0,
                           "source": "nvidia-smi"}


def test_smi_bus_id_refused_falls_back_to_index(monkeypatch):
    import bench

    monkeypatch.setitem(sys.modules, "pynvml", None)
    monkeypatch.setattr(bench, "_pci_bus_id", lambda i: "00000000:3b:00.0")
    line = "0, 1965, 1965, 700.00, 0x0, Not Active, Not Active, Not Active, Not Active\n"
    seen = []

    def fake_run(cmd, **kw):
        seen.append(cmd[1])
        ok = cmd[1] == "--id=0"
        return types.SimpleNamespace(stdout=line if ok else "No devices were found\n")

    monkeypatch.setattr(bench.subprocess, "run", fake_run)
    s = bench.ClockSampler(0)
    with s:
        time.sleep(0.5)
    out = s.summary()
    assert seen[:3] == ["--id=00000000:3b:00.0", "--id=0", "--id=0"]
    assert out["samples"] >= 2 and out["sm_mhz"] == 1965.0 and out["reasons"] == []
