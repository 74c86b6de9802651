"""Host-side pieces of bench.py that need no GPU: the clock sampler against a fake NVML."""
import importlib.util
import os
import sys
import time
import types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def fake_nvml(clocks, reasons):
    m = types.ModuleType("pynvml")
    m.NVML_CLOCK_SM = 1
    m.nvmlClocksEventReasonHwSlowdown = 0x8
    m.nvmlClocksEventReasonSwPowerCap = 0x4
    m.nvmlClocksEventReasonSwThermalSlowdown = 0x20
    m.nvmlClocksEventReasonHwThermalSlowdown = 0x40
    state = {"i": 0, "uuid": None}
    m.nvmlInit = lambda: None

    def by_uuid(u):
        state["uuid"] = u
        return "handle"

    def clock(h, kind):
        assert h == "handle" and kind == 1
        state["i"] += 1
        return clocks[min(state["i"] - 1, len(clocks) - 1)]

    m.nvmlDeviceGetHandleByUUID = by_uuid
    m.nvmlDeviceGetMaxClockInfo = lambda h, kind: 1965
    m.nvmlDeviceGetClockInfo = clock
    m.nvmlDeviceGetCurrentClocksEventReasons = lambda h: reasons
    return m, state


def test_clock_sampler_reads_nvml_by_uuid(monkeypatch):
    import torch
    bench = load_bench()
    m, state = fake_nvml([1965, 1965, 1900, 1965], 0x4)
    monkeypatch.setitem(sys.modules, "pynvml", m)
    monkeypatch.setattr(torch.cuda, "get_device_properties",
                        lambda d: types.SimpleNamespace(uuid="0123abcd-0000-1111-2222-333344445555"))
    s = bench.ClockSampler(0, 0)
    s.start()
    time.sleep(0.08)
    out = s.stop()
    assert state["uuid"] == "GPU-0123abcd-0000-1111-2222-333344445555"
    assert out["samples"] >= 2 and out["sm_max_mhz"] == 1965.0
    assert out["sm_mhz"] in (1900.0, 1965.0) and out["sm_mhz_min"] <= out["sm_mhz"]
    assert out["reasons"] == ["sw_power_cap"] and out["source"].startswith("nvml")


def test_clock_sampler_without_nvml_or_nvidia_smi(monkeypatch):
    bench = load_bench()
    broken = types.ModuleType("pynvml")          # no nvmlInit: NVML unusable

    def no_smi(*a, **k):
        raise FileNotFoundError("nvidia-smi")

    monkeypatch.setitem(sys.modules, "pynvml", broken)
    monkeypatch.setattr(bench.subprocess, "Popen", no_smi)
    s = bench.ClockSampler(0, 0)
    s.start()
    out = s.stop()
    assert out["sm_mhz"] is None and out["reasons"] == ["nvidia-smi unavailable"]
