"""Host logic of bench.py's clock record on CPU: the NVML sampler polls
during the timed region and reports the median SM clock, the maximum and
every clock-event reason seen; without NVML it falls back to nvidia-smi and,
where that is absent too, says the region went unsampled.  A stand-in NVML
module replaces the real one (no GPU here)."""
import os
import sys
import time
import types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _fake_nvml(init_ok=True):
    m = types.ModuleType("pynvml")
    m.NVML_CLOCK_SM = 1
    state = {"n": 0, "shutdown": 0}

    def init():
        if not init_ok:
            raise RuntimeError("no driver")

    def by_uuid(u):
        raise RuntimeError("unknown uuid")

    def clock(h, kind):
        state["n"] += 1
        return 1965 if state["n"] % 2 else 1900

    def reasons(h):
        return 0x4 if state["n"] == 3 else 0

    m.nvmlInit = init
    m.nvmlShutdown = lambda: state.__setitem__("shutdown", state["shutdown"] + 1)
    m.nvmlDeviceGetHandleByUUID = by_uuid
    m.nvmlDeviceGetHandleByIndex = lambda i: ("handle", i)
    m.nvmlDeviceGetMaxClockInfo = lambda h, kind: 1965
    m.nvmlDeviceGetClockInfo = clock
    m.nvmlDeviceGetCurrentClocksEventReasons = reasons
    return m, state


def test_nvml_sampler_records_the_region(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    fake, state = _fake_nvml()
    monkeypatch.setitem(sys.modules, "pynvml", fake)
    with bench.ClockSampler(0) as clk:
        time.sleep(0.05)
    s = clk.summary()
    assert s["source"].startswith("nvml")
    assert s["samples"] >= 4 and s["samples"] == state["n"]
    assert s["sm_max_mhz"] == 1965 and s["sm_mhz"] in (1900, 1932.5, 1965)
    assert s["reasons"] == ["sw_power_cap"]
    assert state["shutdown"] == 1


def test_sampler_without_nvml_or_nvidia_smi_says_unsampled(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    fake, _ = _fake_nvml(init_ok=False)
    monkeypatch.setitem(sys.modules, "pynvml", fake)
    monkeypatch.setenv("PATH", "/nonexistent")
    with bench.ClockSampler(0) as clk:
        time.sleep(0.01)
    s = clk.summary()
    assert s["reasons"] == ["unsampled"] and s["sm_mhz"] is None
