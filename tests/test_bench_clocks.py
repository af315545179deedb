"""The bench's clock record on CPU, against a fake NVML: SM clocks and
clock-event reasons are sampled only between begin() and end() (the timed
steps), and the reason bits map to the names of the run's acceptance rules
(hw_slowdown, hw_thermal_slowdown, sw_thermal_slowdown, sw_power_cap).
Nothing is set through NVML: the fake offers only queries."""
import os
import sys
import time
import types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _fake_nvml(state):
    m = types.ModuleType("pynvml")
    m.NVML_CLOCK_SM = 1
    m.nvmlInit = lambda: None
    m.nvmlShutdown = lambda: None

    def by_uuid(u):
        raise RuntimeError("no such device")

    m.nvmlDeviceGetHandleByUUID = by_uuid
    m.nvmlDeviceGetHandleByIndex = lambda i: ("gpu", i)
    m.nvmlDeviceGetMaxClockInfo = lambda h, c: 1965
    m.nvmlDeviceGetClockInfo = lambda h, c: state["sm"]
    m.nvmlDeviceGetCurrentClocksEventReasons = lambda h: state["reasons"]
    return m


def test_clock_sampler_samples_the_timed_steps_only(monkeypatch):
    import bench
    state = {"sm": 1200, "reasons": 0x8}  # before begin(): hw_slowdown at a low clock
    monkeypatch.setitem(sys.modules, "pynvml", _fake_nvml(state))
    cs = bench.ClockSampler(0)
    cs.start()
    time.sleep(0.06)
    state.update(sm=1965, reasons=0x4)  # the timed steps: full clock, power cap
    cs.begin()
    time.sleep(0.12)
    cs.end()
    time.sleep(0.06)
    state.update(sm=900, reasons=0x40)  # after end(): not sampled
    time.sleep(0.06)
    r = cs.stop()
    assert r["samples"] >= 3, r
    assert r["sm_mhz"] == 1965 and r["sm_max_mhz"] == 1965, r
    assert r["reasons"] == ["sw_power_cap"], r
    assert r["source"].startswith("nvml")


def test_clock_sampler_reason_names():
    import bench
    assert bench.ClockSampler.REASON_BITS == {"sw_power_cap": 0x4, "hw_slowdown": 0x8,
                                              "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}
