"""Host-side pieces of bench.py on the CPU: the clock sampler against a fake
NVML (read-only queries; no GPU setting is touched), and its nvidia-smi
fallback parsing."""
import sys
import time
import types

from conftest import ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _fake_nvml(clocks, reasons, calls):
    m = types.ModuleType("pynvml")
    m.NVML_CLOCK_SM = 1
    state = {"i": 0}

    def clock(h, kind):
        assert kind == 1
        v = clocks[min(state["i"], len(clocks) - 1)]
        state["i"] += 1
        return v

    m.nvmlInit = lambda: calls.append("init")
    m.nvmlShutdown = lambda: calls.append("shutdown")
    m.nvmlDeviceGetHandleByUUID = lambda u: calls.append(("uuid", u)) or "h"
    m.nvmlDeviceGetHandleByIndex = lambda i: calls.append(("index", i)) or "h"
    m.nvmlDeviceGetClockInfo = clock
    m.nvmlDeviceGetMaxClockInfo = lambda h, kind: 1965
    m.nvmlDeviceGetCurrentClocksEventReasons = lambda h: reasons
    return m


def test_clock_sampler_polls_nvml(monkeypatch):
    calls = []
    monkeypatch.setitem(sys.modules, "pynvml", _fake_nvml([1965, 1965, 1900, 1965], 0x4 | 0x1, calls))
    with bench.ClockSampler(0, "GPU-1234") as c:
        time.sleep(0.05)
    s = c.summary()
    assert ("uuid", "GPU-1234") in calls and calls[-1] == "shutdown"
    assert s["source"].startswith("nvml") and s["samples"] >= 3
    assert s["sm_max_mhz"] == 1965 and s["sm_mhz"] == 1965 and s["sm_mhz_min"] == 1900
    assert s["reasons"] == ["sw_power_cap"]  # 0x1 (idle) is not a reported reason


def test_clock_sampler_reports_slowdowns(monkeypatch):
    monkeypatch.setitem(sys.modules, "pynvml", _fake_nvml([1200], 0x8 | 0x20 | 0x40, []))
    with bench.ClockSampler(0) as c:
        time.sleep(0.02)
    assert c.summary()["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]


def test_clock_sampler_nvidia_smi_lines():
    c = bench.ClockSampler(0)
    c.lines = ["0, 1965, 1965, 700.1, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
               "0, 1950, 1965, 710.0, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
               "garbage"]
    s = c.summary()
    assert s["samples"] == 2 and s["sm_max_mhz"] == 1965 and s["reasons"] == ["sw_power_cap"]
    assert s["source"].startswith("nvidia-smi")


def test_algorithmic_bytes_per_pass():
    """Per fluid or interface cell: stream-collide 86 B (+9 B per interface
    cell), FS_1 93 B, the flag pass 39 B with FP32 populations; FP16S
    storage halves the population bytes only."""
    counts = {"fluid": 1000, "interface": 10, "gas": 5000, "wall": 100}
    b32 = bench.algorithmic_bytes(counts)
    assert b32 == {"stream_collide": 1010 * 86.0 + 10 * 9.0, "fs1": 1010 * 93.0, "fs234": 1010 * 39.0}
    b16 = bench.algorithmic_bytes(counts, 2.0)
    assert b16["stream_collide"] == 1010 * (86.0 - 36.0) + 10 * 9.0
    assert b16["fs1"] == 1010 * (93.0 - 34.0)
    assert b16["fs234"] == b32["fs234"]


def test_pass_shares_and_traffic_cover_the_three_passes():
    """The launch-list shares that split the measured step among the three
    free-surface passes name the same passes as the algorithmic bytes, add
    up to the step (within the rounding of the committed figures), and each
    pass has a per-launch DRAM traffic figure."""
    counts = {"fluid": 1, "interface": 0, "gas": 0, "wall": 0}
    passes = set(bench.algorithmic_bytes(counts))
    assert set(bench.PASS_SHARE_NCU) == passes
    assert set(bench.TRAFFIC_NCU) == passes
    assert abs(sum(bench.PASS_SHARE_NCU.values()) - 1.0) < 0.01
    assert all(0.0 < v < 1.0 for v in bench.PASS_SHARE_NCU.values())
    assert all(v > 0 for v in bench.TRAFFIC_NCU.values())
