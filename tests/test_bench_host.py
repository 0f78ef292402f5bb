"""Host-side logic of bench.py that needs no GPU: the clock sampler's
reading of NVML (through a fake NVML module, read-only queries only) and the
launch count per step."""
import time
import types

import bench


def _fake_nvml(clocks, masks):
    """A stand-in for the pynvml module: SM clock and clock-event reason
    mask per call, cycling through the given values."""
    state = {"i": 0}
    nv = types.SimpleNamespace(
        NVML_CLOCK_SM=0,
        nvmlClocksEventReasonSwPowerCap=0x4,
        nvmlClocksEventReasonHwSlowdown=0x8,
        nvmlClocksEventReasonSwThermalSlowdown=0x20,
        nvmlClocksEventReasonHwThermalSlowdown=0x40,
    )

    def clock(h, kind):
        assert h == "handle" and kind == nv.NVML_CLOCK_SM
        return clocks[state["i"] % len(clocks)]

    def reasons(h):
        m = masks[state["i"] % len(masks)]
        state["i"] += 1
        return m

    nv.nvmlDeviceGetClockInfo = clock
    nv.nvmlDeviceGetMaxClockInfo = lambda h, kind: 1965
    nv.nvmlDeviceGetCurrentClocksEventReasons = reasons
    nv.shutdowns = 0

    def shutdown():
        nv.shutdowns += 1

    nv.nvmlShutdown = shutdown
    return nv


def test_clock_sampler_reads_nvml(monkeypatch):
    nv = _fake_nvml([1965, 1950, 1965], [0, 0x4, 0x1])   # 0x1 (idle) is not reported
    monkeypatch.setattr(bench.ClockSampler, "_nvml_handle", lambda self: (nv, "handle"))
    with bench.ClockSampler(0) as c:
        time.sleep(0.08)
    s = c.summary()
    assert s["source"].startswith("nvml")
    assert s["samples"] >= 2
    assert s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    assert 1950.0 <= s["sm_mhz"] <= 1965.0
    assert nv.shutdowns == 1


def test_clock_sampler_flags_throttling(monkeypatch):
    nv = _fake_nvml([1200], [0x8 | 0x40])
    monkeypatch.setattr(bench.ClockSampler, "_nvml_handle", lambda self: (nv, "handle"))
    with bench.ClockSampler(0) as c:
        pass
    s = c.summary()
    assert s["reasons"] == ["hw_slowdown", "hw_thermal_slowdown"]
    assert s["sm_mhz"] == 1200.0


def test_clock_sampler_without_nvml(monkeypatch):
    def fail(self):
        raise RuntimeError("no NVML")
    monkeypatch.setattr(bench.ClockSampler, "_nvml_handle", fail)
    monkeypatch.setattr(bench.subprocess, "Popen", lambda *a, **k: (_ for _ in ()).throw(OSError()))
    with bench.ClockSampler(0) as c:
        pass
    assert c.summary()["reasons"] == ["unsampled"]


def test_kernels_per_step():
    # The finiteness flag, the decimation (6 kernels, or one copy when the
    # rate needs no decimation), then 15 kernels of the fixed stages (the
    # launch list of one pipeline pass counts 22 at 16 kHz).
    assert bench.kernels_per_step(2) == 22
    assert bench.kernels_per_step(1) == 17
