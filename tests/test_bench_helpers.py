"""bench.py's host helpers on the CPU: the clock sampler against a stand-in
nvidia-smi that prints fixed rows (median and maximum clocks, the throttle
reasons that reject a run), and the roofline's peak and traffic sources."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def fake_smi(tmp_path, rows):
    script = tmp_path / "nvidia-smi"
    lines = "".join(f"echo '{r}'\n" for r in rows)
    script.write_text("#!/bin/sh\n" + lines + "exec sleep 30\n")
    script.chmod(0o755)
    return str(tmp_path)


def sample(tmp_path, monkeypatch, rows):
    monkeypatch.setenv("PATH", fake_smi(tmp_path, rows) + os.pathsep + os.environ["PATH"])
    sys.path.insert(0, ROOT)
    import bench
    s = bench.ClockSampler(0)
    s.start()
    return s.stop()


NA, A = "Not Active", "Active"


def test_clock_sampler_power_cap_only(tmp_path, monkeypatch):
    rows = [f"0, {mhz}, 1965, 990.0, 0x4, {NA}, {NA}, {NA}, {A}" for mhz in (1965, 1800, 1900)]
    c = sample(tmp_path, monkeypatch, rows)
    assert c["samples"] == 3 and c["sm_mhz"] == 1900 and c["sm_max_mhz"] == 1965
    assert c["reasons"] == ["sw_power_cap"]


def test_clock_sampler_reports_rejecting_reasons(tmp_path, monkeypatch):
    rows = [f"0, 1965, 1965, 500.0, 0x0, {NA}, {NA}, {NA}, {NA}",
            f"0, 1400, 1965, 500.0, 0x8, {A}, {NA}, {NA}, {NA}",
            f"0, 1300, 1965, 500.0, 0x40, {NA}, {A}, {A}, {NA}",
            "0, [N/A], [N/A], [N/A], [N/A], [N/A], [N/A], [N/A], [N/A]"]
    c = sample(tmp_path, monkeypatch, rows)
    assert c["samples"] == 4 and c["sm_mhz"] == 1400 and c["sm_max_mhz"] == 1965
    assert c["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]


def test_peak_and_traffic_sources():
    sys.path.insert(0, ROOT)
    import bench
    peak, kind = bench.load_peak()
    if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")):
        assert kind == "measured" and peak > 0
    else:
        assert (peak, kind) == (bench.FALLBACK_HBM_GBS, "fallback")
    for kernel in ("ntt_fwd", "ntt_inv"):
        t = bench.load_traffic(kernel, 262144)
        # DRAM bytes per launch from the committed ncu summary: at most the
        # algorithmic 1024 B per polynomial (L2 absorbs part of the writes)
        assert t is not None and 0 < t <= 1024 * 262144
    assert bench.load_traffic("no_such_kernel", 1) is None


def test_clock_sampler_nvml_path(monkeypatch):
    """The NVML path against a stand-in pynvml: clocks and event-reason bits
    read every 2 ms while the sampler runs, so even a window of a few
    milliseconds has samples; median and maximum clocks, reason names."""
    import time
    import types
    fake = types.ModuleType("pynvml")
    fake.NVML_CLOCK_SM = 1
    fake.nvmlClocksEventReasonHwSlowdown = 0x8
    fake.nvmlClocksEventReasonHwThermalSlowdown = 0x40
    fake.nvmlClocksEventReasonSwThermalSlowdown = 0x20
    fake.nvmlClocksEventReasonSwPowerCap = 0x4
    clocks = iter([1965, 1800, 1900] * 1000)
    fake.nvmlInit = lambda: None
    fake.nvmlDeviceGetHandleByPciBusId = lambda bus: "h"
    fake.nvmlDeviceGetHandleByIndex = lambda i: "h"
    fake.nvmlDeviceGetMaxClockInfo = lambda h, c: 1965
    fake.nvmlDeviceGetClockInfo = lambda h, c: next(clocks)
    fake.nvmlDeviceGetCurrentClocksEventReasons = lambda h: 0x4 | 0x1   # power cap, idle
    monkeypatch.setitem(sys.modules, "pynvml", fake)
    sys.path.insert(0, ROOT)
    import bench
    s = bench.ClockSampler(0)
    s.start()
    time.sleep(0.02)
    c = s.stop()
    assert c["samples"] >= 3 and c["source"].startswith("nvml")
    assert c["sm_mhz"] in (1800, 1900, 1965) and c["sm_max_mhz"] == 1965
    assert c["reasons"] == ["sw_power_cap"]
