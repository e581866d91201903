"""bench.py's own arithmetic on CPU: the algorithmic bytes of one SpMV (the
figure the roofline divides by the measured launch time), the peak it divides
by (the measured copy bandwidth, else the stated fallback), and the workloads
the line is quoted on."""
import json
import os

import bench


def test_spmv_algorithmic_bytes():
    # C2: 4,280,989 stored upper blocks, 551,368 block rows
    U, nb = 4_280_989, 551_368
    assert bench.spmv_bytes(U, nb, 4) == U * 40 + 4 * (nb + 1) + 3 * nb * 8 == 186_677_868
    assert bench.spmv_bytes(U, nb, 8) == U * 76 + 4 * (nb + 1) + 3 * nb * 16
    assert bench.spmv_bytes(0, 0, 4) == 4


def test_peak_is_the_measured_copy_bandwidth_else_the_fallback(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench._peaks() == (6650.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6449.1, "bf16_tflops": 1500.0}))
    assert bench._peaks() == (6449.1, "measured")


def test_workloads():
    w = bench.WORKLOADS
    assert w["stack8x40"] == dict(cells=40, n_cubes=8, seed=0)
    assert w["cube10"]["cells"] == 10 and w["cube10"]["n_cubes"] == 1
    for name, cfg in w.items():
        assert {"cells", "n_cubes", "seed"} <= set(cfg), name


class _FakeNVML:
    """Read-only NVML stand-in: a clock that cycles through three values and a
    power-cap reason bit on every other sample."""

    NVML_CLOCK_SM = 1
    nvmlClocksEventReasonHwSlowdown = 0x8
    nvmlClocksEventReasonHwThermalSlowdown = 0x40
    nvmlClocksEventReasonSwThermalSlowdown = 0x20
    nvmlClocksEventReasonSwPowerCap = 0x4

    def __init__(self):
        self.k = 0

    def nvmlDeviceGetMaxClockInfo(self, h, which):
        return 1965

    def nvmlDeviceGetClockInfo(self, h, which):
        self.k += 1
        return (1965, 1950, 1965)[self.k % 3]

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        return self.nvmlClocksEventReasonSwPowerCap if self.k % 2 else 0


def test_clock_sampler_reads_nvml(monkeypatch):
    import time

    fake = _FakeNVML()
    monkeypatch.setattr(bench.ClockSampler, "_nvml_handle", lambda self: (fake, object()))
    c = bench.ClockSampler(0)
    c.start()
    time.sleep(0.1)
    r = c.stop()
    assert r["source"] == "nvml" and r["samples"] >= 3
    assert r["sm_mhz"] in (1950, 1965) and r["sm_max_mhz"] == 1965
    assert r["reasons"] == ["sw_power_cap"]  # no slowdown reason: the run stands


def test_clock_sampler_without_nvml_or_nvidia_smi(monkeypatch):
    def no_nvml(self):
        raise RuntimeError("no NVML")

    monkeypatch.setattr(bench.ClockSampler, "_nvml_handle", no_nvml)
    monkeypatch.setenv("PATH", "/nonexistent")
    c = bench.ClockSampler(0)
    c.start()
    assert c.stop() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
