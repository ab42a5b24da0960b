"""bench.py's host logic (no GPU).  The clock record: NVML samples are taken
only inside the timed region, throttle-reason bits map to their names, and a
missing or failing NVML falls back to the nvidia-smi samples without raising.
The reference arm: only rank 0 works."""
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


class FakeNVML:
    """The read-only NVML queries the sampler makes."""

    NVML_CLOCK_SM = 1

    def __init__(self, reasons=0x4, fail_init=False):
        self.reasons, self.fail_init = reasons, fail_init
        self.first_call = None
        self.shut = False

    def nvmlInit(self):
        if self.fail_init:
            raise RuntimeError("NVML unavailable")

    def nvmlShutdown(self):
        self.shut = True

    def nvmlDeviceGetHandleByIndex(self, i):
        return ("gpu", i)

    def nvmlDeviceGetMaxClockInfo(self, h, clock):
        return 1965

    def nvmlDeviceGetClockInfo(self, h, clock):
        if self.first_call is None:
            self.first_call = time.monotonic()
        return 1950

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        return self.reasons


def test_samples_inside_the_region_only():
    nv = FakeNVML(reasons=0x4 | 0x8)
    with bench.Clocks(0, nvml=nv) as ck:
        entered = time.monotonic()
        time.sleep(0.03)
    s = ck.summary()
    assert nv.first_call is not None and nv.first_call >= entered - 0.005
    assert s["source"].startswith("nvml") and s["samples"] >= 2
    assert s["sm_mhz"] == 1950.0 and s["sm_max_mhz"] is not None
    assert s["reasons"] == ["hw_slowdown", "sw_power_cap"]
    assert nv.shut


def test_failing_nvml_falls_back():
    nv = FakeNVML(fail_init=True)
    with bench.Clocks(0, nvml=nv) as ck:
        time.sleep(0.01)
    s = ck.summary()
    assert s.get("source") != "nvml, inside the timed region"
    assert set(s) >= {"sm_mhz", "sm_max_mhz", "reasons", "samples"}


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    """Under torchrun the reference arm's other ranks exit 0 without work and
    print nothing; rank 0 alone times the CPU search and prints the line."""
    def no_work(*a, **k):
        raise AssertionError("a rank other than 0 built the workload")

    monkeypatch.setattr(bench, "workload", no_work)
    monkeypatch.setenv("RANK", "1")
    assert bench.reference_arm(None) == 0
    assert capsys.readouterr().out == ""


def test_bench_flags(monkeypatch):
    """The default run carries the short filtered-serving grid (--no-filtered-serving
    drops it, --filtered-serving asks for the whole grid); --beam and --no-autotune
    are for profiling runs and default off."""
    import sys

    import bench

    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse()
    assert not a.no_filtered_serving and not a.filtered_serving and a.beam == 0 and not a.no_autotune
    monkeypatch.setattr(sys, "argv", ["bench.py", "--no-filtered-serving", "--beam", "40", "--no-autotune"])
    a = bench.parse()
    assert a.no_filtered_serving and a.beam == 40 and a.no_autotune
    assert bench.config_of(a, 1, 40, "fp32")["variant"] == "fp32"
    assert bench.config_of(a, 1, 40)["variant"] == bench.HEADLINE
