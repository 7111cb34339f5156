"""Host-side logic of bench.py that needs no GPU: the clock sampler's summary
(only samples taken inside the timed span count, throttle reasons are
collected) and the command line."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _line(sm, reasons=("Not Active",) * 4, smax=1965):
    return ", ".join(["0", str(sm), str(smax), "", "0x0"] + list(reasons))


def test_clock_summary_keeps_samples_inside_span():
    c = bench.ClockSampler(0)
    c.lines = [_line(345), _line(1965), _line(1965), _line(1950)]
    c.times = [1.0, 2.0, 2.1, 2.2]
    c.t_start = 1.5  # the idle sample before the span is dropped
    s = c.summary()
    assert s["samples"] == 3 and s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0 and s["reasons"] == []


def test_clock_summary_falls_back_to_last_sample():
    c = bench.ClockSampler(0)
    c.lines = [_line(1900), _line(1965)]
    c.times = [1.0, 1.1]
    c.t_start = 5.0  # a span shorter than the sampling period
    s = c.summary()
    assert s["samples"] == 1 and s["sm_mhz"] == 1965.0


def test_clock_summary_reasons():
    c = bench.ClockSampler(0)
    c.lines = [_line(1700, ("Not Active", "Not Active", "Not Active", "Active")),
               _line(1500, ("Active", "Not Active", "Not Active", "Not Active"))]
    c.times = [2.0, 2.1]
    c.t_start = 1.0
    s = c.summary()
    assert s["reasons"] == ["hw_slowdown", "sw_power_cap"] and s["sm_mhz"] == 1600.0


def test_clock_summary_nvidia_smi_lines():
    """Lines from the nvidia-smi fallback carry no timestamps: all count."""
    c = bench.ClockSampler(0)
    c.lines = ["0, 1965, 1965, 700.5, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
               "garbage", "0, 1955, 1965, 702.1, 0x0000000000000004, Not Active, Not Active, Not Active, Active"]
    s = c.summary()
    assert s["samples"] == 2 and s["sm_mhz"] == 1960.0 and s["reasons"] == ["sw_power_cap"]


def test_no_samples():
    s = bench.ClockSampler(0).summary()
    assert s == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}


def test_args(monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse_args()
    assert (a.gpus, a.steps, a.warmup, a.impl, a.workload, a.tune, a.tuning) == (1, 10, 3, "ours", "heightfield", 1, "")
    assert bench.CPU_STRIDE[a.workload] > 1  # the CPU legs build a bounded sample of the 5M-triangle mesh
    monkeypatch.setattr(sys, "argv", ["bench.py", "--workload", "torus_slivers", "--tuning", "128,256,0,64,0"])
    a = bench.parse_args()
    assert tuple(int(x) for x in a.tuning.split(",")) == (128, 256, 0, 64, 0)
    assert a.warmup >= 3
