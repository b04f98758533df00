"""CPU tests of bench.py's clock record: a fake nvidia-smi on PATH stands in for
the GPU's. The sampler keeps the samples of the timed region, reports their
median SM clock, the largest max clock and every throttle reason seen active,
and degrades to an empty record when nvidia-smi is missing."""
import os
import stat
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _fake_smi(tmp_path, line):
    """An nvidia-smi that prints `line` every 20 ms until it is terminated."""
    d = tmp_path / "bin"
    d.mkdir()
    exe = d / "nvidia-smi"
    exe.write_text(f"#!/bin/sh\nwhile true; do echo '{line}'; sleep 0.02; done\n")
    exe.chmod(exe.stat().st_mode | stat.S_IXUSR | stat.S_IXGRP | stat.S_IXOTH)
    return str(d)


def test_power_cap_is_kept_and_reported(tmp_path, monkeypatch):
    d = _fake_smi(tmp_path, "0, 1400, 1965, 812.5, 0x0000000000000004, Not Active, Not Active, Not Active, Active")
    monkeypatch.setenv("PATH", d + os.pathsep + os.environ["PATH"])
    with bench.ClockSampler(0) as cs:
        time.sleep(0.3)
    s = cs.summary()
    assert s["samples"] >= 3, s
    assert s["sm_mhz"] == 1400.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]


def test_thermal_slowdown_is_reported(tmp_path, monkeypatch):
    d = _fake_smi(tmp_path, "0, 1100, 1965, 990.0, 0x0000000000000020, Not Active, Active, Not Active, Not Active")
    monkeypatch.setenv("PATH", d + os.pathsep + os.environ["PATH"])
    with bench.ClockSampler(0) as cs:
        time.sleep(0.2)
    s = cs.summary()
    assert s["samples"] >= 2 and s["reasons"] == ["hw_thermal_slowdown"], s


def test_samples_outside_the_region_are_dropped(tmp_path, monkeypatch):
    d = _fake_smi(tmp_path, "0, 1500, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, Not Active")
    monkeypatch.setenv("PATH", d + os.pathsep + os.environ["PATH"])
    with bench.ClockSampler(0) as cs:
        time.sleep(0.2)
    # lines stamped before the region began are not counted
    cs.lines.insert(0, (cs.t0 - 10.0, "0, 300, 1965, 100.0, 0x0, Active, Not Active, Not Active, Not Active"))
    s = cs.summary()
    assert s["sm_mhz"] == 1500.0 and s["reasons"] == [], s


def test_missing_nvidia_smi_gives_an_empty_record(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", str(tmp_path))
    with bench.ClockSampler(0) as cs:
        pass
    assert cs.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
