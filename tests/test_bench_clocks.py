"""bench.py's clock record (ClockSampler): the median SM clock, the highest maximum clock and the
throttle reasons seen while it ran, read from nvidia-smi's CSV samples.  A stand-in nvidia-smi on PATH
prints fixed samples, so the parsing and the reason flags are checked without a GPU."""
import os
import sys
import time

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402

IDLE = "1965, 1965, 850.00, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active"


def stand_in(tmp_path, lines):
    """A directory holding an executable `nvidia-smi` that prints `lines`, then waits to be stopped."""
    script = tmp_path / "nvidia-smi"
    script.write_text("#!/bin/sh\n" + "".join("echo '%s'\n" % l for l in lines) + "exec sleep 30\n")
    script.chmod(0o755)
    return str(tmp_path)


def record(tmp_path, monkeypatch, lines):
    monkeypatch.setenv("PATH", stand_in(tmp_path, lines) + os.pathsep + os.environ.get("PATH", ""))
    s = bench.ClockSampler(0)
    s.start()
    time.sleep(0.3)
    return s.stop()


def test_median_clock_and_power_cap(tmp_path, monkeypatch):
    rec = record(tmp_path, monkeypatch, [
        IDLE,
        "1950, 1965, 990.10, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "1965, 1965, 870.00, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
    ])
    assert rec["samples"] == 3
    assert rec["sm_mhz"] == 1965.0
    assert rec["sm_max_mhz"] == 1965.0
    assert rec["reasons"] == ["sw_power_cap"]


@pytest.mark.parametrize("column,name", [(4, "hw_slowdown"), (5, "hw_thermal_slowdown"), (6, "sw_thermal_slowdown")])
def test_each_slowdown_reason_is_reported(tmp_path, monkeypatch, column, name):
    fields = [f.strip() for f in IDLE.split(",")]
    fields[column] = "Active"
    rec = record(tmp_path, monkeypatch, [IDLE, ", ".join(fields), IDLE])
    assert rec["reasons"] == [name]


def test_clock_below_max_is_visible(tmp_path, monkeypatch):
    low = "1200, 1965, 400.00, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active"
    rec = record(tmp_path, monkeypatch, [low, low, IDLE])
    assert rec["sm_mhz"] == 1200.0 and rec["sm_max_mhz"] == 1965.0 and rec["reasons"] == []


def test_without_nvidia_smi(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", str(tmp_path))   # an empty directory: no nvidia-smi to run
    s = bench.ClockSampler(0)
    s.start()
    rec = s.stop()
    assert rec["sm_mhz"] is None and rec["reasons"] == ["nvidia-smi unavailable"]
