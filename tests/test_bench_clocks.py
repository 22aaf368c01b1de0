"""The bench's clock sampler (host logic, CPU): a stand-in ``nvidia-smi`` on
PATH prints the query lines; a timed region shorter than the 200 ms
sampling period must still come back with samples, and slowdown reasons
that are active in any sample must be reported."""

from __future__ import annotations

import os
import stat
import sys
import time
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

import bench  # noqa: E402


def _fake_smi(folder: Path, line: str) -> None:
    script = folder / "nvidia-smi"
    script.write_text("#!/bin/bash\nsleep 0.3\n"
                      f"while true; do echo \"{line}\"; sleep 0.2; done\n")
    script.chmod(script.stat().st_mode | stat.S_IEXEC)


def test_short_region_has_samples(tmp_path, monkeypatch):
    _fake_smi(tmp_path, "1965, 1965, Not Active, Not Active, Not Active, Not Active")
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ['PATH']}")
    with bench.ClockSampler(0) as clocks:
        time.sleep(0.01)
    summary = clocks.summary()
    assert summary["samples"] >= 1
    assert summary["sm_mhz"] == 1965.0 and summary["sm_max_mhz"] == 1965.0
    assert summary["reasons"] == []


def test_active_reasons_are_reported(tmp_path, monkeypatch):
    _fake_smi(tmp_path, "1500, 1965, Not Active, Not Active, Not Active, Active")
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ['PATH']}")
    with bench.ClockSampler(0) as clocks:
        time.sleep(0.5)
    summary = clocks.summary()
    assert summary["samples"] >= 2
    assert summary["sm_mhz"] == 1500.0
    assert summary["reasons"] == ["sw_power_cap"]


def test_missing_tool_gives_no_samples(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", str(tmp_path))
    with bench.ClockSampler(0) as clocks:
        pass
    assert clocks.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
