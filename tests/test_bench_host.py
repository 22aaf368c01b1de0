"""Host logic of bench.py (CPU).  The clock sampler: a stand-in
``nvidia-smi`` on PATH prints the query lines; a timed region shorter than
the 200 ms sampling period must still come back with samples, and slowdown
reasons active in any sample must be reported.  The FFT-convention rate
reported beside the dominant FFT pass's roofline."""

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


def test_plane_fft_rate_convention():
    """64^3 grid, 256 bands in 0.28 ms: 2 x 5 N log2 N + 2 N flops per
    (plane, band) with N = 64 x 64."""
    import json

    rate = bench.plane_fft_rate((64, 64, 64), 256, 0.28e-3)
    flops = (2 * 5 * 4096 * 12 + 2 * 4096) * 64 * 256
    assert abs(rate["achieved"] - flops / 0.28e-3 / 1e12) < 1e-9
    assert abs(rate["frac"] - rate["achieved"] / rate["peak"]) < 1e-12
    json.dumps(rate)


def test_sampler_passes_the_device_id(tmp_path, monkeypatch):
    """nvidia-smi gets the id it was given (a PCI bus id), not a torch index."""
    record = tmp_path / "args.txt"
    script = tmp_path / "nvidia-smi"
    script.write_text("#!/bin/bash\n"
                      f"echo \"$@\" > {record}\n"
                      "while true; do echo \"1965, 1965, Not Active, Not Active, Not Active, "
                      "Not Active\"; sleep 0.2; done\n")
    script.chmod(script.stat().st_mode | stat.S_IEXEC)
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ['PATH']}")
    with bench.ClockSampler("00000000:1B:00.0") as clocks:
        time.sleep(0.01)
    assert clocks.summary()["samples"] >= 1
    args = record.read_text().split()
    assert "--id=00000000:1B:00.0" in args


def test_smi_device_id_format(monkeypatch):
    """domain:bus:device.function in upper-case hex, as nvidia-smi prints it."""
    import types

    import torch

    props = types.SimpleNamespace(pci_domain_id=0, pci_bus_id=0x1B, pci_device_id=0)
    monkeypatch.setattr(torch.cuda, "get_device_properties", lambda index: props)
    assert bench.smi_device_id(3) == "00000000:1B:00.0"


def test_end_to_end_chunks_cover_the_bands():
    """The end-to-end leg's chunks: 1/8, 3/8, 3/8 and 1/8 of the bands, the
    last taking the remainder; every band in exactly one positive chunk."""
    assert bench.e2e_chunks(256) == [32, 96, 96, 32]
    for nbands in (1, 5, 7, 8, 40, 250, 257, 1000):
        sizes = bench.e2e_chunks(nbands)
        assert sum(sizes) == nbands and min(sizes) >= 1
