"""Autotuner bookkeeping on the CPU: cached choices, the JSON cache file and
the disabled mode (timing itself needs a GPU and runs inside the GPU tests
that call the tuned kernels)."""

from __future__ import annotations

import json

from qe_python_b200.autotune import Autotuner, bucket


def test_bucket_is_next_power_of_two():
    assert [bucket(n) for n in (1, 2, 3, 4, 5, 255, 256, 257)] == [1, 2, 4, 4, 8, 256, 256, 512]


def test_cached_choice_wins_and_file_round_trip(tmp_path, monkeypatch):
    path = tmp_path / "tune.json"
    path.write_text(json.dumps({"k1": 64}))
    tuner = Autotuner(str(path))
    calls = []
    assert tuner.choose("k1", [256, 128, 64], lambda c: calls.append(c)) == 64
    assert calls == []  # a cached key runs nothing
    # an unknown key without a GPU (or with timing disabled) takes the first candidate
    monkeypatch.setattr(tuner, "enabled", False)
    assert tuner.choose("k2", [32, 16], lambda c: calls.append(c)) == 32
    assert calls == []


def test_stale_cached_choice_is_ignored(tmp_path):
    path = tmp_path / "tune.json"
    path.write_text(json.dumps({"k": 999}))
    tuner = Autotuner(str(path))
    tuner.enabled = False
    assert tuner.choose("k", [4, 2], lambda c: None) == 4
