"""Launch-shape selection by measurement.

The first time a kernel family meets a new problem class (a key built from
the sizes that change its best shape), each candidate shape is run and timed
with CUDA events on the current stream, and the fastest is kept for the rest
of the process; QEB_AUTOTUNE_CACHE=<file.json> keeps the table across runs.
Tuned choices:
  * the band batch of one local H|psi> launch (the stick buffer of a batch
    that fits the 126 MB L2 is re-read from L2 by pass B and pass C);
  * the K split of the split-TF32 GEMM (CTAs per output tile) and whether a
    mid-sized complex64 product runs on the tensor cores or the FP32 pipes.
Each timed run starts from a cold L2 (a 256 MiB write before it), the
condition of the large operands the kernels meet.  Inside CUDA-graph capture
nothing is timed: a known choice is used, else the
first candidate (the kernels' own default).  QEB_AUTOTUNE=0 turns timing off
(always the first candidate), e.g. for profiler captures.
"""

from __future__ import annotations

import json
import os
import threading

import torch


class Autotuner:
    def __init__(self, path: str | None = None, repeats: int = 3, margin: float = 0.05) -> None:
        self.path = path
        self.repeats = int(repeats)
        self.margin = float(margin)
        self.table: dict[str, object] = {}
        self.timings: dict[str, dict[str, float]] = {}
        self._flush = None
        self._lock = threading.Lock()
        self.enabled = os.environ.get("QEB_AUTOTUNE", "1") != "0"
        if path and os.path.exists(path):
            with open(path) as handle:
                self.table = json.load(handle)

    def _flush_buffer(self) -> torch.Tensor:
        """A device buffer larger than L2, written before every timed run."""
        device = torch.cuda.current_device()
        if self._flush is None or self._flush.device.index != device:
            self._flush = torch.empty(_FLUSH_BYTES // 4, dtype=torch.float32,
                                      device=torch.device("cuda", device))
        return self._flush

    def choose(self, key: str, candidates: list, run) -> object:
        """The fastest candidate for ``key``; ``run(candidate)`` launches the
        work on the current stream (it may run several times)."""
        if not candidates:
            raise ValueError("no candidates")
        known = self.table.get(key)
        if known in candidates:
            return known
        if len(candidates) == 1 or not self.enabled or not _cuda() or \
                torch.cuda.is_current_stream_capturing():
            return candidates[0]
        with self._lock:
            stream = torch.cuda.current_stream(torch.cuda.current_device())
            for c in candidates:  # warm-up: first-use allocations, caches
                run(c)
            samples = {c: [] for c in candidates}
            flush = self._flush_buffer()
            for _ in range(self.repeats):  # interleaved, median per candidate
                for c in candidates:
                    flush.fill_(1.0)  # time each candidate from a cold L2
                    start = torch.cuda.Event(enable_timing=True)
                    end = torch.cuda.Event(enable_timing=True)
                    start.record(stream)
                    run(c)
                    end.record(stream)
                    end.synchronize()
                    samples[c].append(start.elapsed_time(end))
            times = {c: sorted(v)[len(v) // 2] for c, v in samples.items()}
            # the first candidate is the kernel's own default: another one
            # must beat it by the margin to be chosen
            best = min(candidates, key=lambda c: times[c])
            if times[best] > (1.0 - self.margin) * times[candidates[0]]:
                best = candidates[0]
            self.table[key] = best
            self.timings[key] = {str(c): t for c, t in times.items()}
            if self.path:
                with open(self.path, "w") as handle:
                    json.dump(self.table, handle, indent=1, sort_keys=True)
        return best


_HAVE_CUDA = None


def _cuda() -> bool:
    global _HAVE_CUDA
    if _HAVE_CUDA is None:
        _HAVE_CUDA = torch.cuda.is_available()
    return _HAVE_CUDA


_FLUSH_BYTES = 256 << 20  # twice the B200's 126 MB L2


def bucket(n: int) -> int:
    """Smallest power of two >= n (problem-size class of a tuning key)."""
    return 1 << max(0, int(n - 1).bit_length())


TUNER = Autotuner(os.environ.get("QEB_AUTOTUNE_CACHE"))
