"""Device helpers: column-major torch CUDA tensors and the launching stream.

Matrices on the hot path are column-major (the layout qepy-pw's Davidson
allocates, qepy_pw/diagonalization.py:632-635): a tensor of shape (rows, cols)
with strides (1, ld), ld >= rows.  PyTorch supplies device memory, streams and
copies; every computation runs in libqeb200.so.
"""

from __future__ import annotations

import numpy as np
import torch

COMPLEX_OF = {torch.float64: torch.complex128, torch.float32: torch.complex64}
REAL_OF = {torch.complex128: torch.float64, torch.complex64: torch.float32}


_CUDA_SEEN = False


def require_cuda() -> torch.device:
    """The current CUDA device; raises when there is none (no CPU fallback)."""
    global _CUDA_SEEN
    if not _CUDA_SEEN:  # the device query is slow; a process keeps its GPUs
        if not torch.cuda.is_available():
            raise RuntimeError(
                "qe_b200 needs a CUDA device: the hot path has no CPU fallback"
            )
        _CUDA_SEEN = True
    return torch.device("cuda", torch.cuda.current_device())


def stream_handle(stream: torch.cuda.Stream | None = None) -> int:
    # current_stream() without a device asks torch for the available device
    # type, a CUDA device-count query (~0.5 ms) on every call; with the
    # current device index it does not
    if stream is None:
        stream = torch.cuda.current_stream(torch.cuda.current_device())
    return int(stream.cuda_stream)


def is_column_major(t: torch.Tensor) -> bool:
    if t.numel() == 0:
        return t.dim() in (1, 2)
    if t.dim() == 1:
        return t.stride(0) == 1
    return t.dim() == 2 and t.stride(0) == 1 and (t.shape[1] <= 1 or t.stride(1) >= t.shape[0])


def leading_dimension(t: torch.Tensor) -> int:
    """Column stride of a column-major matrix (any value >= rows for one column)."""
    if t.dim() == 1 or t.numel() == 0:
        return max(1, t.shape[0])
    if t.shape[1] <= 1:
        return max(1, t.shape[0], t.stride(1))
    return t.stride(1)


def aligned_ld(rows: int) -> int:
    """Leading dimension of the matrices this package allocates: rows rounded
    up to even, so every complex64 column starts on a 16-byte boundary (the
    TMA loads of the tensor-core GEMMs need that)."""
    return max(2, rows + (rows & 1))


def empty_f(rows: int, cols: int, dtype, device=None, ld: int | None = None) -> torch.Tensor:
    """Uninitialised column-major (rows, cols) tensor."""
    device = device if device is not None else require_cuda()
    ld = aligned_ld(rows) if ld is None else ld
    storage = torch.empty((cols, ld), dtype=dtype, device=device)
    return storage.T[:rows]


def zeros_f(rows: int, cols: int, dtype, device=None) -> torch.Tensor:
    device = device if device is not None else require_cuda()
    storage = torch.zeros((cols, aligned_ld(rows)), dtype=dtype, device=device)
    return storage.T[:rows]


def to_device_f(values, dtype, device=None) -> torch.Tensor:
    """Column-major device copy (no copy if already a matching tensor)."""
    device = device if device is not None else require_cuda()
    if isinstance(values, torch.Tensor):
        t = values
        if t.dim() == 2 and (t.device != device or t.dtype != dtype or not is_column_major(t)):
            out = empty_f(t.shape[0], t.shape[1], dtype, device)
            out.copy_(t)
            return out
        if t.device != device or t.dtype != dtype:
            t = t.to(device=device, dtype=dtype)
        if t.dim() == 1 and t.stride(0) != 1:
            t = t.contiguous()
        return t
    array = np.asarray(values)
    t = torch.from_numpy(np.asfortranarray(array) if array.ndim == 2 else np.ascontiguousarray(array))
    return to_device_f(t.to(dtype=dtype), dtype, device)


def as_numpy(t: torch.Tensor) -> np.ndarray:
    array = t.detach().cpu().numpy()
    return np.asfortranarray(array) if array.ndim == 2 else array
