"""The Davidson reduced eigensolve without a host synchronisation.

The reduced problem H c = e S c (complex128, a few hundred to about a
thousand columns) is solved in FP64 on the device as in LAPACK zhegv: the
Cholesky factor S = L L^H, the standard problem L^-1 H L^-H, its Hermitian
eigensolve and the back-substitution (the reference solves the same problem
with LAPACK: qepy_pw/diagonalization.py:83-110, _native_fft.pyx:667-691).
``torch.linalg.eigh`` reads its error code back to the host, so the host
waits for every eigensolve; here the Hermitian eigensolve is cuSOLVER's
zheevd called directly (cuSOLVER is a library called like cuBLAS: the one
torch links, from its ``nvidia.cusolver`` package) with the error codes left
on the device, and the whole solve runs on a stream of the caller's choice.
Several k points' solves, each a chain of small latency-bound kernels, then
run side by side on the GPU; the host reads the error codes when it reads
the eigenvalues.

``ReducedSolve.launch`` enqueues a solve on a stream and returns at once;
``ReducedSolve.result`` makes the current stream wait for it and returns the
lowest ``roots`` pairs, or falls back to the canonical orthogonalisation of
the overlap when S was not numerically positive definite.
"""

from __future__ import annotations

import ctypes
import os
import threading

import torch

_P, _I = ctypes.c_void_p, ctypes.c_int
_MODE_VECTOR, _FILL_LOWER = 1, 0

_lock = threading.Lock()
_state: dict = {}


def _library():
    lib = _state.get("lib")
    if lib is None:
        import nvidia.cusolver

        path = os.path.join(list(nvidia.cusolver.__path__)[0], "lib", "libcusolver.so.11")
        lib = ctypes.CDLL(path)
        lib.cusolverDnCreate.argtypes = [ctypes.POINTER(_P)]
        lib.cusolverDnCreate.restype = _I
        lib.cusolverDnSetStream.argtypes = [_P, _P]
        lib.cusolverDnSetStream.restype = _I
        lib.cusolverDnZheevd_bufferSize.argtypes = [_P, _I, _I, _I, _P, _I, _P,
                                                    ctypes.POINTER(_I)]
        lib.cusolverDnZheevd_bufferSize.restype = _I
        lib.cusolverDnZheevd.argtypes = [_P, _I, _I, _I, _P, _I, _P, _P, _I, _P]
        lib.cusolverDnZheevd.restype = _I
        _state["lib"] = lib
    return lib


def _handle(device: torch.device):
    """One cuSOLVER handle per device, created with that device's context
    current (torch's primary context)."""
    key = ("handle", device.index)
    handle = _state.get(key)
    if handle is None:
        handle = _P()
        with torch.cuda.device(device):
            torch.cuda.current_stream(device)  # the context exists from here on
            status = _library().cusolverDnCreate(ctypes.byref(handle))
        if status != 0:
            raise RuntimeError(f"cusolverDnCreate failed ({status})")
        _state[key] = handle
    return handle


def zheevd_async(matrix: torch.Tensor, stream: torch.cuda.Stream):
    """All eigenpairs of a Hermitian complex128 CUDA matrix, enqueued on
    ``stream`` without a host synchronisation.  Returns (values, vectors,
    info): ascending values, column-major vectors (as a tensor whose columns
    are the eigenvectors) and cuSOLVER's device error code.  ``matrix`` is
    read through its lower triangle in row-major order, i.e. as the
    conjugate matrix column-major; its eigenvectors are conjugated back."""
    n = matrix.shape[0]
    device = matrix.device
    lib = _library()
    with torch.cuda.stream(stream):
        work_matrix = matrix.contiguous().clone()
        values = torch.empty(n, dtype=torch.float64, device=device)
        info = torch.zeros(1, dtype=torch.int32, device=device)
        with _lock:
            handle = _handle(device)
            status = lib.cusolverDnSetStream(handle, _P(stream.cuda_stream))
            if status != 0:
                raise RuntimeError(f"cusolverDnSetStream failed ({status})")
            lwork = _I()
            status = lib.cusolverDnZheevd_bufferSize(
                handle, _MODE_VECTOR, _FILL_LOWER, n, _P(work_matrix.data_ptr()), n,
                _P(values.data_ptr()), ctypes.byref(lwork))
            if status != 0:
                raise RuntimeError(f"cusolverDnZheevd_bufferSize failed ({status})")
            work = torch.empty(max(1, lwork.value), dtype=torch.complex128, device=device)
            status = lib.cusolverDnZheevd(
                handle, _MODE_VECTOR, _FILL_LOWER, n, _P(work_matrix.data_ptr()), n,
                _P(values.data_ptr()), _P(work.data_ptr()), lwork.value, _P(info.data_ptr()))
            if status != 0:
                raise RuntimeError(f"cusolverDnZheevd failed ({status})")
        # row-major storage read column-major: the rows of work_matrix are the
        # conjugated eigenvectors
        vectors = work_matrix.T.conj()
    return values, vectors, info


class ReducedSolve:
    """One asynchronous solve of H c = e S c for the lowest ``roots`` pairs."""

    def __init__(self, stream: torch.cuda.Stream) -> None:
        self.stream = stream
        self._pending = None

    def launch(self, h: torch.Tensor, s: torch.Tensor, roots: int) -> None:
        """Enqueue the solve of the Hermitian pair (h, s) on the stream after
        the work the current stream has enqueued so far."""
        from .diagonalization import _hermitize

        current = torch.cuda.current_stream(h.device)
        self.stream.wait_stream(current)
        with torch.cuda.stream(self.stream):
            h = h.to(torch.complex128)
            s = s.to(torch.complex128)
            lower, chol_info = torch.linalg.cholesky_ex(s)
            left = torch.linalg.solve_triangular(lower, h, upper=False)
            reduced = _hermitize(torch.linalg.solve_triangular(lower, left.conj().T,
                                                               upper=False).conj().T)
            values, vectors, eig_info = zheevd_async(reduced, self.stream)
            vectors = torch.linalg.solve_triangular(lower.conj().T, vectors[:, :roots],
                                                    upper=True)
            values = values[:roots]
            done = torch.cuda.Event()
            done.record(self.stream)
        self._pending = (h, s, roots, values, vectors, chol_info, eig_info, done, current)

    def result(self):
        """(values, vectors) of the launched solve, on the current stream."""
        from .diagonalization import _canonical_generalized_eigh

        h, s, roots, values, vectors, chol_info, eig_info, done, current = self._pending
        self._pending = None
        current.wait_event(done)
        for tensor in (h, s, values, vectors, chol_info, eig_info):
            tensor.record_stream(current)
        chol_code, eig_code = (int(v) for v in
                               torch.cat([chol_info.reshape(1), eig_info.reshape(1)]).tolist())
        if chol_code != 0:
            # S numerically indefinite (a subspace built from FP32 vectors):
            # solve in the well-conditioned part of its range instead
            return _canonical_generalized_eigh(h, s, roots)
        if eig_code != 0:
            raise RuntimeError(f"cusolverDnZheevd reported info {eig_code}")
        return values, vectors
