"""Lowest eigenpairs of the Davidson reduced problem by cuSOLVER's zhegvdx.

The reduced problem H x = e S x (complex128, n up to a few thousand) is
solved on the device in FP64.  Davidson needs only its lowest ``roots``
pairs (the reference asks LAPACK zhegvd for all of them and keeps the lowest:
qepy_pw/diagonalization.py:83-110, _native_fft.pyx:667-691).  zhegvdx with an
index range does the same Cholesky reduction and tridiagonalisation but
computes and back-transforms only those eigenvectors.

cuSOLVER is a library called like cuBLAS: it is the one torch links (the
``nvidia.cusolver`` package of its wheel).  Matrices are passed as torch
tensors; a row-major Hermitian matrix read column-major is its complex
conjugate, whose eigenvalues are the same and whose eigenvectors are the
conjugates, which this module undoes.
"""

from __future__ import annotations

import ctypes
import os
import threading

import torch

_P, _I, _D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
_EIG_TYPE_1, _MODE_VECTOR, _RANGE_I, _FILL_LOWER = 1, 1, 1002, 0

_lock = threading.Lock()
_state: dict = {}


def _library():
    lib = _state.get("lib")
    if lib is None:
        import nvidia.cusolver

        path = os.path.join(list(nvidia.cusolver.__path__)[0], "lib", "libcusolver.so.11")
        lib = ctypes.CDLL(path)
        lib.cusolverDnCreate.argtypes = [ctypes.POINTER(_P)]
        lib.cusolverDnSetStream.argtypes = [_P, _P]
        lib.cusolverDnZhegvdx_bufferSize.argtypes = [
            _P, _I, _I, _I, _I, _I, _P, _I, _P, _I, _D, _D, _I, _I, ctypes.POINTER(_I), _P,
            ctypes.POINTER(_I)]
        lib.cusolverDnZhegvdx.argtypes = [
            _P, _I, _I, _I, _I, _I, _P, _I, _P, _I, _D, _D, _I, _I, ctypes.POINTER(_I), _P, _P,
            _I, _P]
        _state["lib"] = lib
    return lib


def _handle(device: torch.device):
    """One cuSOLVER handle per device (created with that device current)."""
    key = ("handle", device.index)
    handle = _state.get(key)
    if handle is None:
        handle = _P()
        with torch.cuda.device(device):
            status = _library().cusolverDnCreate(ctypes.byref(handle))
        if status != 0:
            raise RuntimeError(f"cusolverDnCreate failed ({status})")
        _state[key] = handle
    return handle


def lowest_pairs(h: torch.Tensor, s: torch.Tensor, roots: int):
    """(values, vectors) of the ``roots`` lowest pairs of h x = e s x, or
    None when s is not numerically positive definite (the caller then falls
    back to a canonical orthogonalisation).  h, s: Hermitian complex128 CUDA
    tensors (n, n); vectors is (n, roots), s-orthonormal."""
    n = h.shape[0]
    device = h.device
    a = h.to(torch.complex128).contiguous().clone()
    b = s.to(torch.complex128).contiguous().clone()
    values = torch.empty(n, dtype=torch.float64, device=device)
    info = torch.zeros(1, dtype=torch.int32, device=device)
    lib = _library()
    with _lock:
        handle = _handle(device)
        stream = torch.cuda.current_stream(device)
        lib.cusolverDnSetStream(handle, _P(stream.cuda_stream))
        lwork, found = _I(), _I()
        status = lib.cusolverDnZhegvdx_bufferSize(
            handle, _EIG_TYPE_1, _MODE_VECTOR, _RANGE_I, _FILL_LOWER, n, _P(a.data_ptr()), n,
            _P(b.data_ptr()), n, 0.0, 0.0, 1, roots, ctypes.byref(found), _P(values.data_ptr()),
            ctypes.byref(lwork))
        if status != 0:
            raise RuntimeError(f"cusolverDnZhegvdx_bufferSize failed ({status})")
        work = torch.empty(max(1, lwork.value), dtype=torch.complex128, device=device)
        status = lib.cusolverDnZhegvdx(
            handle, _EIG_TYPE_1, _MODE_VECTOR, _RANGE_I, _FILL_LOWER, n, _P(a.data_ptr()), n,
            _P(b.data_ptr()), n, 0.0, 0.0, 1, roots, ctypes.byref(found), _P(values.data_ptr()),
            _P(work.data_ptr()), lwork.value, _P(info.data_ptr()))
        if status != 0:
            raise RuntimeError(f"cusolverDnZhegvdx failed ({status})")
    if int(info) != 0:
        return None
    # column-major eigenvectors of the conjugate problem, first ``roots`` columns
    vectors = a.T[:, :roots].conj()
    return values[:roots], vectors
