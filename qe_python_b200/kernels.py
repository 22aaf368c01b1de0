"""Torch-tensor front end of the C ABI (GEMMs and Davidson column kernels).

Each function validates shapes, resolves leading dimensions and launches on
the current torch stream.  Matrices are column-major torch CUDA tensors
(strides (1, ld)); scalars in FP64.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np
import torch

from . import _lib
from .autotune import TUNER, bucket
from .device import empty_f, is_column_major, leading_dimension, stream_handle

OP_N = 0
OP_C = 1

_PREC = {torch.complex128: _lib.QEB_F64, torch.complex64: _lib.QEB_F32}


class _Scratch:
    """Grow-only device scratch for split-K partial tiles, one buffer per
    (device, stream): products issued on different streams never share it.
    A buffer that grows keeps its predecessors alive (at least doubling, so
    few of them): a CUDA graph captured earlier on the stream holds the old
    address, and freeing it would hand that memory to other tensors."""

    def __init__(self) -> None:
        self._buffers: dict[tuple, torch.Tensor] = {}
        self._retired: list[torch.Tensor] = []

    def get(self, nbytes: int, device: torch.device) -> torch.Tensor:
        key = (device, torch.cuda.current_stream(device).cuda_stream)
        current = self._buffers.get(key)
        if current is None or current.numel() < nbytes:
            size = max(int(nbytes), 256)
            if current is not None:
                self._retired.append(current)
                size = max(size, 2 * current.numel())
            current = torch.empty(size, dtype=torch.uint8, device=device)
            self._buffers[key] = current
        return current


_SCRATCH = _Scratch()


def _precision(t: torch.Tensor) -> int:
    try:
        return _PREC[t.dtype]
    except KeyError as exc:
        raise TypeError(f"complex128 or complex64 tensor required, got {t.dtype}") from exc


def _check_matrix(name: str, t: torch.Tensor) -> None:
    if t.dim() != 2 or not t.is_cuda or not is_column_major(t):
        raise ValueError(f"{name} must be a column-major 2-D CUDA tensor")


# complex64 products with at least this many complex multiply-adds run as
# split-TF32 on the tensor cores (cgemm_tf32x3); smaller ones on the FP32 pipes
TENSOR_MIN_MACS = 1 << 21


TUNE_MIN_FLOP = 2.0e9  # split-TF32 products below this are not worth timing (~20 us)
# Timing the K split on first use (QEB_TUNE_SPLITS=1).  Off by default: on every
# shape of the benchmark cells the library's two-wave default was the tuned
# choice (within 5 %), and the first-use timing cost about a second per SCF.
TUNE_SPLITS = os.environ.get("QEB_TUNE_SPLITS") == "1"
SKINNY_MAX = 16  # narrow output side at or below which qeb_zgemm/qeb_cgemm stream the wide operand


def is_skinny(op_a: int, m: int, n: int) -> bool:
    """Whether the FMA library routes op(a) b (output m x n) to its skinny
    kernels: n <= 16, or m <= 16 for op_a = OP_C.  Those stream the large
    operand once at HBM speed, which the tiled tensor-core kernel cannot do
    for so narrow an output."""
    return n <= SKINNY_MAX or (op_a == OP_C and m <= SKINNY_MAX)


def gemm(op_a: int, a: torch.Tensor, b: torch.Tensor, c: torch.Tensor | None = None,
         alpha: complex = 1.0, beta: complex = 0.0, tensor: bool | None = None) -> torch.Tensor:
    """c = alpha op(a) b + beta c with op(a) = a (OP_N) or a^H (OP_C).

    complex128: FP64 (qeb_zgemm).  complex64: split-TF32 tensor-core products
    (qeb_cgemm_tf32x3) when ``tensor`` is True, or when it is None and the
    product is large and not skinny; else FP32 FMA (qeb_cgemm).
    """
    if tensor is not False and a.dtype == torch.complex64 and b.dtype == torch.complex64:
        m = a.shape[1] if op_a == OP_C else a.shape[0]
        k = a.shape[0] if op_a == OP_C else a.shape[1]
        n = b.shape[1] if b.dim() == 2 else 1
        if tensor or (m * n * k >= TENSOR_MIN_MACS and not is_skinny(op_a, m, n)):
            out = cgemm_tf32x3(op_a, a, b, c, alpha, beta)
            if out is not None:
                return out
    _check_matrix("a", a)
    _check_matrix("b", b)
    if a.dtype != b.dtype:
        raise TypeError("operands must share a dtype")
    prec = _precision(a)
    if op_a == OP_N:
        m, k = a.shape
    elif op_a == OP_C:
        k, m = a.shape
    else:
        raise ValueError("op_a must be OP_N or OP_C")
    if b.shape[0] != k:
        raise ValueError(f"inner dimensions disagree: op(a) is {m}x{k}, b is {tuple(b.shape)}")
    n = b.shape[1]
    if c is None:
        c = empty_f(m, n, a.dtype, a.device)
        beta = 0.0
    else:
        _check_matrix("c", c)
        if tuple(c.shape) != (m, n) or c.dtype != a.dtype:
            raise ValueError("c has the wrong shape or dtype")
    if m == 0 or n == 0:
        return c
    lib = _lib.load()
    al = (ctypes.c_double * 2)(complex(alpha).real, complex(alpha).imag)
    be = (ctypes.c_double * 2)(complex(beta).real, complex(beta).imag)
    need = int(lib.qeb_zgemm_scratch_bytes(op_a, m, n, k, prec))
    scratch = _SCRATCH.get(need, a.device) if need > 0 else None
    fn = lib.qeb_zgemm if prec == _lib.QEB_F64 else lib.qeb_cgemm
    status = fn(op_a, m, n, k, al, a.data_ptr(), leading_dimension(a), b.data_ptr(),
                leading_dimension(b), be, c.data_ptr(), leading_dimension(c),
                0 if scratch is None else scratch.data_ptr(), need, stream_handle())
    _lib.check("qeb_zgemm" if prec == _lib.QEB_F64 else "qeb_cgemm", status)
    return c


def diagonal_blocks(coupling: np.ndarray) -> list[tuple[int, int]]:
    """Smallest contiguous diagonal blocks (start, size) covering every
    nonzero entry of a square matrix.

    One scan: index i reaches the last row or column that shares a nonzero
    with row or column i; a block closes at the first i that no index since
    its start reaches past."""
    nz = np.asarray(coupling) != 0
    n = nz.shape[0]
    if n == 0:
        return []
    index = np.arange(n)
    last_col = np.where(nz.any(axis=1), n - 1 - np.argmax(nz[:, ::-1], axis=1), index)
    last_row = np.where(nz.any(axis=0), n - 1 - np.argmax(nz[::-1, :], axis=0), index)
    reach = (np.maximum(np.maximum(last_col, last_row), index) + 1).tolist()
    blocks, start, end = [], 0, 0
    for i in range(n):
        end = max(end, reach[i])
        if end == i + 1:
            blocks.append((start, end - start))
            start = end
    return blocks


class BlockCoupling:
    """coupled = D becp with D block diagonal (qeb_block_coupling)."""

    def __init__(self, coupling: np.ndarray, dtype: torch.dtype, device) -> None:
        coupling = np.asarray(coupling)
        self.channels = coupling.shape[0]
        self.dtype = dtype
        blocks = diagonal_blocks(coupling)
        starts = np.array([s for s, _ in blocks], dtype=np.int32)
        sizes = np.array([n for _, n in blocks], dtype=np.int32)
        offsets = np.concatenate(([0], np.cumsum(sizes.astype(np.int64) ** 2)[:-1])).astype(np.int64)
        values = np.concatenate([coupling[s:s + n, s:s + n].reshape(-1) for s, n in blocks]) \
            if blocks else np.zeros(1)
        row_block = np.repeat(np.arange(len(blocks), dtype=np.int32), sizes)
        self.nblocks = len(blocks)
        self.max_block = int(sizes.max(initial=0))
        self._row_block = torch.from_numpy(row_block).to(device)
        self._start = torch.from_numpy(starts).to(device)
        self._size = torch.from_numpy(sizes).to(device)
        self._offset = torch.from_numpy(offsets).to(device)
        self._values = torch.from_numpy(values.astype(np.complex128)).to(device).to(dtype)

    def apply(self, becp: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        _check_matrix("becp", becp)
        if becp.shape[0] != self.channels or becp.dtype != self.dtype:
            raise ValueError("becp does not match the coupling")
        if out is None:
            out = empty_f(becp.shape[0], becp.shape[1], becp.dtype, becp.device)
        _lib.check("qeb_block_coupling", _lib.load().qeb_block_coupling(
            _precision(becp), self.channels, becp.shape[1], self.nblocks,
            self._row_block.data_ptr(), self._start.data_ptr(), self._size.data_ptr(),
            self._offset.data_ptr(), self._values.data_ptr(), becp.data_ptr(),
            leading_dimension(becp), out.data_ptr(), leading_dimension(out), stream_handle()))
        return out


PACK_RAW, PACK_SWAPNEG, PACK_NEGIM, PACK_SWAP = 0, 1, 2, 3


def tf32_width(k: int) -> int:
    """Packed row length: 2K reals rounded up to the 32-wide K tile."""
    return (2 * int(k) + 31) // 32 * 32


class PackedOperand:
    """K-major hi/lo FP32 planes of a complex operand (qeb_tf32_pack)."""

    def __init__(self, rows: int, k: int, device) -> None:
        self.rows, self.k, self.kp = int(rows), int(k), tf32_width(k)
        self.hi = torch.empty((max(self.rows, 1), self.kp), dtype=torch.float32, device=device)
        self.lo = torch.empty_like(self.hi)


def tf32_pack(src: torch.Tensor, layout: int, transposed: bool = False,
              out: PackedOperand | None = None) -> PackedOperand:
    """Pack columns (or, transposed, rows) of a complex matrix for qeb_tf32_gemm."""
    _check_matrix("src", src)
    rows, k = (src.shape[0], src.shape[1]) if transposed else (src.shape[1], src.shape[0])
    if out is None or out.rows != rows or out.k != k:
        out = PackedOperand(rows, k, src.device)
    _lib.check("qeb_tf32_pack", _lib.load().qeb_tf32_pack(
        _precision(src), layout, int(transposed), rows, k, src.data_ptr(), leading_dimension(src),
        out.hi.data_ptr(), out.lo.data_ptr(), out.kp, stream_handle()))
    return out


def tf32_gemm(a: PackedOperand, b0: PackedOperand, b1: PackedOperand, c: torch.Tensor,
              alpha: complex = 1.0, beta: complex = 0.0) -> torch.Tensor:
    """c = alpha (A B0^T + i A B1^T) + beta c on tcgen05 (split TF32)."""
    _check_matrix("c", c)
    if c.dtype != torch.complex64:
        raise TypeError("the split-TF32 GEMM writes complex64")
    if a.kp != b0.kp or b0.kp != b1.kp or b0.rows != b1.rows:
        raise ValueError("packed operands disagree")
    m, n = a.rows, b0.rows
    if tuple(c.shape) != (m, n):
        raise ValueError("c has the wrong shape")
    if m == 0 or n == 0:
        return c
    lib = _lib.load()
    al = (ctypes.c_double * 2)(complex(alpha).real, complex(alpha).imag)
    be = (ctypes.c_double * 2)(complex(beta).real, complex(beta).imag)
    need = int(lib.qeb_tf32_gemm_scratch_bytes(m, n, a.kp))
    scratch = _SCRATCH.get(need, c.device) if need > 0 else None
    _lib.check("qeb_tf32_gemm", lib.qeb_tf32_gemm(
        m, n, a.kp, a.hi.data_ptr(), a.lo.data_ptr(), a.kp, b0.hi.data_ptr(), b0.lo.data_ptr(),
        b1.hi.data_ptr(), b1.lo.data_ptr(), b0.kp, al, be, c.data_ptr(), leading_dimension(c),
        0 if scratch is None else scratch.data_ptr(), need, stream_handle()))
    return c


def tf32_error() -> int:
    """Non-zero if a bounded wait inside the tcgen05 GEMM timed out (synchronises)."""
    value = ctypes.c_int(0)
    _lib.check("qeb_tf32_gemm_error", _lib.load().qeb_tf32_gemm_error(ctypes.byref(value)))
    return int(value.value)


def cgemm_tf32x3(op_a: int, a: torch.Tensor, b: torch.Tensor, c: torch.Tensor | None = None,
                 alpha: complex = 1.0, beta: complex = 0.0,
                 splits: int | None = None) -> torch.Tensor | None:
    """Split-TF32 c = alpha op(a) b + beta c reading complex64 a and b directly
    (qeb_cgemm_tf32x3_ex).  Returns None, touching nothing, when a or b lacks
    16-byte aligned columns (odd leading dimension); callers then use the
    packed path.  ``splits``: CTAs per output tile along K; None takes the
    library's choice or, with QEB_TUNE_SPLITS=1, lets the autotuner pick among
    it, half, twice and four times it (each K slice at least four 32-wide K
    tiles deep)."""
    _check_matrix("a", a)
    _check_matrix("b", b)
    if a.dtype != torch.complex64 or b.dtype != torch.complex64:
        raise TypeError("cgemm_tf32x3 takes complex64 operands")
    if op_a == OP_C:
        k, m = a.shape
    elif op_a == OP_N:
        m, k = a.shape
    else:
        raise ValueError("op_a must be OP_N or OP_C")
    if b.shape[0] != k:
        raise ValueError(f"inner dimensions disagree: op(a) is {m}x{k}, b is {tuple(b.shape)}")
    n = b.shape[1]
    lda, ldb = leading_dimension(a), leading_dimension(b)
    if (a.data_ptr() % 16 or b.data_ptr() % 16 or lda % 2 or ldb % 2) and m * n * k > 0:
        return None
    if c is None:
        c = empty_f(m, n, torch.complex64, b.device)
        beta = 0.0
    else:
        _check_matrix("c", c)
        if tuple(c.shape) != (m, n) or c.dtype != torch.complex64:
            raise ValueError("c has the wrong shape or dtype")
    if m == 0 or n == 0:
        return c
    if k == 0:  # empty contraction: c = beta c
        return c.zero_() if complex(beta) == 0 else c.mul_(beta)
    lib = _lib.load()
    if splits is None and not TUNE_SPLITS:
        splits = 0  # the library's choice: two whole waves, or a split tail wave
    if splits is None:
        default = int(lib.qeb_cgemm_tf32x3_default_splits(op_a, m, n, k))
        kblocks = (2 * k + 31) // 32
        tiles = ((m + 127) // 128) * ((n + 127) // 128)
        if default == 1 and not 148 < tiles < 296:
            # enough output tiles for full waves: the K split stays off
            candidates = [1]
        elif 8 * m * n * k < TUNE_MIN_FLOP:
            # a few microseconds of work: timing candidates costs more than
            # a better split could save
            candidates = [default]
        else:
            candidates = sorted({default, max(1, default // 2),
                                 min(2 * default, max(1, kblocks // 4)),
                                 min(4 * default, max(1, kblocks // 4))})
            candidates.remove(default)
            candidates.insert(0, default)
        key = f"cgemm_tf32x3/{op_a}/{bucket(m)}/{bucket(n)}/{bucket(k)}"
        probe = []

        def run(s_):  # into a scratch output: c may be accumulated into (beta != 0)
            if not probe:
                probe.append(empty_f(m, n, torch.complex64, c.device))
            _cgemm_tf32x3_launch(lib, op_a, m, n, k, 1.0, a, lda, b, ldb, 0.0, probe[0], s_)

        splits = TUNER.choose(key, candidates, run)
    _cgemm_tf32x3_launch(lib, op_a, m, n, k, alpha, a, lda, b, ldb, beta, c, splits)
    return c


def _cgemm_tf32x3_launch(lib, op_a, m, n, k, alpha, a, lda, b, ldb, beta, c, splits):
    al = (ctypes.c_double * 2)(complex(alpha).real, complex(alpha).imag)
    be = (ctypes.c_double * 2)(complex(beta).real, complex(beta).imag)
    if splits and splits > 1:
        need = int(splits) * m * n * 8
    else:
        # the default split, or for an unsplit product the K split of its
        # partial last wave of output tiles
        need = int(lib.qeb_cgemm_tf32x3_scratch_bytes(op_a, m, n, k))
    scratch = _SCRATCH.get(need, c.device) if need > 0 else None
    _lib.check("qeb_cgemm_tf32x3_ex", lib.qeb_cgemm_tf32x3_ex(
        op_a, m, n, k, al, a.data_ptr(), lda, b.data_ptr(), ldb, be, c.data_ptr(),
        leading_dimension(c), 0 if scratch is None else scratch.data_ptr(), need,
        int(splits or 0), stream_handle()))


def gemm_tf32(op_a: int, a: torch.Tensor, b: torch.Tensor, c: torch.Tensor | None = None,
              alpha: complex = 1.0, beta: complex = 0.0,
              a_packed: PackedOperand | None = None) -> torch.Tensor:
    """Complex c = alpha op(a) b + beta c with split-TF32 tensor-core products.

    op_a = OP_C: a is K x M (op(a) = a^H); OP_N: a is M x K.  complex64
    operands with aligned columns go straight to cgemm_tf32x3; otherwise
    both are packed (``a_packed`` reuses an operand packed earlier with the
    matching layout) for qeb_tf32_gemm.
    """
    if a.dtype == torch.complex64 and b.dtype == torch.complex64:
        out = cgemm_tf32x3(op_a, a, b, c, alpha, beta)
        if out is not None:
            return out
    _check_matrix("b", b)
    if op_a == OP_C:
        a_op = a_packed if a_packed is not None else tf32_pack(a, PACK_RAW)
        b0, b1 = tf32_pack(b, PACK_RAW), tf32_pack(b, PACK_SWAPNEG)
    elif op_a == OP_N:
        a_op = a_packed if a_packed is not None else tf32_pack(a, PACK_RAW, transposed=True)
        b0, b1 = tf32_pack(b, PACK_NEGIM), tf32_pack(b, PACK_SWAP)
    else:
        raise ValueError("op_a must be OP_N or OP_C")
    if a_op.k != b.shape[0]:
        raise ValueError("inner dimensions disagree")
    if c is None:
        c = empty_f(a_op.rows, b.shape[1], torch.complex64, b.device)
        beta = 0.0
        if a_op.k == 0:
            return c.zero_()
    elif a_op.k == 0:  # empty contraction: c = beta c
        return c.mul_(beta)
    return tf32_gemm(a_op, b0, b1, c, alpha, beta)


def column_squared_norms(v: torch.Tensor) -> torch.Tensor:
    _check_matrix("v", v)
    out = torch.empty(v.shape[1], dtype=torch.float64, device=v.device)
    _lib.check("qeb_column_squared_norms", _lib.load().qeb_column_squared_norms(
        _precision(v), v.shape[0], v.shape[1], v.data_ptr(), leading_dimension(v),
        out.data_ptr(), stream_handle()))
    return out


def column_diagonal_expectations(v: torch.Tensor, diagonal: torch.Tensor) -> torch.Tensor:
    _check_matrix("v", v)
    d = diagonal.to(dtype=torch.float64).contiguous()
    out = torch.empty(v.shape[1], dtype=torch.float64, device=v.device)
    _lib.check("qeb_column_diagonal_expectations", _lib.load().qeb_column_diagonal_expectations(
        _precision(v), v.shape[0], v.shape[1], v.data_ptr(), leading_dimension(v),
        d.data_ptr(), out.data_ptr(), stream_handle()))
    return out


def column_inner_products(left: torch.Tensor, right: torch.Tensor) -> torch.Tensor:
    _check_matrix("left", left)
    _check_matrix("right", right)
    if left.shape != right.shape or left.dtype != right.dtype:
        raise ValueError("inner-product matrices disagree")
    out = torch.empty((left.shape[1], 2), dtype=torch.float64, device=left.device)
    _lib.check("qeb_column_inner_products", _lib.load().qeb_column_inner_products(
        _precision(left), left.shape[0], left.shape[1], left.data_ptr(), leading_dimension(left),
        right.data_ptr(), leading_dimension(right), out.data_ptr(), stream_handle()))
    return torch.view_as_complex(out)


def precondition(residuals: torch.Tensor, eigenvalues: torch.Tensor, diagonal: torch.Tensor,
                 out: torch.Tensor | None = None) -> torch.Tensor:
    """QE g_psi (qepy_pw/_native_fft.pyx:852-899)."""
    _check_matrix("residuals", residuals)
    rows, cols = residuals.shape
    e = eigenvalues.to(dtype=torch.float64).contiguous()
    d = diagonal.to(dtype=torch.float64).contiguous()
    if e.numel() != cols or d.numel() != rows:
        raise ValueError("eigenvalues/diagonal do not match the residual block")
    if out is None:
        out = empty_f(rows, cols, residuals.dtype, residuals.device)
    _lib.check("qeb_precondition", _lib.load().qeb_precondition(
        _precision(residuals), rows, cols, residuals.data_ptr(), leading_dimension(residuals),
        e.data_ptr(), d.data_ptr(), out.data_ptr(), leading_dimension(out), stream_handle()))
    return out


def normalize_columns(v: torch.Tensor, norms2: torch.Tensor, selected: torch.Tensor | None,
                      out: torch.Tensor) -> torch.Tensor:
    _check_matrix("v", v)
    _check_matrix("out", out)
    n2 = norms2.to(dtype=torch.float64).contiguous()
    sel = None if selected is None else selected.to(dtype=torch.int64).contiguous()
    cols = out.shape[1]
    _lib.check("qeb_normalize_columns", _lib.load().qeb_normalize_columns(
        _precision(v), v.shape[0], cols, v.data_ptr(), leading_dimension(v), n2.data_ptr(),
        0 if sel is None else sel.data_ptr(), out.data_ptr(), leading_dimension(out),
        stream_handle()))
    return out


def subtract_band_energies(residual: torch.Tensor, v: torch.Tensor,
                           energies: torch.Tensor) -> torch.Tensor:
    _check_matrix("residual", residual)
    _check_matrix("v", v)
    e = energies.to(dtype=torch.float64).contiguous()
    if residual.shape != v.shape or e.numel() != v.shape[1]:
        raise ValueError("residual matrices disagree")
    _lib.check("qeb_subtract_band_energies", _lib.load().qeb_subtract_band_energies(
        _precision(v), v.shape[0], v.shape[1], residual.data_ptr(), leading_dimension(residual),
        v.data_ptr(), leading_dimension(v), e.data_ptr(), stream_handle()))
    return residual


def accumulate_projector_diagonal(diagonal: torch.Tensor, coupled: torch.Tensor,
                                  beta: torch.Tensor, multiplicity: float) -> torch.Tensor:
    """diag += m Re sum_i coupled[:, i] conj(beta[:, i]) (qepy_pw/_native_fft.pyx:734-779)."""
    _check_matrix("coupled", coupled)
    _check_matrix("beta", beta)
    if coupled.shape != beta.shape or diagonal.numel() != beta.shape[0]:
        raise ValueError("projector diagonal operands disagree")
    if diagonal.dtype != torch.float64 or not diagonal.is_contiguous():
        raise ValueError("diagonal must be contiguous float64")
    _lib.check("qeb_accumulate_projector_diagonal", _lib.load().qeb_accumulate_projector_diagonal(
        _precision(beta), beta.shape[0], beta.shape[1], coupled.data_ptr(),
        leading_dimension(coupled), beta.data_ptr(), leading_dimension(beta),
        float(multiplicity), diagonal.data_ptr(), stream_handle()))
    return diagonal
