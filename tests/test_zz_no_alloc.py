"""The allocation-free GEMM entry point against the regular one.

``qeb_zgemm_static_scratch`` serves callers that cannot allocate device
memory (for example code running inside a memory pool it does not own): its
split-K partial tiles live in a fixed array inside the library instead of in
caller scratch.  This test calls it through the C ABI several times in a
row, with different operands, and checks each result against an
independent complex128 product on the host (NumPy) and against
``qeb_zgemm`` with caller-provided scratch, at the GEMM tolerance used
elsewhere (1e-13 relative, scaled by sqrt(K)).  The shapes cover the tiled
split-K path and both skinny split-K paths (a narrow output of at most 16
columns on either side).
It is collected last so that a failure here leaves every other test already
run; it passes on its own in a fresh process as well.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1.0e-13


def _operands(rng, m, n, k, torch):
    def rnd(rows, cols):
        host = rng.standard_normal((cols, rows)) + 1j * rng.standard_normal((cols, rows))
        return torch.from_numpy(host).cuda().T  # column-major (rows, cols)
    return rnd(k, m), rnd(k, n), rnd(m, n)


def _pair(v: complex):
    return (ctypes.c_double * 2)(v.real, v.imag)


def test_static_scratch_gemm_matches_regular_entry(cuda_device):
    import torch

    from qe_python_b200 import _lib

    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(20261203)
    # Shapes whose long K makes both entry points split K across blocks: two
    # tiled products, then a narrow M (swapped skinny plan) and a narrow N.
    cases = [(96, 80, 20000, 0.75 - 0.25j, 0.0), (40, 33, 11019, 1.0, 0.5 + 1.0j),
             (8, 300, 20000, 1.0, 0.0), (300, 12, 20000, -0.5 + 0.5j, 1.0)]
    for m, n, k, alpha, beta in cases:
        a, b, c0 = _operands(rng, m, n, k, torch)
        expected = c0.clone()
        need = int(lib.qeb_zgemm_scratch_bytes(1, m, n, k, 0))
        assert need > 0, "the case must exercise the split-K partial buffer"
        scratch = torch.empty(need, dtype=torch.uint8, device="cuda")
        status = lib.qeb_zgemm(1, m, n, k, _pair(complex(alpha)), a.data_ptr(), a.stride(1),
                               b.data_ptr(), b.stride(1), _pair(complex(beta)),
                               expected.data_ptr(), expected.stride(1), scratch.data_ptr(), need,
                               stream)
        _lib.check("qeb_zgemm", status)
        got = c0.clone()
        status = lib.qeb_zgemm_static_scratch(m, n, k, _pair(complex(alpha)), a.data_ptr(),
                                              a.stride(1), b.data_ptr(), b.stride(1),
                                              _pair(complex(beta)), got.data_ptr(), got.stride(1),
                                              stream)
        _lib.check("qeb_zgemm_static_scratch", status)
        torch.cuda.synchronize()
        host = alpha * (a.cpu().numpy().conj().T @ b.cpu().numpy()) + beta * c0.cpu().numpy()
        bound = RTOL * max(1.0, np.sqrt(k)) * np.max(np.abs(host))
        result = got.cpu().numpy()
        assert np.max(np.abs(result - host)) <= bound, (m, n, k)
        assert np.max(np.abs(result - expected.cpu().numpy())) <= bound, (m, n, k)


def test_static_scratch_gemm_rejects_oversized_output(cuda_device):
    import torch

    from qe_python_b200 import _lib

    lib = _lib.load()
    capacity = int(lib.qeb_zgemm_static_scratch_capacity())
    side = int(np.sqrt(capacity // 32)) + 2  # M*N*16*2 just above capacity
    status = lib.qeb_zgemm_static_scratch(side, side, 64, _pair(1.0), None, 64, None, 64,
                                          _pair(0.0), None, side,
                                          torch.cuda.current_stream().cuda_stream)
    assert status == -2
    assert "exceeds" in _lib.last_error()
