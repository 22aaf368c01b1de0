"""Split-TF32 tcgen05 complex GEMM against complex128 products (GPU).

Tolerance: split TF32 (hi*hi + hi*lo + lo*hi, FP32 accumulation in tensor
memory) is FP32-level accurate: |error| <= 2e-6 * sqrt(2K) * max|C| (the
accumulation error of 2K FP32 additions), for unit-variance inputs.
"""

from __future__ import annotations

import numpy as np
import pytest

from qe_python_b200 import kernels as K

pytestmark = pytest.mark.gpu


def _f(a, dtype):
    import torch

    return torch.from_numpy(np.asfortranarray(a)).to(dtype).cuda().T.contiguous().T


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (128, 64, 16), (130, 70, 33), (512, 256, 11019),
                                   (40, 300, 2000), (7, 5, 0)])
def test_tf32_gemm_conj_transpose(cuda_device, m, n, k):
    import torch

    rng = np.random.default_rng(m + 7 * n + 13 * k)
    a = rng.standard_normal((k, m)) + 1j * rng.standard_normal((k, m))
    b = rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))
    c0 = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
    alpha, beta = 0.5 - 0.25j, 1.0 + 0.5j
    got = K.gemm_tf32(K.OP_C, _f(a, torch.complex64), _f(b, torch.complex64),
                      _f(c0, torch.complex64), alpha, beta).cpu().numpy()
    exp = alpha * (a.astype(np.complex64).astype(complex).conj().T
                   @ b.astype(np.complex64).astype(complex)) + beta * c0.astype(np.complex64)
    tol = 2e-6 * max(1.0, np.sqrt(2 * k)) * max(1.0, np.max(np.abs(exp), initial=0.0))
    assert np.max(np.abs(got - exp), initial=0.0) <= tol
    assert K.tf32_error() == 0


@pytest.mark.parametrize("m,n,k", [(11019, 256, 512), (300, 20, 9), (64, 64, 64)])
def test_tf32_gemm_plain(cuda_device, m, n, k):
    import torch

    rng = np.random.default_rng(m + n + k)
    a = rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))
    b = rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))
    c0 = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
    got = K.gemm_tf32(K.OP_N, _f(a, torch.complex64), _f(b, torch.complex64),
                      _f(c0, torch.complex64), 1.0, 1.0).cpu().numpy()
    exp = a.astype(np.complex64).astype(complex) @ b.astype(np.complex64).astype(complex) \
        + c0.astype(np.complex64)
    tol = 2e-6 * max(1.0, np.sqrt(2 * k)) * np.max(np.abs(exp))
    assert np.max(np.abs(got - exp)) <= tol
    assert K.tf32_error() == 0


def test_tf32_pack_layouts(cuda_device):
    import torch

    rng = np.random.default_rng(3)
    a = (rng.standard_normal((5, 3)) + 1j * rng.standard_normal((5, 3))).astype(np.complex64)
    t = _f(a, torch.complex64)
    for layout, fn in ((K.PACK_RAW, lambda z: (z.real, z.imag)),
                       (K.PACK_SWAPNEG, lambda z: (z.imag, -z.real)),
                       (K.PACK_NEGIM, lambda z: (z.real, -z.imag)),
                       (K.PACK_SWAP, lambda z: (z.imag, z.real))):
        p = K.tf32_pack(t, layout)
        full = (p.hi + p.lo).cpu().numpy()
        assert full.shape == (3, 32)
        for col in range(3):
            x, y = fn(a[:, col])
            np.testing.assert_allclose(full[col, 0:10:2], x, rtol=1e-6)
            np.testing.assert_allclose(full[col, 1:10:2], y, rtol=1e-6)
            assert np.all(full[col, 10:] == 0)
        hi = p.hi.cpu().numpy().view(np.uint32)
        assert np.all(hi & 0x1FFF == 0)  # hi is exactly representable in TF32
    pt = K.tf32_pack(t, K.PACK_RAW, transposed=True)
    full = (pt.hi + pt.lo).cpu().numpy()
    np.testing.assert_allclose(full[:, 0:6:2], a.real, rtol=1e-6)
    np.testing.assert_allclose(full[:, 1:6:2], a.imag, rtol=1e-6)
