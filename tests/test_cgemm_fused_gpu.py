"""Split-TF32 GEMM on unpacked complex64 operands (qeb_cgemm_tf32x3) against
complex128 products (GPU).

Tolerance as for the packed kernel: |error| <= 2e-6 * sqrt(2K) * max|C| for
unit-variance inputs (FP32 accumulation of 2K products).  Shapes cover
partial tiles in M, N and K, split-K (few output tiles, long K), the H|psi>
projector shapes (11019 x 512 x 256) and the Davidson subspace shapes.
"""

from __future__ import annotations

import numpy as np
import pytest

from qe_python_b200 import kernels as K

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch

    from qe_python_b200.device import to_device_f

    return to_device_f(a, torch.complex64)


def _ref(op, a, b, c0, alpha, beta):
    a = a.astype(np.complex64).astype(complex)
    b = b.astype(np.complex64).astype(complex)
    prod = a.conj().T @ b if op == K.OP_C else a @ b
    return alpha * prod + beta * c0.astype(np.complex64)


def _tol(k, exp):
    return 2e-6 * max(1.0, np.sqrt(2 * k)) * max(1.0, np.max(np.abs(exp), initial=0.0))


@pytest.mark.parametrize("op,m,n,k", [
    (K.OP_C, 1, 1, 1), (K.OP_C, 128, 128, 16), (K.OP_C, 130, 70, 33), (K.OP_C, 512, 256, 11019),
    (K.OP_C, 480, 960, 4001), (K.OP_C, 3, 300, 20000),
    (K.OP_N, 1, 1, 1), (K.OP_N, 128, 128, 16), (K.OP_N, 129, 65, 17), (K.OP_N, 11019, 256, 512),
    (K.OP_N, 4001, 480, 960), (K.OP_N, 300, 3, 7),
])
def test_fused_matches_complex128(cuda_device, op, m, n, k):
    rng = np.random.default_rng(m + 7 * n + 13 * k + op)
    shape_a = (k, m) if op == K.OP_C else (m, k)
    a = rng.standard_normal(shape_a) + 1j * rng.standard_normal(shape_a)
    b = rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))
    c0 = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
    alpha, beta = 0.5 - 0.25j, 1.0 + 0.5j
    got = K.cgemm_tf32x3(op, _dev(a), _dev(b), _dev(c0), alpha, beta)
    assert got is not None
    exp = _ref(op, a, b, c0, alpha, beta)
    assert np.max(np.abs(got.cpu().numpy() - exp)) <= _tol(k, exp)
    # beta = 0 with a fresh output
    got0 = K.cgemm_tf32x3(op, _dev(a), _dev(b)).cpu().numpy()
    exp0 = _ref(op, a, b, c0, 1.0, 0.0)
    assert np.max(np.abs(got0 - exp0)) <= _tol(k, exp0)
    assert K.tf32_error() == 0


def test_fused_declines_odd_leading_dimension(cuda_device):
    import torch

    a = torch.zeros((5, 3), dtype=torch.complex64, device="cuda").T.contiguous().T  # ld = 5
    b = torch.zeros((6, 2), dtype=torch.complex64, device="cuda").T.contiguous().T
    assert K.cgemm_tf32x3(K.OP_C, a, b[:5]) is None
    # the generic entry point still answers through the packed kernel
    out = K.gemm_tf32(K.OP_C, a, b[:5])
    assert out.shape == (3, 2) and float(out.abs().max()) == 0.0


def test_gemm_routes_large_complex64_to_tensor_cores(cuda_device):
    import torch

    rng = np.random.default_rng(5)
    a = rng.standard_normal((3000, 200)) + 1j * rng.standard_normal((3000, 200))
    b = rng.standard_normal((3000, 100)) + 1j * rng.standard_normal((3000, 100))
    from qe_python_b200 import _lib

    launches = _lib.load().qeb_launch_count()
    got = K.gemm(K.OP_C, _dev(a), _dev(b)).cpu().numpy()
    exp = _ref(K.OP_C, a, b, np.zeros((200, 100)), 1.0, 0.0)
    assert np.max(np.abs(got - exp)) <= _tol(3000, exp)
    assert _lib.load().qeb_launch_count() > launches
    # forced FP32-pipe path agrees to the same tolerance
    simt = K.gemm(K.OP_C, _dev(a), _dev(b), tensor=False).cpu().numpy()
    assert np.max(np.abs(simt - exp)) <= _tol(3000, exp)
    assert torch.cuda.is_available()


@pytest.mark.parametrize("op,m,n,k", [
    (K.OP_N, 11019, 256, 512),   # 174 output tiles: one wave + a 26-tile tail
    (K.OP_C, 20000, 130, 300),   # 314 tiles: two waves + an 18-tile tail
    (K.OP_N, 19100, 260, 96),    # 450 tiles: three waves + a 6-tile tail, short K
])
def test_unsplit_product_with_tail_wave(cuda_device, op, m, n, k):
    """An unsplit product (splits=1) whose last wave of output tiles is at most
    half full runs that tail with its K range split and reduced apart from
    the full waves; the result must be the same product."""
    rng = np.random.default_rng(m + n + k)
    shape_a = (k, m) if op == K.OP_C else (m, k)
    a = rng.standard_normal(shape_a) + 1j * rng.standard_normal(shape_a)
    b = rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))
    c0 = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
    alpha, beta = 0.75 + 0.5j, -0.5 + 1.0j
    exp = _ref(op, a, b, c0, alpha, beta)
    for _ in range(2):
        got = K.cgemm_tf32x3(op, _dev(a), _dev(b), _dev(c0), alpha, beta, splits=1)
        assert got is not None
        assert np.max(np.abs(got.cpu().numpy() - exp)) <= _tol(k, exp)
    assert K.tf32_error() == 0
