"""The reduced eigensolve without a host synchronisation (eigensolver.py).

* zheevd_async (cuSOLVER zheevd on a chosen stream, error code on the
  device) against NumPy's Hermitian eigensolver;
* ReducedSolve (Cholesky reduction, zheevd, back-substitution) against
  SciPy's generalized eigensolver on a Davidson-like pencil, and its
  fallback to the canonical orthogonalisation when S is singular;
* four solves enqueued on four streams before any is read give the same
  pairs as the same solves one after another.
"""

from __future__ import annotations

import numpy as np
import pytest
import scipy.linalg

pytestmark = pytest.mark.gpu


def _hermitian(rng, n, scale=1.0):
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    return scale * 0.5 * (a + a.conj().T)


def test_zheevd_async_matches_numpy(cuda_device):
    import torch

    from qe_python_b200.eigensolver import zheevd_async

    rng = np.random.default_rng(3)
    for n in (1, 7, 300):
        m = _hermitian(rng, n)
        stream = torch.cuda.Stream(cuda_device)
        values, vectors, info = zheevd_async(torch.from_numpy(m).to(cuda_device), stream)
        torch.cuda.synchronize()
        assert int(info) == 0
        want = np.linalg.eigvalsh(m)
        got = values.cpu().numpy()
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-12 * max(1.0, np.abs(want).max()))
        v = vectors.cpu().numpy()
        assert np.max(np.abs(m @ v - v * got[None, :])) < 1e-11 * np.abs(want).max()
        assert np.max(np.abs(v.conj().T @ v - np.eye(n))) < 1e-12


def test_reduced_solve_matches_scipy_generalized(cuda_device):
    import torch

    from qe_python_b200.diagonalization import lowest_generalized_eigh

    rng = np.random.default_rng(4)
    n, roots = 400, 150
    # Davidson-like: a diagonal Ritz block bordered by correction rows, with
    # an overlap near the identity
    h = _hermitian(rng, n, 0.05)
    h[np.arange(roots), np.arange(roots)] += np.sort(rng.uniform(-1.0, 1.0, roots))
    g = 0.01 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    s = np.eye(n) + 0.5 * (g + g.conj().T)
    want_values, want_vectors = scipy.linalg.eigh(h, s, subset_by_index=(0, roots - 1))
    values, vectors = lowest_generalized_eigh(torch.from_numpy(h).to(cuda_device),
                                              torch.from_numpy(s).to(cuda_device), roots)
    got = values.cpu().numpy()
    np.testing.assert_allclose(got, want_values, rtol=0, atol=1e-12)
    x = vectors.cpu().numpy()
    assert np.max(np.abs(h @ x - (s @ x) * got[None, :])) < 1e-11
    assert np.max(np.abs(x.conj().T @ s @ x - np.eye(roots))) < 1e-11


def test_reduced_solve_falls_back_on_a_singular_overlap(cuda_device):
    import torch

    from qe_python_b200.diagonalization import _canonical_generalized_eigh, lowest_generalized_eigh

    rng = np.random.default_rng(5)
    n, roots = 60, 20
    basis = rng.standard_normal((n, n - 5)) + 1j * rng.standard_normal((n, n - 5))
    # five columns repeat others: S = B^H B with B of rank n - 5, pushed
    # slightly negative along the null directions so that the Cholesky
    # factorisation fails for certain
    full = np.concatenate([basis, basis[:, :5]], axis=1)
    op = _hermitian(rng, n)
    h = full.conj().T @ op @ full
    s = full.conj().T @ full
    for i in range(5):
        u = np.zeros(n)
        u[i], u[n - 5 + i] = 1.0, -1.0
        s -= 1.0e-9 * np.outer(u, u)
    h_d, s_d = torch.from_numpy(h).to(cuda_device), torch.from_numpy(s).to(cuda_device)
    values, vectors = lowest_generalized_eigh(h_d, s_d, roots)
    want_values, _ = _canonical_generalized_eigh(h_d, s_d, roots)
    np.testing.assert_allclose(values.cpu().numpy(), want_values.cpu().numpy(), rtol=0,
                               atol=1e-9)
    # the pencil's finite eigenvalues are those of op on span(basis)
    q, _ = np.linalg.qr(basis)
    exact = np.linalg.eigvalsh(q.conj().T @ op @ q)[:roots]
    np.testing.assert_allclose(values.cpu().numpy(), exact, rtol=0, atol=1e-8)


def test_solves_on_four_streams_equal_sequential_solves(cuda_device):
    import torch

    from qe_python_b200.eigensolver import ReducedSolve

    rng = np.random.default_rng(6)
    pencils = []
    for n in (210, 233, 180, 256):
        h = _hermitian(rng, n)
        g = 0.01 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
        s = np.eye(n) + 0.5 * (g + g.conj().T)
        pencils.append((torch.from_numpy(h).to(cuda_device), torch.from_numpy(s).to(cuda_device)))
    sequential = []
    for h, s in pencils:
        solve = ReducedSolve(torch.cuda.current_stream(cuda_device))
        solve.launch(h, s, 100)
        values, vectors = solve.result()
        sequential.append((values.cpu().numpy(), vectors.cpu().numpy()))
    solves = [ReducedSolve(torch.cuda.Stream(cuda_device)) for _ in pencils]
    for solve, (h, s) in zip(solves, pencils):
        solve.launch(h, s, 100)
    for solve, (h, s), (want_values, want_vectors) in zip(solves, pencils, sequential):
        values, vectors = solve.result()
        np.testing.assert_allclose(values.cpu().numpy(), want_values, rtol=0, atol=1e-13)
        # S-orthonormal eigenvectors, equal up to a phase per column
        got = vectors.cpu().numpy()
        phase = np.sum(want_vectors.conj() * (s.cpu().numpy() @ got), axis=0)
        assert np.allclose(np.abs(phase), 1.0, atol=1e-10)
