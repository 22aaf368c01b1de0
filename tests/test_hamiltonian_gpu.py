"""GPU parity of the complex GEMMs, Davidson column kernels, the full
Hamiltonian and the Davidson solver.

Oracles: NumPy restatements of the reference kernels (oracle/native_fft.py)
and, for Davidson, dense diagonalisation of the explicit H matrix.
Tolerances: FP64 1e-12 relative for single contractions; eigenvalues 1e-9 Ha.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import native_fft as oracle
from qe_python_b200 import kernels as K
from qe_python_b200.basis import LocalPotentialWorkspace, grid_slots, make_bases, fft_shape, potential_matrix
from qe_python_b200.diagonalization import (
    FactorizedProjectorTerm,
    PackedProjectorTerm,
    PlaneWaveHamiltonian,
    davidson,
)

pytestmark = pytest.mark.gpu


def _f(t):
    import torch

    return torch.from_numpy(np.asfortranarray(t)).cuda().T.contiguous().T if t.ndim == 2 else torch.from_numpy(t).cuda()


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (7, 5, 3), (64, 64, 16), (100, 37, 1000), (513, 257, 11019), (3, 4, 0)])
@pytest.mark.parametrize("dtype,rtol", [(np.complex128, 1e-13), (np.complex64, 2e-5)])
def test_gemm_conj_and_plain(cuda_device, m, n, k, dtype, rtol):
    rng = np.random.default_rng(m * 1000 + n + k)
    def rnd(*shape):
        return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)
    a_c, a_n, b, c0 = rnd(k, m), rnd(m, k), rnd(k, n), rnd(m, n)
    alpha, beta = 0.7 - 0.2j, 1.0 + 0.5j
    got_c = K.gemm(K.OP_C, _f(a_c), _f(b), _f(c0.copy()), alpha=alpha, beta=beta).cpu().numpy()
    exp_c = alpha * (a_c.astype(np.complex128).conj().T @ b) + beta * c0
    got_n = K.gemm(K.OP_N, _f(a_n), _f(b)).cpu().numpy()
    exp_n = a_n.astype(np.complex128) @ b
    scale = max(1.0, np.sqrt(k))
    assert np.max(np.abs(got_c - exp_c), initial=0.0) <= rtol * scale * max(1.0, np.max(np.abs(exp_c), initial=0.0))
    assert np.max(np.abs(got_n - exp_n), initial=0.0) <= rtol * scale * max(1.0, np.max(np.abs(exp_n), initial=0.0))


def test_gemm_strided_views(cuda_device):
    import torch

    rng = np.random.default_rng(4)
    big = rng.standard_normal((300, 50)) + 1j * rng.standard_normal((300, 50))
    t = _f(big)
    a = t[10:210, 3:20]
    b = t[10:210, 25:40]
    got = K.gemm(K.OP_C, a, b).cpu().numpy()
    exp = big[10:210, 3:20].conj().T @ big[10:210, 25:40]
    assert np.max(np.abs(got - exp)) < 1e-12 * np.max(np.abs(exp))


def test_column_kernels_match_oracle(cuda_device):
    rng = np.random.default_rng(8)
    v = np.asfortranarray(rng.standard_normal((777, 9)) + 1j * rng.standard_normal((777, 9)))
    w = np.asfortranarray(rng.standard_normal((777, 9)) + 1j * rng.standard_normal((777, 9)))
    e = rng.uniform(-1, 3, 9)
    d = rng.uniform(0, 20, 777)
    tv, tw = _f(v), _f(w)
    np.testing.assert_allclose(K.column_squared_norms(tv).cpu().numpy(), oracle.column_squared_norms(v), rtol=1e-13)
    np.testing.assert_allclose(K.column_inner_products(tv, tw).cpu().numpy(), oracle.column_inner_products(v, w), rtol=1e-13)
    np.testing.assert_allclose(K.column_diagonal_expectations(tv, _f(d)).cpu().numpy(), oracle.column_diagonal_expectations(v, d), rtol=1e-13)
    np.testing.assert_allclose(K.precondition(tv, _f(e), _f(d)).cpu().numpy(), oracle.qe_precondition(v, e, d), rtol=1e-14)
    r = w.copy()
    oracle.subtract_band_energies(r, v, e)
    tr = _f(w.copy())
    K.subtract_band_energies(tr, tv, _f(e))
    np.testing.assert_allclose(tr.cpu().numpy(), r, rtol=1e-14, atol=1e-14)
    norms = oracle.column_squared_norms(v)
    sel = np.array([0, 3, 8], dtype=np.int64)
    import torch
    out = torch.empty((3, 777), dtype=torch.complex128, device="cuda").T
    K.normalize_columns(tv, _f(norms), _f(sel), out)
    np.testing.assert_allclose(out.cpu().numpy(), oracle.normalize_selected_columns(v, norms, sel), rtol=1e-14)


FCC = 10.26 / 2.0 * np.array([[-1.0, 0.0, 1.0], [0.0, 1.0, 1.0], [-1.0, 1.0, 0.0]])


def _system(seed=3, nproj_atoms=2, k=(0.125, 0.125, 0.375), ecut=20.0):
    reciprocal = 2.0 * np.pi * np.linalg.inv(FCC).T
    basis = make_bases(reciprocal, np.asarray(k), ecut)[0].materialize()
    shape = fft_shape([basis], reciprocal, 4 * ecut)
    rng = np.random.default_rng(seed)
    npw = len(basis)
    # smooth potential: a few low Fourier components
    vg = np.zeros(shape, dtype=complex)
    for _ in range(12):
        idx = tuple(rng.integers(-2, 3, 3) % np.array(shape))
        vg[idx] += rng.uniform(-0.3, 0.3)
    vr = np.real(np.fft.ifftn(vg) * np.prod(shape))
    vr = 0.5 * (vr + vr)  # real part of a non-Hermitian vg is a valid real potential
    # amplitude 0.05 keeps the nonlocal eigenvalues O(1) Ha, like real projectors
    species = (rng.standard_normal((npw, 4)) + 1j * rng.standard_normal((npw, 4))) \
        * 0.05 * np.exp(-basis.kinetic / 4)[:, None]
    positions = rng.uniform(0, 5, (nproj_atoms, 3))
    phases = np.exp(-1j * basis.vectors @ positions.T)
    d = rng.uniform(-1, 1, (4, 4))
    coupling = 0.5 * (d + d.T)
    return basis, shape, vr, np.asfortranarray(species), np.asfortranarray(phases), coupling


def _dense_h(basis, shape, vr, beta_packed, coupling_packed):
    vg = np.fft.fftn(vr) / np.prod(shape)
    h = potential_matrix(vg, basis.indices) + np.diag(basis.kinetic)
    return h + beta_packed @ coupling_packed @ beta_packed.conj().T


def test_hamiltonian_matches_oracle_composition(cuda_device):
    basis, shape, vr, species, phases, coupling = _system()
    natoms = phases.shape[1]
    packed = np.asfortranarray(np.concatenate([species * phases[:, [a]] for a in range(natoms)], axis=1))
    cpacked = np.kron(np.eye(natoms), coupling)
    rng = np.random.default_rng(1)
    psi = np.asfortranarray(rng.standard_normal((len(basis), 6)) + 1j * rng.standard_normal((len(basis), 6)))
    # oracle: apply_serial + kinetic, then projector_overlaps / add_projector_product
    linear, *_ = grid_slots(basis.indices, shape)
    size = int(np.prod(shape))
    grid = np.zeros((6, size), dtype=complex)
    plan = oracle.NativeFFTWPlan(grid, shape, 6, 1, size)
    expected = np.zeros_like(psi)
    oracle.apply_serial(grid, psi, vr, linear, plan, size, size, expected, 0, basis.kinetic)
    becp = oracle.projector_overlaps(packed, psi)
    coupled = np.asfortranarray(cpacked @ becp)
    assert oracle.add_projector_product(expected, packed, coupled)
    ws = LocalPotentialWorkspace(basis, shape)
    for terms in ((FactorizedProjectorTerm(species, phases, coupling),),
                  ((packed, cpacked),),
                  (PackedProjectorTerm(packed, cpacked, np.zeros(len(basis))),)):
        h = PlaneWaveHamiltonian(basis, np.zeros(shape), terms, local_workspace=ws, real_potential=vr)
        got = h.apply(_f(psi)).cpu().numpy()
        assert np.max(np.abs(got - expected)) <= 1e-12 * np.max(np.abs(expected))
    dense = _dense_h(basis, shape, vr, packed, cpacked)
    assert np.max(np.abs(dense @ psi - expected)) <= 1e-11 * np.max(np.abs(expected))
    # preconditioner diagonal: kinetic + v_of_0 + Re diag(beta D beta^H)
    h = PlaneWaveHamiltonian(basis, np.zeros(shape), (FactorizedProjectorTerm(species, phases, coupling),),
                             local_workspace=ws, real_potential=vr, potential_average=0.25)
    want = basis.kinetic + 0.25 + np.real(np.einsum("gi,ij,gj->g", packed, cpacked, packed.conj()))
    np.testing.assert_allclose(h.diagonal.cpu().numpy(), want, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("lock", [False, True])
@pytest.mark.parametrize("precision,tol", [("f64", 1e-9), ("f32", 2e-5)])
def test_davidson_matches_dense_eigenvalues(cuda_device, precision, tol, lock):
    """With ``lock_converged`` the roots converged at a restart leave the
    reduced problem (subspace of twice the roots, so restarts happen); the
    eigenpairs must be the same to the tolerance."""
    import torch

    basis, shape, vr, species, phases, coupling = _system(seed=5)
    natoms = phases.shape[1]
    packed = np.concatenate([species * phases[:, [a]] for a in range(natoms)], axis=1)
    cpacked = np.kron(np.eye(natoms), coupling)
    exact = np.linalg.eigvalsh(_dense_h(basis, shape, vr, packed, cpacked))[:8]
    ws = LocalPotentialWorkspace(basis, shape, precision=precision)
    h = PlaneWaveHamiltonian(basis, np.zeros(shape), (FactorizedProjectorTerm(species, phases, coupling),),
                             local_workspace=ws, real_potential=vr, potential_average=float(np.mean(vr)))
    rng = np.random.default_rng(2)
    start = rng.standard_normal((len(basis), 8)) + 1j * rng.standard_normal((len(basis), 8))
    start *= (1.0 / (1.0 + basis.kinetic))[:, None]
    dtype = torch.complex128 if precision == "f64" else torch.complex64
    # FP32 residual norms floor near 1e-6 |H|: the FP32 form converges on the
    # eigenvalue change alone (residual_factor=None, as the SCF driver calls it)
    result = davidson(h.apply, h.diagonal, 8, initial_vectors=_f(start).to(dtype),
                      tolerance=1e-11 if precision == "f64" else 1e-6, max_iterations=200,
                      subspace_multiplier=2 if lock else 4, operator_into=h.apply_into,
                      residual_factor=10.0 if precision == "f64" else None, lock_converged=lock)
    assert result.converged
    assert np.all(np.diff(result.eigenvalues) >= 0)
    np.testing.assert_allclose(result.eigenvalues, exact, atol=tol)
    # Ritz vectors are H-eigenvectors: ||H x - e x|| small
    hx = h.apply(result.eigenvectors)
    res = (hx - result.eigenvectors * torch.as_tensor(result.eigenvalues, device="cuda").to(hx.real.dtype)[None, :]).abs().max()
    assert float(res) < (1e-6 if precision == "f64" else 5e-3)


def test_hamiltonian_matches_reference_golden(cuda_device):
    """Reference PlaneWaveHamiltonian.apply (factorized + packed + materialised
    terms; tests/golden/hamiltonian_small.npz) against the GPU operator."""
    from pathlib import Path

    g = np.load(Path(__file__).resolve().parent / "golden" / "hamiltonian_small.npz")
    shape = tuple(int(v) for v in g["shape"])
    from qe_python_b200.basis import PlaneWaveBasis

    basis = PlaneWaveBasis(g["miller"], np.zeros((len(g["miller"]), 3)), g["kinetic"])
    ws = LocalPotentialWorkspace(basis, shape)
    terms = (FactorizedProjectorTerm(g["species"], g["phases"], g["coupling"]),
             PackedProjectorTerm(g["packed_beta"], g["packed_coupling"], g["packed_diag"]),
             (g["mat_beta"], g["mat_coupling"]))
    h = PlaneWaveHamiltonian(basis, None, terms, local_workspace=ws, real_potential=g["potential"],
                             potential_average=0.125)
    got = h.apply(_f(g["psi"])).cpu().numpy()
    assert np.max(np.abs(got - g["hpsi"])) <= 1e-12 * np.max(np.abs(g["hpsi"]))
    np.testing.assert_allclose(h.diagonal.cpu().numpy(), g["diagonal"], rtol=1e-12, atol=1e-13)


def test_davidson_matches_reference_golden(cuda_device):
    """Same operator, start vectors and settings as the reference davidson run
    of tests/golden/davidson_small.npz (tolerance 1e-9 Ha, ndim 2)."""
    from pathlib import Path

    here = Path(__file__).resolve().parent / "golden"
    g = np.load(here / "hamiltonian_small.npz")
    d = np.load(here / "davidson_small.npz")
    shape = tuple(int(v) for v in g["shape"])
    from qe_python_b200.basis import PlaneWaveBasis

    basis = PlaneWaveBasis(g["miller"], np.zeros((len(g["miller"]), 3)), g["kinetic"])
    ws = LocalPotentialWorkspace(basis, shape)
    terms = (FactorizedProjectorTerm(g["species"], g["phases"], g["coupling"]),
             PackedProjectorTerm(g["packed_beta"], g["packed_coupling"], g["packed_diag"]),
             (g["mat_beta"], g["mat_coupling"]))
    h = PlaneWaveHamiltonian(basis, None, terms, local_workspace=ws, real_potential=g["potential"],
                             potential_average=0.125)
    result = davidson(h.apply, h.diagonal, 8, initial_vectors=_f(d["start"]), tolerance=1e-9,
                      max_iterations=100, subspace_multiplier=2, residual_factor=None,
                      operator_into=h.apply_into)
    assert result.converged == bool(d["converged"])
    np.testing.assert_allclose(result.eigenvalues, d["eigenvalues"], atol=5e-9)
    # the trajectory follows the reference's within a couple of iterations
    assert abs(result.iterations - float(d["iterations"])) <= 2


@pytest.mark.parametrize("op,m,n,k", [
    (K.OP_C, 300, 3, 30000),   # calbec of a few bands: narrow N, split K
    (K.OP_C, 5, 700, 30000),   # Davidson rows of a few new vectors: narrow M (swapped)
    (K.OP_C, 16, 16, 2000),    # both narrow, at the limit
    (K.OP_C, 40, 9, 100),      # one K slice
    (K.OP_N, 30000, 3, 960),   # Ritz columns / projector add of a few bands
    (K.OP_N, 5000, 16, 37),    # ragged K chunk
    (K.OP_N, 77, 1, 1),
])
@pytest.mark.parametrize("dtype,rtol", [(np.complex128, 1e-13), (np.complex64, 2e-6)])
def test_skinny_products(cuda_device, op, m, n, k, dtype, rtol):
    """Outputs with at most 16 columns on one side go through the streaming
    kernels of qeb_zgemm / qeb_cgemm; strided operands (leading dimension
    above the row count) and alpha, beta != 0 included."""
    import torch

    rng = np.random.default_rng(m + 7 * n + 13 * k)
    def rnd(*shape):
        return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)
    rows_a = k if op == K.OP_C else m
    a_full, b_full, c_full = rnd(rows_a + 3, (m if op == K.OP_C else k)), rnd(k + 5, n), rnd(m + 2, n)
    a, b, c0 = a_full[:rows_a], b_full[:k], c_full[:m]
    alpha, beta = 0.3 + 0.9j, -0.5 + 0.25j
    ta, tb, tc = _f(a_full)[:rows_a], _f(b_full)[:k], _f(c_full.copy())[:m]
    assert K.is_skinny(op, m, n)
    got = K.gemm(op, ta, tb, tc, alpha=alpha, beta=beta).cpu().numpy()
    a64, b64 = a.astype(np.complex128), b.astype(np.complex128)
    exp = alpha * ((a64.conj().T if op == K.OP_C else a64) @ b64) + beta * c0
    scale = max(1.0, np.sqrt(k)) * max(1.0, np.max(np.abs(exp)))
    assert np.max(np.abs(got - exp)) <= rtol * scale
