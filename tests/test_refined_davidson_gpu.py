"""The chosen form's refined Davidson (FP64 Ritz block, FP32 corrections).

* Small cell: ``refined_davidson_steps`` driven with the FP64 and the
  chosen-form (FP32 FFT passes, split-TF32 / FP32 GEMMs) Hamiltonians gives
  the eigenvalues of dense diagonalisation of the FP64 operator within its
  rounding budget (1e-8 Ha by default; 1e-10 Ha with a 1e-12 budget),
  through restarts (subspace of twice the roots), and FP64 residuals of
  its eigenvectors at the Davidson threshold's level.
* Benchmark cells (64 atoms, 4 k; 216 atoms, Gamma): the mixed SCF's final
  eigenvalues against a tight plain-FP64 Davidson on the same fixed
  potential (the mixed SCF's last V_eff) from the mixed eigenvectors:
  every one of the nbnd eigenvalues within 1e-7 Ry, the plain form's bar
  (measured 4e-11 Ry; the chosen form's bar is 1e-6 Ry).  This is the arithmetic
  error of the chosen form alone; differences between two separately
  converged SCFs also carry the difference of their mixing paths.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _small_operators(device):
    import torch

    from qe_python_b200.basis import LocalPotentialWorkspace, fft_shape, make_bases
    from qe_python_b200.diagonalization import PlaneWaveHamiltonian

    lattice = 10.26 / 2.0 * np.array([[-1.0, 0.0, 1.0], [0.0, 1.0, 1.0], [-1.0, 1.0, 0.0]])
    reciprocal = 2.0 * np.pi * np.linalg.inv(lattice).T
    basis = make_bases(reciprocal, np.array([0.125, 0.375, -0.25]), 20.0)[0]
    shape = fft_shape([basis], reciprocal, 80.0)
    rng = np.random.default_rng(31)
    npw = len(basis)
    beta = np.asfortranarray((rng.standard_normal((npw, 8)) + 1j * rng.standard_normal((npw, 8)))
                             * 0.3 * np.exp(-basis.kinetic / 3.0)[:, None])
    d = rng.uniform(-1.0, 1.0, (8, 8))
    coupling = 0.5 * (d + d.T)
    v = torch.from_numpy(np.ascontiguousarray(rng.uniform(-0.5, 0.5, shape))).to(device)
    hams = {}
    for precision in ("f64", "f32"):
        ws = LocalPotentialWorkspace(basis, shape, precision=precision, device=device)
        hams[precision] = PlaneWaveHamiltonian(basis, None, ((beta, coupling),),
                                               local_workspace=ws, real_potential=v,
                                               potential_average=0.0)
    return basis, hams


def test_refined_davidson_matches_dense(cuda_device):
    import torch

    from qe_python_b200.device import to_device_f
    from qe_python_b200.diagonalization import refined_davidson_steps
    from qe_python_b200.scf import _drive

    basis, hams = _small_operators(cuda_device)
    ham64, ham32 = hams["f64"], hams["f32"]
    npw = len(basis)
    dense = np.zeros((npw, npw), dtype=np.complex128)
    eye = np.eye(npw, dtype=np.complex128)
    for start in range(0, npw, 64):
        block = torch.from_numpy(np.asfortranarray(eye[:, start:start + 64])).to(cuda_device)
        dense[:, start:start + 64] = ham64.apply(block).cpu().numpy()
    exact = np.linalg.eigvalsh(0.5 * (dense + dense.conj().T))
    roots = 8
    rng = np.random.default_rng(5)
    start = rng.standard_normal((npw, roots)) + 1j * rng.standard_normal((npw, roots))
    start = np.linalg.qr(start)[0]
    # the default rounding budget (1e-8 Ha), then a tight one: the FP64
    # Rayleigh-Ritz step is redone whenever the carried residual's FP32
    # rounding would pass the budget, which bounds the eigenvalue error
    for budget, bound in ((None, 1.0e-8), (1.0e-12, 1.0e-10)):
        steps = refined_davidson_steps(
            ham64.diagonal, roots, initial_vectors=to_device_f(start, torch.complex128, cuda_device),
            tolerance=1.0e-11, max_iterations=80, subspace_multiplier=2, budget=budget)
        result = _drive(steps, ham64, ham32)
        assert result.converged
        assert result.eigenvectors.dtype == torch.complex128
        assert np.max(np.abs(result.eigenvalues - exact[:roots])) < bound, budget
    hx = ham64.apply(result.eigenvectors).cpu().numpy()
    x = result.eigenvectors.cpu().numpy()
    residual = hx - x * result.eigenvalues[None, :]
    assert np.max(np.linalg.norm(residual, axis=0)) < 1.0e-4
    overlap = x.conj().T @ x
    assert np.max(np.abs(overlap - np.eye(roots))) < 1.0e-6


@pytest.mark.parametrize("name", ["scf-dia64", "scf-dia216"])
def test_mixed_scf_eigenvalues_at_fixed_potential(cuda_device, name):
    import torch

    from qe_python_b200.basis import LocalPotentialWorkspace
    from qe_python_b200.diagonalization import PlaneWaveHamiltonian, davidson
    from qe_python_b200.scf import benchmark_system, projector_terms, run_scf, scf_setup

    system = benchmark_system(name)
    mixed = run_scf(system, precision="mixed")
    assert mixed.converged
    assert "refined" in mixed.precision_log
    setup = scf_setup(system, cuda_device)
    worst = 0.0
    for k, basis in enumerate(setup.bases):
        ws = LocalPotentialWorkspace(basis, setup.shape, precision="f64", device=cuda_device)
        ham = PlaneWaveHamiltonian(basis, None, projector_terms(system, setup.tables, basis),
                                   local_workspace=ws, real_potential=mixed.potential,
                                   potential_average=setup.v_ion_average)
        vectors = mixed.eigenvectors[k]
        check = davidson(ham.apply, ham.diagonal, vectors.shape[1], initial_vectors=vectors,
                         tolerance=1.0e-10, max_iterations=200,
                         subspace_multiplier=system.diago_david_ndim, residual_factor=None,
                         occupied_roots=system.nbnd, initial_is_orthonormal=True,
                         operator_into=ham.apply_into)
        diff = 2.0 * np.max(np.abs(np.asarray(check.eigenvalues)[:system.nbnd]
                                   - np.asarray(mixed.eigenvalues_ha[k])[:system.nbnd]))
        worst = max(worst, diff)
    assert worst <= 1.0e-7, f"{name}: mixed vs FP64 at the same potential {worst:.3e} Ry"
