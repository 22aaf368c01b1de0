"""Size-independent properties of H|psi> at the full benchmark sizes (GPU).

The oracle finishes in seconds only on small cells; at the 216-atom Gamma
cell (135^3 grid, 80 725 plane waves, 216 x 8 projectors) H is checked for
Hermiticity, <phi|H psi> = conj(<psi|H phi>), and linearity,
H(a psi + b phi) = a H psi + b H phi, in both forms, and the mixed form
against the FP64 form.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cell216(cuda_device):
    import torch

    from qe_python_b200.basis import LocalPotentialWorkspace, fft_shape, make_bases
    from qe_python_b200.pseudo_tables import SpeciesTables
    from qe_python_b200.scf import benchmark_system, projector_terms
    from qe_python_b200.symmetry import fft_factors

    system = benchmark_system("scf-dia216")
    basis = make_bases(system.reciprocal, system.kpoints, system.ecutwfc)[0]
    shape = fft_shape([basis], system.reciprocal, system.ecutrho, fft_factors(system.operations))
    tables = {l: SpeciesTables(p, system.volume) for l, p in system.pseudos.items()}
    terms = projector_terms(system, tables, basis)
    rng = np.random.default_rng(216)
    potential = torch.from_numpy(rng.uniform(-1.0, 0.5, shape)).cuda()
    return basis, shape, terms, potential, rng


def _ham(cell, precision):
    from qe_python_b200.basis import LocalPotentialWorkspace
    from qe_python_b200.diagonalization import PlaneWaveHamiltonian

    basis, shape, terms, potential, _ = cell
    ws = LocalPotentialWorkspace(basis, shape, precision=precision)
    return PlaneWaveHamiltonian(basis, None, terms, local_workspace=ws, real_potential=potential,
                                potential_average=0.0)


@pytest.mark.parametrize("precision,tol", [("f64", 1e-12), ("f32", 2e-6)])
def test_hermitian_and_linear_at_216_atoms(cell216, precision, tol):
    import torch

    from qe_python_b200.device import to_device_f

    basis, shape, _, _, rng = cell216
    assert shape == (135, 135, 135) and len(basis) == 80725
    ham = _ham(cell216, precision)
    npw = len(basis)
    damp = np.exp(-basis.kinetic / 20.0)[:, None]
    x = (rng.standard_normal((npw, 6)) + 1j * rng.standard_normal((npw, 6))) * damp
    v = to_device_f(x, ham.dtype, ham.device)
    hv = ham.apply(v).to(torch.complex128)
    v64 = v.to(torch.complex128)
    m = (v64.conj().T @ hv).cpu().numpy()  # <v_i|H v_j>
    scale = np.max(np.abs(m))
    assert np.max(np.abs(m - m.conj().T)) <= tol * scale
    a, b = 0.3 - 0.7j, -1.1 + 0.2j
    combo = to_device_f(a * x[:, :3] + b * x[:, 3:], ham.dtype, ham.device)
    lhs = ham.apply(combo).to(torch.complex128)
    rhs = a * hv[:, :3] + b * hv[:, 3:]
    assert float((lhs - rhs).abs().max()) <= 10 * tol * float(hv.abs().max())


def test_mixed_matches_fp64_at_216_atoms(cell216):
    import torch

    from qe_python_b200.device import to_device_f

    basis, _, _, _, rng = cell216
    npw = len(basis)
    damp = np.exp(-basis.kinetic / 20.0)[:, None]
    x = ((rng.standard_normal((npw, 4)) + 1j * rng.standard_normal((npw, 4))) * damp)
    x = x.astype(np.complex64).astype(np.complex128)  # representable in both forms
    h64 = _ham(cell216, "f64").apply(to_device_f(x, torch.complex128))
    h32 = _ham(cell216, "f32").apply(to_device_f(x, torch.complex64)).to(torch.complex128)
    err = float((h32 - h64).abs().max()) / float(h64.abs().max())
    assert err < 2e-6
