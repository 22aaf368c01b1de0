"""Host pieces of the analytic stress (qe_python_b200/stress.py).

* The Ewald stress is minus the homogeneous-strain derivative of the Ewald
  energy per volume, every tensor component (qepy_pw/ewald.py:49-143,
  261-365), checked by central differences of ``ewald_energy``.
* The radial and angular derivatives the local and nonlocal terms use:
  lagrange4_derivative, vloc_with_derivative and projectors_with_gradient
  against central differences of lagrange4, vloc and projectors
  (qepy_pw/upf.py:224-261, 558-597, 880-914).
* symmetrize_stress projects onto tensors that every operation of the
  space group leaves unchanged (qepy_pw/symmetry.py:1006-1027).
The terms themselves are compared with the reference's stress fixtures on
the GPU (tests/test_stress_gpu.py).
"""

from __future__ import annotations

import numpy as np
import pytest

from qe_python_b200.pseudo import synthetic_pseudo
from qe_python_b200.pseudo_tables import (
    SpeciesTables,
    ewald_energy,
    lagrange4,
    lagrange4_derivative,
)
from qe_python_b200.scf import benchmark_system
from qe_python_b200.stress import ewald_stress, symmetrize_stress


def _strained(lattice, positions, strain):
    deformation = np.eye(3) + strain
    return lattice @ deformation, positions @ deformation


def test_ewald_stress_is_the_strain_derivative_of_the_energy():
    system = benchmark_system("scf-dia8-disp")
    lattice, positions = system.lattice, system.positions
    charges = np.full(len(positions), 4.0)
    ecut = 40.0
    stress = ewald_stress(lattice, positions, charges, ecut, _sphere(lattice, ecut))
    volume = abs(np.linalg.det(lattice))
    step = 2.0e-5
    for i in range(3):
        for j in range(i, 3):
            strain = np.zeros((3, 3))
            strain[i, j] += 0.5 * step
            strain[j, i] += 0.5 * step
            plus = ewald_energy(*_strained(lattice, positions, strain), charges, ecut)
            minus = ewald_energy(*_strained(lattice, positions, -strain), charges, ecut)
            derivative = (plus - minus) / (2.0 * step)
            assert -derivative / volume == pytest.approx(stress[i, j], abs=3.0e-8), (i, j)
    np.testing.assert_allclose(stress, stress.T, atol=1e-15)


def _sphere(lattice, ecut_ry):
    """G vectors with |G|^2 <= ecutrho (the Ewald energy's own set)."""
    reciprocal = 2.0 * np.pi * np.linalg.inv(lattice).T
    bound = int(np.ceil(np.sqrt(ecut_ry) / np.linalg.svd(reciprocal, compute_uv=False)[-1])) + 1
    axis = np.arange(-bound, bound + 1)
    cube = np.stack(np.meshgrid(axis, axis, axis, indexing="ij"), axis=-1).reshape(-1, 3)
    g = cube @ reciprocal
    return g[np.einsum("ij,ij->i", g, g) <= ecut_ry + 1e-12]


def test_lagrange4_derivative_matches_central_differences():
    rng = np.random.default_rng(2)
    table = rng.standard_normal((400, 2))
    q = rng.uniform(0.05, 3.5, 200)
    # stay inside one interpolation interval for the difference
    q = 0.01 * (np.floor(q / 0.01) + rng.uniform(0.2, 0.8, q.size))
    h = 1.0e-7
    numeric = (lagrange4(table, q + h) - lagrange4(table, q - h)) / (2.0 * h)
    np.testing.assert_allclose(lagrange4_derivative(table, q), numeric, rtol=0, atol=2e-6)


def test_vloc_and_projector_gradients_match_central_differences():
    tables = SpeciesTables(synthetic_pseudo("X"), 1079.0)
    rng = np.random.default_rng(3)
    q = 0.01 * (np.floor(rng.uniform(0.2, 6.0, 100) / 0.01) + 0.5)
    h = 1.0e-6
    values, derivative = tables.vloc_with_derivative(q)
    np.testing.assert_array_equal(values, tables.vloc(q))
    numeric = (tables.vloc(q + h) - tables.vloc(q - h)) / (2.0 * h)
    np.testing.assert_allclose(derivative, numeric, rtol=1e-6, atol=1e-9)
    kg = rng.uniform(-3.0, 3.0, (60, 3))
    beta, coupling, gradient = tables.projectors_with_gradient(kg)
    beta0, coupling0 = tables.projectors(kg)
    np.testing.assert_array_equal(beta, beta0)
    np.testing.assert_array_equal(coupling, coupling0)
    for axis in range(3):
        step = np.zeros(3)
        step[axis] = h
        plus, _ = tables.projectors(kg + step)
        minus, _ = tables.projectors(kg - step)
        numeric = (plus - minus) / (2.0 * h)
        np.testing.assert_allclose(gradient[:, :, axis], numeric, rtol=0,
                                   atol=2e-6 * np.max(np.abs(beta)))


@pytest.mark.parametrize("name", ["scf-fcc2", "scf-dia64"])
def test_symmetrized_stress_is_invariant_under_the_point_group(name):
    system = benchmark_system(name)
    rng = np.random.default_rng(4)
    raw = rng.standard_normal((3, 3))
    raw = 0.5 * (raw + raw.T)
    sym = symmetrize_stress(raw, system.lattice, system.operations)
    inverse = np.linalg.inv(system.lattice)
    for op in system.operations:
        rotation = inverse @ np.asarray(op.matrix, dtype=float) @ system.lattice
        np.testing.assert_allclose(rotation.T @ sym @ rotation, sym, atol=1e-14)
    np.testing.assert_allclose(symmetrize_stress(sym, system.lattice, system.operations), sym,
                               atol=1e-15)
