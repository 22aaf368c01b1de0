"""Pin the CPU oracle against the reference's own known answers (CPU only).

* The reference's recorded Si regression (tests/qe_reference/reference/
  pw_scf/scf.in.out: E = -16.87457024 Ry) is reproduced by the reference's
  pure-Python SCF driver running on the oracle native module (needs the
  reference tree; skipped where it is absent).
* The convolution identity of tests/unit/core/test_basis.py:76-88.
* The reference's PlaneWaveHamiltonian output (golden fixture generated by
  tests/golden/make_golden.py) equals the oracle's restated composition.
* apply_serial and apply_serial_spatial agree (two factorisations).
"""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from oracle import native_fft as oracle
from qe_python_b200.basis import grid_slots, potential_matrix
from tests.golden import reference_env

GOLDEN = Path(__file__).resolve().parent / "golden"


def _oracle_apply(miller, shape, psi, potential, kinetic):
    linear, *_ = grid_slots(miller, shape)
    size = int(np.prod(shape))
    grid = np.zeros((psi.shape[1], size), dtype=np.complex128)
    plan = oracle.NativeFFTWPlan(grid, shape, psi.shape[1], 1, size)
    out = np.zeros_like(psi)
    oracle.apply_serial(grid, psi, potential, linear, plan, size, size, out, 0, kinetic)
    return out


def test_oracle_convolution_identity():
    shape = (6, 6, 6)
    grid = np.indices(shape).sum(axis=0)
    potential_r = 0.3 + 0.2 * np.cos(2.0 * np.pi * grid / shape[0])
    potential_g = np.fft.fftn(potential_r) / np.prod(shape)
    indices = np.asarray([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0]], dtype=np.int32)
    coefficients = np.asarray([1.0 + 0.2j, -0.3j, 0.4, -0.1 + 0.5j])
    expected = potential_matrix(potential_g, indices) @ coefficients
    values = np.array(potential_g, dtype=np.complex128, order="C", copy=True)
    real = oracle.inverse_real(values, shape)
    got = _oracle_apply(indices, shape, coefficients[:, None], real, None)[:, 0]
    np.testing.assert_allclose(got, expected, atol=2.0e-14)


def test_oracle_reproduces_reference_hamiltonian_golden():
    g = np.load(GOLDEN / "hamiltonian_small.npz")
    shape = tuple(int(v) for v in g["shape"])
    psi = g["psi"]
    out = _oracle_apply(g["miller"], shape, psi, g["potential"], g["kinetic"])
    species, phases, coupling = g["species"], g["phases"], g["coupling"]
    for atom in range(phases.shape[1]):
        beta = np.asfortranarray(species * phases[:, [atom]])
        becp = oracle.projector_overlaps(beta, np.asfortranarray(psi))
        assert oracle.add_projector_product(out, beta, np.asfortranarray(coupling @ becp))
    for beta, cpl in ((g["packed_beta"], g["packed_coupling"]), (g["mat_beta"], g["mat_coupling"])):
        becp = oracle.projector_overlaps(np.asfortranarray(beta), np.asfortranarray(psi))
        assert oracle.add_projector_product(out, np.asfortranarray(beta), np.asfortranarray(cpl @ becp))
    expected = g["hpsi"]
    assert np.max(np.abs(out - expected)) <= 1e-12 * np.max(np.abs(expected))


def test_serial_and_spatial_factorisations_agree():
    g = np.load(GOLDEN / "hamiltonian_small.npz")
    shape = tuple(int(v) for v in g["shape"])
    psi = g["psi"][:, :3]
    serial = _oracle_apply(g["miller"], shape, psi, g["potential"], g["kinetic"])
    _l, zslots, positions, _s = grid_slots(g["miller"], shape)
    size = int(np.prod(shape))
    spatial = np.zeros_like(psi)
    oracle.apply_serial_spatial(np.zeros((3, size), complex), psi,
                                np.ascontiguousarray(np.moveaxis(g["potential"], 2, 0)), zslots,
                                positions, None, None, size, size, spatial, 0, g["kinetic"])
    assert np.max(np.abs(serial - spatial)) <= 1e-12 * np.max(np.abs(serial))


def test_hartree_metric_matches_direct_sum():
    rng = np.random.default_rng(3)
    residual = rng.standard_normal(500) + 1j * rng.standard_normal(500)
    g2 = np.concatenate(([0.0], rng.uniform(0.1, 9.0, 499)))
    direct = np.sum(4 * np.pi * np.abs(residual[1:]) ** 2 / g2[1:])
    assert abs(oracle.hartree_residual_metric(residual, g2) - direct) <= 1e-12 * direct


def test_qe_random_stream_is_deterministic():
    table = np.arange(97, dtype=np.int64) * 7351 % 714025
    a1, p1, c1, s1 = oracle.qe_random_pairs(5, 2, table.copy(), 11, 12345)
    a2, p2, c2, s2 = oracle.qe_random_pairs(5, 2, table.copy(), 11, 12345)
    np.testing.assert_array_equal(a1, a2)
    np.testing.assert_array_equal(p1, p2)
    assert (c1, s1) == (c2, s2)
    assert np.all((a1 >= 0) & (a1 < 1))


@pytest.mark.skipif(not (reference_env.reference_available() and reference_env.source_available()),
                    reason="the reference tree is only present in the build container")
def test_oracle_reproduces_reference_si_regression():
    from tests.golden.reference_env import SOURCE_ROOT, load_reference

    load_reference()
    from qepy_pw.input import read_pw_input
    from qepy_pw.scf import run_scf

    record = json.loads((GOLDEN / "si_regression.json").read_text())
    upstream = SOURCE_ROOT / "tests/qe_reference/upstream"
    pw = read_pw_input(upstream / "pw_scf" / "scf.in")
    pw.control["pseudo_dir"] = str(upstream / "pseudo")
    pw.control["disk_io"] = "none"
    result = run_scf(pw)
    energy_ry = 2.0 * result.iterations[-1].total_energy_ha
    assert abs(energy_ry - record["total_energy_ry"]) <= record["tolerance_ry"]
    bands_ev = [np.asarray(k) * 27.211386245988 for k in result.eigenvalues_ha]
    for got, want in zip(bands_ev, record["bands_ev"]):
        np.testing.assert_allclose(got, want, atol=1.0e-4)
