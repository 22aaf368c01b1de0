"""SCF set-up pieces against reference values (CPU only).

Golden: tests/golden/setup_tables.npz (reference V_loc(q), projector
columns, Ewald energy/forces and PZ81 for the synthetic pseudopotential),
index_maps.json (reference k points and weights of each benchmark cell) and
scf_*.json energy terms.
"""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from qe_python_b200.forces import ewald_forces
from qe_python_b200.pseudo import read_synthetic_upf, synthetic_pseudo, write_synthetic_upf
from qe_python_b200.pseudo_tables import SpeciesTables, ewald_energy, pz81
from qe_python_b200.scf import BroydenMixer, ChargeGrid, LinearMixer, QERandom, benchmark_system, neumaier_metric

GOLDEN = Path(__file__).resolve().parent / "golden"
T = np.load(GOLDEN / "setup_tables.npz")
MAPS = json.loads((GOLDEN / "index_maps.json").read_text())


def test_upf_round_trip(tmp_path):
    path = write_synthetic_upf(tmp_path / "X.upf")
    back = read_synthetic_upf(path)
    direct = synthetic_pseudo()
    np.testing.assert_array_equal(back.r, direct.r)
    np.testing.assert_array_equal(back.vloc_ry, direct.vloc_ry)
    assert back.angular_momenta == (0, 1)
    np.testing.assert_array_equal(back.dij_ry, np.diag([2.0, 1.0]))


def test_local_potential_table_matches_reference(tmp_path):
    pseudo = read_synthetic_upf(write_synthetic_upf(tmp_path / "X.upf"))
    got = SpeciesTables(pseudo, float(T["volume"])).vloc(T["q"])
    np.testing.assert_allclose(got, T["vloc"], rtol=1e-13, atol=1e-15)


def test_projector_basis_matches_reference(tmp_path):
    pseudo = read_synthetic_upf(write_synthetic_upf(tmp_path / "X.upf"))
    beta, coupling = SpeciesTables(pseudo, float(T["volume"])).projectors(T["kg"])
    np.testing.assert_allclose(beta, T["beta"], rtol=1e-13, atol=1e-15)
    np.testing.assert_array_equal(coupling, T["coupling"])


def test_ewald_matches_reference():
    charges = np.full(8, 4.0)
    e = ewald_energy(T["lattice"], T["positions"], charges, 100.0)
    assert abs(e - float(T["ewald_energy"])) < 1e-12
    system = benchmark_system("scf-dia8-disp")
    from qe_python_b200.basis import fft_shape, make_bases
    from qe_python_b200.symmetry import fft_factors

    bases = make_bases(system.reciprocal, system.kpoints, system.ecutwfc)
    grid = ChargeGrid(fft_shape(bases, system.reciprocal, 100.0, fft_factors(system.operations)),
                      system.reciprocal, 100.0)
    # the reference's default G set for ewald_forces is the full cutoff sphere;
    # the SCF passes the charge sphere of the FFT grid, identical here
    f = ewald_forces(T["lattice"], T["positions"], charges, 100.0, grid.vectors)
    np.testing.assert_allclose(f, T["ewald_forces"], atol=1e-12)


def test_ewald_term_of_reference_scf():
    ref = json.loads((GOLDEN / "scf_fcc2.json").read_text())
    s = benchmark_system("scf-fcc2")
    e = ewald_energy(s.lattice, s.positions, np.full(2, 4.0), s.ecutrho)
    assert abs(2.0 * e - ref["energy_terms_ry"]["ewald_ha"]) < 1e-12


def test_pz81_matches_reference():
    eps, v = pz81(T["rho"])
    np.testing.assert_allclose(eps, T["eps"], rtol=1e-14, atol=1e-300)
    np.testing.assert_allclose(v, T["vxc"], rtol=1e-14, atol=1e-300)


@pytest.mark.parametrize("name", ["scf-fcc2", "scf-dia64", "scf-dia8-disp"])
def test_kpoints_match_reference(name):
    s = benchmark_system(name)
    np.testing.assert_allclose(s.kpoints, MAPS[name]["kpoints"], atol=1e-12)
    np.testing.assert_allclose(s.weights, MAPS[name]["weights"], atol=1e-14)


def test_qe_random_stream_matches_oracle():
    from oracle import native_fft as oracle

    a = QERandom()
    table, cur, seed = a.table.copy(), a.current, a.seed
    f1, s1 = a.pairs(7, 3)
    f2, s2, c2, sd2 = oracle.qe_random_pairs(7, 3, table, cur, seed)
    np.testing.assert_array_equal(f1, f2)
    np.testing.assert_array_equal(s1, s2)
    assert (a.current, a.seed) == (c2, sd2)


def test_qe_random_integer_draws_match_pairs():
    """The int32 stream values divided by 714025 are the double pairs, and
    the stream state advances the same way, across several calls and a
    draw longer than the 97-entry table."""
    a, b = QERandom(), QERandom()
    for npw, bands in ((7, 3), (1, 1), (0, 4), (300, 5)):
        f1, s1 = a.pairs(npw, bands)
        f2, s2 = b.draws(npw, bands)
        assert f2.dtype == np.int32 and f2.flags.f_contiguous and f2.shape == (npw, bands)
        np.testing.assert_array_equal(f1, f2 / 714025.0)
        np.testing.assert_array_equal(s1, s2 / 714025.0)
        assert (a.current, a.seed) == (b.current, b.seed)
        np.testing.assert_array_equal(a.table, b.table)


def test_starting_draws_follow_one_stream_in_kpoint_order():
    """StartingDraws draws every k point in order on its thread; a pool
    keeps only its own k points, and the values equal a sequential draw."""
    from qe_python_b200.scf import StartingDraws

    sizes, bands = [50, 37, 64], 4
    serial = QERandom()
    expected = [serial.draws(n, bands) for n in sizes]
    everything = StartingDraws(QERandom(), sizes, bands)
    for k in range(3):
        got = everything.take(k)
        np.testing.assert_array_equal(got[0], expected[k][0])
        np.testing.assert_array_equal(got[1], expected[k][1])
    with pytest.raises(RuntimeError, match="already taken"):
        everything.take(0)
    pool = StartingDraws(QERandom(), sizes, bands, keep=[1])
    np.testing.assert_array_equal(pool.take(1)[1], expected[1][1])
    with pytest.raises(RuntimeError, match="not kept"):
        pool.take(2)


def test_starting_draws_report_a_failed_draw():
    from qe_python_b200.scf import StartingDraws

    broken = QERandom()
    broken.current = 714025  # outside the stream's range: the host routine refuses it
    draws = StartingDraws(broken, [10, 10], 2)
    with pytest.raises(RuntimeError, match="random starting draws failed"):
        draws.take(1)


def test_mixers_reduce_to_linear_on_first_step():
    s = benchmark_system("scf-fcc2")
    grid = ChargeGrid((24, 24, 24), s.reciprocal, s.ecutrho)
    rng = np.random.default_rng(1)
    rho_in = 0.1 + 0.01 * rng.random((24, 24, 24))
    rho_out = 0.1 + 0.01 * rng.random((24, 24, 24))
    # band-limit both densities to the charge sphere
    rho_in = grid.to_r(grid.to_g(rho_in))
    rho_out = grid.to_r(grid.to_g(rho_out))
    linear = LinearMixer(0.7).mix(rho_in, rho_out)
    broyden = BroydenMixer(grid, 0.7, 8, s.ecutrho).mix(rho_in, grid.to_g(rho_out - rho_in))
    # Broyden keeps rho(G=0) of the input; linear keeps the same because both
    # densities carry the same electron count after band limiting
    np.testing.assert_allclose(broyden - broyden.mean(), linear - linear.mean(), atol=1e-12)


def test_neumaier_metric():
    rng = np.random.default_rng(0)
    r = rng.standard_normal(1000) + 1j * rng.standard_normal(1000)
    g2 = np.concatenate(([0.0], rng.uniform(0.5, 5.0, 999)))
    assert abs(neumaier_metric(r, g2) - np.sum(4 * np.pi * np.abs(r[1:]) ** 2 / g2[1:])) < 1e-10
