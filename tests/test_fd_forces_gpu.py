"""Forces and the band-energy adjoint against finite differences of the
reference's total energy (the adjoint-forces configuration: 8-atom displaced
diamond cell, ecutwfc 25 Ry, 3x3x3 mesh, 24 bands).

tests/golden/fd_forces_dia8.json holds the reference's own SCF total
energies (qepy_pw/pw/scf.py:1968, conv_thr 1e-10 Ry) with one atom
coordinate moved by +-1e-3 bohr, for four coordinates, and their central
differences F_FD = -(E+ - E-)/2h (made by tests/golden/make_golden.py).

* The plain FP64 SCF on the GPU reproduces every one of those energies
  within 1e-8 Ry, so its own energy differences equal the reference's
  within 1e-5 Ry/bohr.
* Forces: the reference's Hellmann-Feynman forces (tests/golden/
  scf_dia8_disp.json) differ from its own F_FD by up to 5.7e-4 Ry/bohr on
  this cell: the exchange-correlation energy is evaluated on the real-space
  FFT grid, which is not invariant under a translation of the atoms, and
  the Hellmann-Feynman force omits that grid term.  So the check of the
  GPU forces against F_FD is |F - F_FD| <= |F_ref - F_FD| + 1e-4 Ry/bohr
  (1e-4 Ry/bohr being the bar of the chosen form), for the SCF forces in
  both forms and for the hand-written adjoint (-dE_band/dtau from
  BandEnergy's backward at the converged V_Hxc, plus the Ewald force) in
  both forms; the forces themselves equal the reference's within 1e-8
  Ry/bohr (FP64) and 1e-4 Ry/bohr (mixed) in tests/test_scf_gpu.py.
"""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
BAR = 1.0e-4  # Ry/bohr


def _golden():
    return json.loads((GOLDEN / "fd_forces_dia8.json").read_text())


def _reference_forces():
    return np.asarray(json.loads((GOLDEN / "scf_dia8_disp.json").read_text())
                      ["forces_ry_per_bohr"])


def _check(forces, label):
    record, reference = _golden(), _reference_forces()
    for entry in record["entries"]:
        a, x, fd = entry["atom"], entry["axis"], entry["force_ry_per_bohr"]
        allowed = abs(reference[a, x] - fd) + BAR
        assert abs(forces[a, x] - fd) <= allowed, (label, entry, forces[a, x], allowed)


def test_displaced_energies_match_reference(cuda_device):
    from qe_python_b200.scf import benchmark_system, run_scf

    record = _golden()
    for entry in record["entries"][:2]:
        energies = {}
        for sign in (+1, -1):
            system = benchmark_system("scf-dia8-disp")
            system.conv_thr = record["conv_thr_ry"]
            system.forces = False
            system.positions = system.positions.copy()
            system.positions[entry["atom"], entry["axis"]] += sign * record["step_bohr"]
            result = run_scf(system, precision="f64")
            assert result.converged
            energies[sign] = result.total_energy_ry
        assert abs(energies[+1] - entry["energy_plus_ry"]) <= 1e-8
        assert abs(energies[-1] - entry["energy_minus_ry"]) <= 1e-8
        fd = -(energies[+1] - energies[-1]) / (2.0 * record["step_bohr"])
        assert abs(fd - entry["force_ry_per_bohr"]) <= 1e-5


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_scf_forces_against_reference_energy_differences(cuda_device, precision):
    from qe_python_b200.scf import benchmark_system, run_scf

    result = run_scf(benchmark_system("scf-dia8-disp"), precision=precision)
    assert result.converged
    _check(2.0 * np.asarray(result.forces_ha_per_bohr), precision)


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_adjoint_forces_against_reference_energy_differences(cuda_device, precision):
    import torch

    from qe_python_b200.adjoint import BandEnergy, BandProblem
    from qe_python_b200.forces import ewald_forces
    from qe_python_b200.scf import benchmark_system, run_scf

    system = benchmark_system("scf-dia8-disp")
    scf = run_scf(system, precision="f64")
    assert scf.converged
    problem = BandProblem(benchmark_system("scf-dia8-disp"), precision=precision,
                          tolerance=1e-10)
    v_ion, _ = problem.v_ion(system.positions)
    v = torch.from_numpy(scf.potential.cpu().numpy() - v_ion).cuda().requires_grad_(True)
    tau = torch.from_numpy(system.positions.copy()).cuda().requires_grad_(True)
    BandEnergy.apply(v, tau, problem).backward()
    charges = np.array([system.pseudos[l].z_valence for l in system.labels])
    ewald = ewald_forces(system.lattice, system.positions, charges, system.ecutrho,
                         problem.grid.vectors)
    forces = 2.0 * (-tau.grad.cpu().numpy() + ewald)
    # the adjoint's forces are the SCF's Hellmann-Feynman forces before the
    # mean is removed (up to that constant per axis), from the density of a
    # fresh solve at the converged potential instead of the SCF's last one
    hf = 2.0 * np.asarray(scf.forces_ha_per_bohr)
    drift = forces - hf
    assert np.max(np.abs(drift - drift.mean(axis=0))) < (1e-5 if precision == "f64" else BAR)
    _check(forces, "adjoint " + precision)
