"""Forces and the band-energy adjoint against finite differences of the
reference's total energy (the adjoint-forces configuration: 8-atom displaced
diamond cell, ecutwfc 25 Ry, 3x3x3 mesh, 24 bands).

tests/golden/fd_forces_dia8.json holds the reference's own SCF total
energies (qepy_pw/pw/scf.py:1968, conv_thr 1e-10 Ry) with one atom
coordinate moved by +-1e-3 bohr, for four coordinates, and their central
differences -(E+ - E-)/2h (made by tests/golden/make_golden.py).  Checked
against them, within 1e-4 Ry/bohr:
  * the SCF's Hellmann-Feynman forces (local, nonlocal, Ewald) in the plain
    FP64 form and in the chosen form;
  * the hand-written adjoint: -dE_band/dtau from BandEnergy's backward at
    the converged V_Hxc (its local and nonlocal projector derivatives),
    plus the Ewald force, in FP64 and in the mixed form.
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


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_scf_forces_match_reference_energy_differences(cuda_device, precision):
    from qe_python_b200.scf import benchmark_system, run_scf

    record = _golden()
    result = run_scf(benchmark_system("scf-dia8-disp"), precision=precision)
    assert result.converged
    forces = 2.0 * np.asarray(result.forces_ha_per_bohr)
    for entry in record["entries"]:
        got = forces[entry["atom"], entry["axis"]]
        assert abs(got - entry["force_ry_per_bohr"]) < BAR, (precision, entry, got)


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_adjoint_forces_match_reference_energy_differences(cuda_device, precision):
    import torch

    from qe_python_b200.adjoint import BandEnergy, BandProblem
    from qe_python_b200.forces import ewald_forces
    from qe_python_b200.scf import benchmark_system, run_scf

    record = _golden()
    system = benchmark_system("scf-dia8-disp")
    scf = run_scf(system, precision="f64")
    assert scf.converged
    problem = BandProblem(benchmark_system("scf-dia8-disp"), precision=precision,
                          tolerance=1e-10)
    v_ion, _ = problem.v_ion(system.positions)
    v_hxc = scf.potential.cpu().numpy() - v_ion
    v = torch.from_numpy(v_hxc).cuda().requires_grad_(True)
    tau = torch.from_numpy(system.positions.copy()).cuda().requires_grad_(True)
    BandEnergy.apply(v, tau, problem).backward()
    charges = np.array([system.pseudos[l].z_valence for l in system.labels])
    ewald = ewald_forces(system.lattice, system.positions, charges, system.ecutrho,
                         problem.grid.vectors)
    forces = 2.0 * (-tau.grad.cpu().numpy() + ewald)
    for entry in record["entries"]:
        got = forces[entry["atom"], entry["axis"]]
        assert abs(got - entry["force_ry_per_bohr"]) < BAR, (precision, entry, got)
