"""Generate the golden fixtures of tests/golden/ from the reference.

Runs in the build container only: imports the reference qepy-pw package
(QEPY_REFERENCE_ROOT, default the read-only mount) with the NumPy oracle as
its native module (reference_env.py) and records its outputs:

  index_maps.json       per benchmark cell: k points, weights, FFT grid,
                        plane waves per k and SHA-256 of every basis' Miller
                        array and of the shared catalog (bit-exact pins)
  index_maps_fcc2.npz   full Miller arrays and serial slot maps of scf-fcc2
  hamiltonian_small.npz reference PlaneWaveHamiltonian.apply on a small cell
                        (factorized, packed and materialised projector terms)
  davidson_small.npz    reference davidson on the same operator
  scf_fcc2.json         reference SCF of scf-fcc2 (energy, bands, iterations)
  scf_dia8_disp.json    reference SCF + forces of scf-dia8-disp
  si_regression.json    the reference's own recorded Si regression numbers
                        (tests/qe_reference/reference/pw_scf/scf.in.out)

Usage: python tests/golden/make_golden.py [--skip-scf]
"""

from __future__ import annotations

import argparse
import hashlib
import json
import re
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))

from tests.golden.reference_env import SOURCE_ROOT, load_reference  # noqa: E402


def sha(array: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(array, dtype=np.int32).tobytes()).hexdigest()


def read_config(name: str, workdir: Path):
    from qepy_pw.input import read_pw_input

    from qe_python_b200.configs import ELECTRON_OVERRIDES, config_input
    from qe_python_b200.pseudo import write_synthetic_upf

    write_synthetic_upf(workdir / "X.upf")
    path = workdir / f"{name}.in"
    path.write_text(config_input(name, str(workdir)))
    pw = read_pw_input(path)
    pw.electrons.update(ELECTRON_OVERRIDES.get(name, {}))
    return pw


def index_maps(workdir: Path) -> None:
    from qepy_pw.basis import LocalPotentialWorkspace, fft_shape, make_bases
    from qepy_pw.symmetry import fft_factors

    from qe_python_b200.configs import CONFIGS
    from qe_python_b200.workloads import hpsi_microbench

    out = {}
    for name in CONFIGS:
        pw = read_config(name, workdir)
        kpoints = np.array([p.crystal for p in pw.kpoints])
        weights = np.array([p.weight for p in pw.kpoints])
        ecut = float(pw.system["ecutwfc"])
        ecutrho = float(pw.system.get("ecutrho", 4.0 * ecut))
        bases = make_bases(pw.reciprocal, kpoints, ecut)
        factors = fft_factors(pw.symmetry_operations,
                              use_all_frac=bool(pw.system.get("use_all_frac", False)))
        shape = fft_shape(bases, pw.reciprocal, ecutrho, factors)
        out[name] = {
            "reciprocal": pw.reciprocal.tolist(),
            "kpoints": kpoints.tolist(), "weights": weights.tolist(),
            "ecutwfc": ecut, "ecutrho": ecutrho, "fft_factors": list(map(int, factors)),
            "fft_shape": list(map(int, shape)), "npw": [len(b) for b in bases],
            "miller_sha256": [sha(b.indices) for b in bases],
            "catalog_sha256": sha(bases[0].catalog.indices),
        }
        if name == "scf-fcc2":
            ws = LocalPotentialWorkspace(bases[0], shape, retain_serial_sticks=True)
            np.savez_compressed(
                HERE / "index_maps_fcc2.npz",
                miller=np.concatenate([b.indices for b in bases]),
                offsets=np.cumsum([0] + [len(b) for b in bases]),
                linear_slots=ws.linear_slots, z_major_slots=ws.z_major_slots,
                stick_positions=ws.serial_stick_positions, sticks=ws.sticks,
            )
        print(f"{name}: {len(bases)} k, grid {shape}, npw {[len(b) for b in bases][:4]}...")
    work = hpsi_microbench(nbands=1)
    from qepy_pw.basis import make_bases as ref_make_bases

    basis = ref_make_bases(work.reciprocal, np.zeros(3), 30.0)[0]
    shape = fft_shape([basis], work.reciprocal, 150.0)
    out["hpsi-microbench"] = {
        "reciprocal": work.reciprocal.tolist(), "kpoints": [[0.0, 0.0, 0.0]], "weights": [2.0],
        "ecutwfc": 30.0, "ecutrho": 150.0, "fft_factors": [1, 1, 1],
        "fft_shape": list(map(int, shape)), "npw": [len(basis)],
        "miller_sha256": [sha(basis.indices)], "catalog_sha256": sha(basis.catalog.indices),
    }
    (HERE / "index_maps.json").write_text(json.dumps(out, indent=1))


def small_operator():
    """A small fcc cell with all three projector term kinds (seeded)."""
    from qepy_pw.basis import fft_shape, make_bases

    lattice = 10.26 / 2.0 * np.array([[-1.0, 0.0, 1.0], [0.0, 1.0, 1.0], [-1.0, 1.0, 0.0]])
    reciprocal = 2.0 * np.pi * np.linalg.inv(lattice).T
    k = np.array([0.125, 0.375, -0.25])
    basis = make_bases(reciprocal, k, 20.0)[0].materialize()
    shape = fft_shape([basis], reciprocal, 80.0)
    rng = np.random.default_rng(20261203)
    npw = len(basis)
    decay = 0.05 * np.exp(-basis.kinetic / 3.0)[:, None]
    species = np.asfortranarray((rng.standard_normal((npw, 4)) + 1j * rng.standard_normal((npw, 4))) * decay)
    positions = rng.uniform(0.0, 5.0, (3, 3))
    phases = np.asfortranarray(np.exp(-1j * basis.vectors @ positions.T))
    d = rng.uniform(-1.0, 1.0, (4, 4))
    coupling = 0.5 * (d + d.T)
    packed_beta = np.asfortranarray((rng.standard_normal((npw, 6)) + 1j * rng.standard_normal((npw, 6))) * decay)
    d6 = rng.uniform(-1.0, 1.0, (6, 6))
    packed_coupling = 0.5 * (d6 + d6.T)
    packed_diag = np.real(np.einsum("gi,ij,gj->g", packed_beta, packed_coupling, packed_beta.conj()))
    mat_beta = np.asfortranarray((rng.standard_normal((npw, 2)) + 1j * rng.standard_normal((npw, 2))) * decay)
    mat_coupling = np.array([[0.7, 0.1], [0.1, -0.4]])
    potential = np.ascontiguousarray(rng.uniform(-0.6, 0.6, shape))
    psi = np.asfortranarray(rng.standard_normal((npw, 6)) + 1j * rng.standard_normal((npw, 6)))
    return dict(reciprocal=reciprocal, k=k, ecut=20.0, shape=np.array(shape), miller=basis.indices,
                kinetic=basis.kinetic, species=species, phases=phases, coupling=coupling,
                packed_beta=packed_beta, packed_coupling=packed_coupling, packed_diag=packed_diag,
                mat_beta=mat_beta, mat_coupling=mat_coupling, potential=potential, psi=psi)


def hamiltonian_and_davidson() -> None:
    from qepy_pw.basis import LocalPotentialWorkspace, PlaneWaveBasis
    from qepy_pw.diagonalization import (
        FactorizedProjectorTerm,
        PackedProjectorTerm,
        PlaneWaveHamiltonian,
        davidson,
    )

    s = small_operator()
    basis = PlaneWaveBasis(s["miller"], None, s["kinetic"])
    object.__setattr__(basis, "_legacy_vectors", np.zeros((len(s["miller"]), 3)))
    shape = tuple(int(v) for v in s["shape"])
    ws = LocalPotentialWorkspace(s["miller"], shape)
    terms = (
        FactorizedProjectorTerm(s["species"], s["phases"], s["coupling"]),
        PackedProjectorTerm(s["packed_beta"], s["packed_coupling"], s["packed_diag"]),
        (s["mat_beta"], s["mat_coupling"]),
    )
    h = PlaneWaveHamiltonian(basis, np.zeros(shape, dtype=complex), terms, local_workspace=ws,
                             real_potential=s["potential"], potential_average=0.125)
    hpsi = h.apply(s["psi"])
    diagonal = h.diagonal
    rng = np.random.default_rng(7)
    start = np.asfortranarray(rng.standard_normal((len(basis), 8)) + 1j * rng.standard_normal((len(basis), 8)))
    result = davidson(h.apply, diagonal, 8, initial_vectors=start, tolerance=1e-9,
                      max_iterations=100, subspace_multiplier=2, residual_factor=None,
                      operator_into=h.apply_into)
    np.savez_compressed(HERE / "hamiltonian_small.npz", hpsi=hpsi, diagonal=diagonal, **s)
    np.savez_compressed(HERE / "davidson_small.npz", start=start,
                        eigenvalues=result.eigenvalues, iterations=result.iterations,
                        converged=result.converged,
                        applications=result.hamiltonian_applications)
    print("davidson:", result.iterations, result.converged, result.eigenvalues[:3])


def scf(name: str, workdir: Path, filename: str) -> None:
    from qepy_pw.scf import run_scf

    pw = read_config(name, workdir)
    started = time.perf_counter()
    result = run_scf(pw)
    elapsed = time.perf_counter() - started
    record = {
        "config": name,
        "total_energy_ry": 2.0 * float(result.iterations[-1].total_energy_ha),
        "iterations": len(result.iterations),
        "energies_ry": [2.0 * float(it.total_energy_ha) for it in result.iterations],
        "estimated_accuracy_ry": [2.0 * float(it.estimated_accuracy_ha) for it in result.iterations],
        "davidson_thresholds_ha": [float(it.davidson_threshold_ha) for it in result.iterations],
        "average_davidson_iterations": [float(it.average_diagonalization_iterations)
                                        for it in result.iterations],
        "eigenvalues_ry": [[2.0 * float(e) for e in k] for k in result.eigenvalues_ha],
        "energy_terms_ry": {k: 2.0 * float(v) for k, v in vars(result.energy_terms).items()},
        "forces_ry_per_bohr": None if result.forces_ha_per_bohr is None
        else (2.0 * np.asarray(result.forces_ha_per_bohr)).tolist(),
        "fermi_energy_ry": None if getattr(result, "fermi_energy_ha", None) is None
        else 2.0 * float(result.fermi_energy_ha),
        "reference_wall_seconds": elapsed,
        "reference_runner": "reference Python + NumPy oracle native module, 1 process",
    }
    (HERE / filename).write_text(json.dumps(record, indent=1))
    print(f"{name}: E = {record['total_energy_ry']:.10f} Ry in {elapsed:.1f} s, "
          f"{record['iterations']} iterations")


def setup_tables(workdir: Path) -> None:
    """Reference V_loc(q), projector columns, Ewald energies/forces and PZ81
    values for the synthetic pseudopotential (setup_tables.npz)."""
    from qepy_pw.ewald import ewald_energy, ewald_forces
    from qepy_pw.upf import read_upf
    from qepy_pw.xc import pz81_unpolarized

    from qe_python_b200.configs import DIAMOND_CUBIC, displacements
    from qe_python_b200.pseudo import write_synthetic_upf

    write_synthetic_upf(workdir / "X.upf")
    pseudo = read_upf(workdir / "X.upf")
    volume = 270.0
    q = np.linspace(0.0, 13.0, 1500)
    rng = np.random.default_rng(11)
    kg = rng.normal(size=(400, 3)) * 3.0
    beta, coupling = pseudo.projector_basis(kg, volume)
    rho = 10.0 ** rng.uniform(-12.0, 1.0, 4000)
    eps, vxc = pz81_unpolarized(rho)
    a = 10.26
    lattice = np.eye(3) * a
    positions = DIAMOND_CUBIC * a + displacements(8, 0.05)
    charges = np.full(8, 4.0)
    np.savez_compressed(
        HERE / "setup_tables.npz", volume=volume, q=q, vloc=pseudo.fourier(q, volume), kg=kg,
        beta=beta, coupling=coupling, rho=rho, eps=eps, vxc=vxc, lattice=lattice,
        positions=positions, ewald_energy=ewald_energy(lattice, positions, charges, 100.0),
        ewald_forces=ewald_forces(lattice, positions, charges, 100.0))


def smearing_tables() -> None:
    """Reference Fermi levels, occupations and smearing energies for seeded
    eigenvalue sets and every broadening order (smearing.json)."""
    from qepy_pw.occupations import smeared_occupations, w1gauss, wgauss

    rng = np.random.default_rng(5)
    cases = []
    for order in (0, 1, -1, -99):
        for degauss in (0.005, 0.02):
            nk = 3
            eigenvalues = [np.sort(rng.uniform(-0.5, 0.6, 10)) for _ in range(nk)]
            weights = rng.uniform(0.5, 1.5, nk)
            weights /= weights.sum()
            nelec = 11.0
            fermi, occ, demet = smeared_occupations(eigenvalues, weights, nelec, degauss, order)
            cases.append({"order": order, "degauss_ha": degauss, "nelec": nelec,
                          "eigenvalues_ha": [e.tolist() for e in eigenvalues],
                          "weights": weights.tolist(), "fermi_ha": fermi,
                          "occupations": [o.tolist() for o in occ], "demet_ha": demet})
    x = np.linspace(-8.0, 8.0, 161)
    functions = {str(order): {"wgauss": wgauss(x, order).tolist(), "w1gauss": w1gauss(x, order).tolist()}
                 for order in (0, 1, 2, -1, -99)}
    record = {"source": "qepy_pw/occupations.py smeared_occupations, wgauss, w1gauss",
              "x": x.tolist(), "functions": functions, "cases": cases}
    (HERE / "smearing.json").write_text(json.dumps(record))
    print("smearing: %d cases" % len(cases))


def mixer_tables() -> None:
    """The reference SCF's Broyden mixer (DistributedBroydenMixer on the
    charge-sphere coefficients, qepy_pw/pw/scf.py:3027-3041) in 'plain' and
    'TF' modes over seven steps of seeded densities on a 9^3 grid of the
    2-atom fcc cell, sphere |G|^2 <= 20 (broyden.npz)."""
    from qepy_pw.basis import LocalPotentialWorkspace as RefWorkspace
    from qepy_pw.mixing import DistributedBroydenMixer

    from qe_python_b200.scf import ChargeGrid

    lattice = 10.26 / 2.0 * np.array([[-1.0, 0.0, 1.0], [0.0, 1.0, 1.0], [-1.0, 1.0, 0.0]])
    reciprocal = 2.0 * np.pi * np.linalg.inv(lattice).T
    volume = abs(np.linalg.det(lattice))
    shape = (9, 9, 9)
    grid = ChargeGrid(shape, reciprocal, 20.0)
    rng = np.random.default_rng(8)
    outs = 0.05 + 0.02 * rng.random((7, *shape))
    start = 0.05 + 0.02 * rng.random(shape)
    record = {"shape": np.array(shape), "lattice": lattice, "start": start, "outs": outs}
    for mode in ("plain", "TF"):
        workspace = RefWorkspace(grid.miller, shape)
        mixer = DistributedBroydenMixer(workspace, grid.g2, beta=0.7, ndim=4, g2_cutoff=20.0,
                                        mode=mode, nelec=8.0, volume=volume)
        rho, seq = start.copy(), []
        for out in outs:
            rho = mixer.mix(rho, out)
            seq.append(rho.copy())
        record[f"mixed_{mode}"] = np.array(seq)
    np.savez_compressed(HERE / "broyden.npz", **record)
    print("broyden: plain and TF sequences")


class _Captured(Exception):
    """Raised by the capturing Davidson stand-in once every k point's
    first-iteration Hamiltonian has been built."""


def _c_order_potential(ham) -> np.ndarray:
    """The reference Hamiltonian's real V_eff(r) as a C-order (nx, ny, nz) grid."""
    v = np.asarray(ham.real_potential, dtype=np.float64)
    shape = tuple(int(s) for s in ham.local_workspace.shape)
    if ham.native_potential_layout:  # (nz, nx, ny) native layout
        v = v.reshape(shape[2], shape[0], shape[1]).transpose(1, 2, 0)
    return np.ascontiguousarray(v.reshape(shape))


def potential_checksums(v: np.ndarray, seed: int) -> dict:
    """Size-independent fingerprints of a real grid: sum, sum of squares and
    the dot product with a seeded uniform field."""
    field = np.random.default_rng(seed).uniform(-1.0, 1.0, v.shape)
    return {"sum": float(np.sum(v)), "sum_sq": float(np.sum(v * v)),
            "probe": float(np.sum(v * field))}


def probe_vectors(npw: int, count: int, seed: int, kinetic: np.ndarray) -> np.ndarray:
    """Seeded complex Gaussian columns scaled by exp(-T_G/10) (the test
    draws the same columns with the same generator)."""
    rng = np.random.default_rng(seed)
    psi = rng.standard_normal((npw, count)) + 1j * rng.standard_normal((npw, count))
    return np.asfortranarray(psi * np.exp(-np.asarray(kinetic) / 10.0)[:, None])


def first_iteration(name: str, workdir: Path, filename: str, roots: int,
                    tolerance: float = 1.0e-9) -> None:
    """The reference's first-SCF-iteration Hamiltonian of every k point of a
    benchmark cell (starting V_eff from the uniform density, the reference's
    own projector construction qepy_pw/pw/scf.py:596-718, its
    PlaneWaveHamiltonian qepy_pw/diagonalization.py:124-368), captured at
    its Davidson call site (qepy_pw/pw/scf.py:3510) and then:
      * fingerprints of V_eff(r) and of the preconditioner diagonal,
      * <psi|H|psi> and <w|H|psi> of seeded probe columns,
      * the lowest ``roots`` eigenvalues by the reference's davidson from its
        default start (unit vectors on the lowest plane waves), converged to
        ``tolerance`` Ha (tight, so path independent).
    The run stops once every k point's operator is captured; the starting
    subspace and rotate_wfc are skipped (they play no part here)."""
    import qepy_pw.pw.scf as ref_scf
    from qepy_pw.diagonalization import DavidsonResult, davidson
    from qepy_pw.scf import run_scf

    pw = read_config(name, workdir)
    nk = len(pw.kpoints)
    captured = []

    def capture(operator, diagonal, number, **options):
        captured.append(operator.__self__)
        if len(captured) == nk:
            raise _Captured
        start = options["initial_vectors"]
        return DavidsonResult(np.zeros(number), np.asfortranarray(start[:, :number]),
                              np.zeros(number), 1, True, 0, 0)

    def cheap_orbitals(pw_, pseudos, basis, bands, **_kw):
        out = np.zeros((len(basis), bands), dtype=np.complex128, order="F")
        out[np.arange(bands), np.arange(bands)] = 1.0
        return out

    def no_rotation(operator, trials, bands, mpi=None):
        return np.asfortranarray(trials[:, :bands]), np.zeros(bands), None

    saved = (ref_scf.davidson, ref_scf._atomic_starting_orbitals,
             ref_scf._rotate_starting_subspace)
    ref_scf.davidson = capture
    ref_scf._atomic_starting_orbitals = cheap_orbitals
    ref_scf._rotate_starting_subspace = no_rotation
    started = time.perf_counter()
    try:
        run_scf(pw)
    except _Captured:
        pass
    finally:
        (ref_scf.davidson, ref_scf._atomic_starting_orbitals,
         ref_scf._rotate_starting_subspace) = saved
    print(f"{name}: captured {len(captured)} operators in {time.perf_counter() - started:.1f} s")
    record = {"config": name, "roots": roots, "davidson_tolerance_ha": tolerance,
              "probe_seed": 20261203, "probe_columns": 4, "kpoints": []}
    for k, ham in enumerate(captured):
        basis = ham.basis
        v = _c_order_potential(ham)
        diagonal = np.asarray(ham.diagonal)
        psi = probe_vectors(len(basis), 4, 20261203 + k, basis.kinetic)
        probes = probe_vectors(len(basis), 4, 20261303 + k, np.zeros(len(basis)))
        hpsi = ham.apply(psi)
        quad = psi.conj().T @ hpsi
        cross = probes.conj().T @ hpsi
        t0 = time.perf_counter()
        solution = davidson(ham.apply, diagonal, roots, tolerance=tolerance, max_iterations=400,
                            subspace_multiplier=4, residual_factor=None,
                            operator_into=ham.apply_into)
        print(f"  k {k}: npw {len(basis)} davidson {solution.iterations} its "
              f"converged {solution.converged} in {time.perf_counter() - t0:.1f} s; "
              f"lowest {solution.eigenvalues[:3]}")
        record["kpoints"].append({
            "npw": len(basis),
            "miller_sha256": sha(basis.indices),
            "potential": potential_checksums(v, 7),
            "potential_average": float(ham.potential_average),
            "diagonal": {"sum": float(np.sum(diagonal)),
                         "sum_sq": float(np.sum(diagonal * diagonal)),
                         "max": float(np.max(diagonal))},
            "hpsi_norms": np.linalg.norm(hpsi, axis=0).tolist(),
            "psi_h_psi": {"re": quad.real.tolist(), "im": quad.imag.tolist()},
            "probe_h_psi": {"re": cross.real.tolist(), "im": cross.imag.tolist()},
            "eigenvalues_ha": np.asarray(solution.eigenvalues).tolist(),
            "davidson_converged": bool(solution.converged),
            "davidson_iterations": float(solution.iterations),
        })
    record["reference_wall_seconds"] = time.perf_counter() - started
    record["reference_runner"] = "reference Python + NumPy oracle native module, 1 process"
    (HERE / filename).write_text(json.dumps(record, indent=1))


def displaced_energies(workdir: Path, filename: str, coordinates, step: float) -> None:
    """Reference total energies of scf-dia8-disp with one atom coordinate
    moved by +-``step`` bohr (central differences of E_tot give the force
    on that coordinate), conv_thr tightened to 1e-10 Ry so the energy error
    stays well below step x 1e-4 Ry/bohr."""
    from qepy_pw.pw.input import read_pw_input
    from qepy_pw.scf import run_scf

    from qe_python_b200.configs import config_input
    from qe_python_b200.pseudo import write_synthetic_upf

    write_synthetic_upf(workdir / "X.upf")
    base = config_input("scf-dia8-disp", str(workdir))
    record = {"config": "scf-dia8-disp", "step_bohr": step, "conv_thr_ry": 1.0e-10,
              "entries": []}
    for atom, axis in coordinates:
        energies = {}
        for sign in (+1, -1):
            text = _displace(base, atom, axis, sign * step)
            text = text.replace("conv_thr = 1e-08", "conv_thr = 1e-10")
            path = workdir / f"disp_{atom}_{axis}_{sign}.in"
            path.write_text(text)
            pw = read_pw_input(path)
            t0 = time.perf_counter()
            result = run_scf(pw)
            energies[sign] = 2.0 * float(result.iterations[-1].total_energy_ha)
            print(f"atom {atom} axis {axis} sign {sign:+d}: E = {energies[sign]:.10f} Ry "
                  f"({len(result.iterations)} its, {time.perf_counter() - t0:.1f} s)")
        record["entries"].append({
            "atom": atom, "axis": axis, "energy_plus_ry": energies[+1],
            "energy_minus_ry": energies[-1],
            "force_ry_per_bohr": -(energies[+1] - energies[-1]) / (2.0 * step)})
        (HERE / filename).write_text(json.dumps(record, indent=1))


def stress(name: str, workdir: Path, filename: str) -> None:
    """The reference's analytic stress (tstress) at SCF convergence and its
    seven terms, Ha/bohr^3 (qepy_pw/pw/scf.py:1676-1931, ewald.py:261)."""
    from qepy_pw.pw.input import read_pw_input
    from qepy_pw.scf import run_scf

    from qe_python_b200.configs import ELECTRON_OVERRIDES, config_input
    from qe_python_b200.pseudo import write_synthetic_upf

    write_synthetic_upf(workdir / "X.upf")
    text = config_input(name, str(workdir))
    text = text.replace("disk_io = 'none'", "disk_io = 'none',\n  tstress = .true.", 1)
    text = text.replace("conv_thr = 1e-08", "conv_thr = 1e-10")
    path = workdir / f"{name}-stress.in"
    path.write_text(text)
    pw = read_pw_input(path)
    pw.electrons.update({k: v for k, v in ELECTRON_OVERRIDES.get(name, {}).items()
                         if k != "conv_thr"})
    started = time.perf_counter()
    result = run_scf(pw)
    elapsed = time.perf_counter() - started
    terms = result.stress_terms
    record = {
        "config": name, "conv_thr_ry": 1.0e-10,
        "total_energy_ry": 2.0 * float(result.iterations[-1].total_energy_ha),
        "stress_ha_per_bohr3": np.asarray(result.stress_ha_per_bohr3).tolist(),
        "terms_ha_per_bohr3": {field: np.asarray(getattr(terms, field)).tolist()
                               for field in ("kinetic_ha_per_bohr3", "local_ha_per_bohr3",
                                             "nonlocal_ha_per_bohr3", "hartree_ha_per_bohr3",
                                             "xc_ha_per_bohr3", "core_correction_ha_per_bohr3",
                                             "ewald_ha_per_bohr3")},
        "reference_wall_seconds": elapsed,
    }
    (HERE / filename).write_text(json.dumps(record, indent=1))
    print(f"{name}: stress (Ha/bohr^3) {record['stress_ha_per_bohr3']} in {elapsed:.1f} s")


def _displace(text: str, atom: int, axis: int, delta: float) -> str:
    """Move one atom of a pw.x input's ATOMIC_POSITIONS (bohr) block."""
    lines = text.splitlines()
    start = next(i for i, line in enumerate(lines) if line.startswith("ATOMIC_POSITIONS"))
    fields = lines[start + 1 + atom].split()
    values = [float(v) for v in fields[1:4]]
    values[axis] += delta
    lines[start + 1 + atom] = f"  {fields[0]} {values[0]:.12f} {values[1]:.12f} {values[2]:.12f}"
    return "\n".join(lines) + "\n"


def si_regression() -> None:
    path = SOURCE_ROOT / "tests/qe_reference/reference/pw_scf/scf.in.out"
    text = path.read_text()
    energy = float(re.search(r"!\s+total energy\s+=\s+(-?\d+\.\d+)\s+Ry", text).group(1))
    blocks = re.findall(r"k =.*?bands \(ev\):\s*\n\s*\n(.*?)\n\s*\n", text, flags=re.S)
    bands = [[float(v) for v in b.split()] for b in blocks]
    record = {"source": "tests/qe_reference/reference/pw_scf/scf.in.out",
              "input": "tests/qe_reference/upstream/pw_scf/scf.in",
              "total_energy_ry": energy, "bands_ev": bands,
              "tolerance_ry": 5.0e-8}
    (HERE / "si_regression.json").write_text(json.dumps(record, indent=1))
    print("si regression:", energy, bands)


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--skip-scf", action="store_true")
    parser.add_argument("--only", default=None,
                        help="comma-separated subset: first-iteration-dia64, "
                             "first-iteration-dia216, fd-forces, stress")
    args = parser.parse_args()
    load_reference()
    if args.only:
        with tempfile.TemporaryDirectory() as tmp:
            workdir = Path(tmp)
            for part in args.only.split(","):
                if part == "first-iteration-dia64":
                    first_iteration("scf-dia64", workdir, "first_iteration_dia64.json", 16)
                elif part == "first-iteration-dia216":
                    first_iteration("scf-dia216", workdir, "first_iteration_dia216.json", 20,
                                    tolerance=1.0e-8)
                elif part == "stress":
                    stress("scf-fcc2", workdir, "stress_fcc2.json")
                    stress("scf-dia8-disp", workdir, "stress_dia8.json")
                elif part == "fd-forces":
                    displaced_energies(workdir, "fd_forces_dia8.json",
                                       [(0, 0), (3, 1), (5, 2), (6, 0)], 1.0e-3)
                else:
                    raise SystemExit(f"unknown part {part!r}")
        return
    with tempfile.TemporaryDirectory() as tmp:
        workdir = Path(tmp)
        index_maps(workdir)
        hamiltonian_and_davidson()
        setup_tables(workdir)
        si_regression()
        smearing_tables()
        mixer_tables()
        if not args.skip_scf:
            scf("scf-fcc2", workdir, "scf_fcc2.json")
            scf("scf-fcc2-smear", workdir, "scf_fcc2_smear.json")
            scf("scf-dia8-disp", workdir, "scf_dia8_disp.json")


if __name__ == "__main__":
    main()
