"""pw.x-style inputs of the benchmark cells (synthetic pseudopotential).

  scf-fcc2      2-atom diamond-structure fcc, a = 10.26 bohr, ecutwfc 20 / ecutrho
                80 Ry, 4x4x4 shifted Monkhorst-Pack mesh, 8 bands, linear mixing 0.7
  scf-fcc2-smear the same cell with Broyden mixing and Marzari-Vanderbilt
                smearing (degauss 0.02 Ry): the small pin of broadened filling
  scf-dia64     2x2x2 supercell of the 8-atom cubic diamond cell (a = 20.52),
                ecutwfc 30 / ecutrho 180 Ry, unshifted 2x2x2 mesh (4 k), 160 bands,
                Gaussian smearing 0.02 Ry, Thomas-Fermi mixing
  scf-dia8-disp 8-atom cubic diamond (a = 10.26), each atom displaced by a seeded
                uniform vector of length <= 0.05 bohr, ecutwfc 25 Ry, 3x3x3 mesh,
                24 bands, forces
  scf-dia216    3x3x3 supercell (a = 30.78), seeded 0.03-bohr displacements,
                ecutwfc 30 / ecutrho 180 Ry, Gamma only, 480 bands, forces,
                Gaussian smearing 0.02 Ry, Thomas-Fermi mixing
All converge to conv_thr = 1e-8 Ry.  The text is readable by the reference's
read_pw_input (qepy_pw/pw/input.py:1063).
"""

from __future__ import annotations

import numpy as np

SEED = 20261203

DIAMOND_CUBIC = np.array([
    [0.00, 0.00, 0.00], [0.50, 0.50, 0.00], [0.50, 0.00, 0.50], [0.00, 0.50, 0.50],
    [0.25, 0.25, 0.25], [0.75, 0.75, 0.25], [0.75, 0.25, 0.75], [0.25, 0.75, 0.75],
])


def supercell(frac: np.ndarray, n: int) -> np.ndarray:
    cells = [np.array([i, j, k]) for i in range(n) for j in range(n) for k in range(n)]
    return np.array([(site + cell) / n for cell in cells for site in frac])


def displacements(count: int, maximum: float, seed: int = SEED) -> np.ndarray:
    """Seeded vectors with uniform direction and length uniform in [0, maximum]."""
    rng = np.random.default_rng(seed)
    direction = rng.standard_normal((count, 3))
    direction /= np.linalg.norm(direction, axis=1)[:, None]
    return direction * rng.uniform(0.0, maximum, count)[:, None]


# The synthetic pseudopotential makes the diamond lattice a semimetal (the
# highest occupied band of the displaced 8-atom cell reaches 1.90 eV, the
# lowest empty one starts at 1.24 eV).  A supercell folds those k-points onto
# one another, and fixed filling of the lowest bands then swaps states at the
# Fermi level between iterations and never converges (the 216-atom Gamma cell
# was measured oscillating for 100 iterations).  The supercells therefore use
# Gaussian broadening, which the reference supports (qepy_pw/pw/scf.py:2146),
# and Thomas-Fermi-preconditioned Broyden mixing (mixing_mode 'TF',
# qepy_pw/mixing.py:51-59, 398-399) against long-wavelength charge sloshing,
# which plain Broyden from a uniform start does not damp in these cells.
SUPERCELL_SMEARING = {"occupations": "smearing", "smearing": "gaussian", "degauss": 0.02}
SUPERCELL_MIXING = {"mixing_mode": "TF"}


def _positions_block(unit: str, labels, positions) -> str:
    rows = "\n".join(f"  {lab} {p[0]:.12f} {p[1]:.12f} {p[2]:.12f}" for lab, p in zip(labels, positions))
    return f"ATOMIC_POSITIONS ({unit})\n{rows}\n"


def _namelists(system: dict, electrons: dict, control: dict) -> str:
    def block(name, values):
        body = ",\n".join(f"  {k} = {v}" for k, v in values.items())
        return f"&{name}\n{body}\n/\n"
    return block("control", control) + block("system", system) + block("electrons", electrons)


def _value(v):
    if isinstance(v, bool):
        return ".true." if v else ".false."
    if isinstance(v, str):
        return f"'{v}'"
    return repr(v)


def config_input(name: str, pseudo_dir: str, pseudo_file: str = "X.upf") -> str:
    control = {"calculation": "scf", "pseudo_dir": pseudo_dir, "disk_io": "none"}
    electrons = {"conv_thr": 1.0e-8, "diagonalization": "david"}
    if name == "scf-fcc2-smear":
        system = {"ibrav": 2, "celldm(1)": 10.26, "nat": 2, "ntyp": 1, "ecutwfc": 20.0,
                  "ecutrho": 80.0, "nbnd": 8, "occupations": "smearing",
                  "smearing": "marzari-vanderbilt", "degauss": 0.02}
        positions = _positions_block("alat", ["X", "X"], [[0, 0, 0], [0.25, 0.25, 0.25]])
        kpoints = "K_POINTS automatic\n 4 4 4 1 1 1\n"
    elif name == "scf-fcc2":
        system = {"ibrav": 2, "celldm(1)": 10.26, "nat": 2, "ntyp": 1, "ecutwfc": 20.0,
                  "ecutrho": 80.0, "nbnd": 8}
        # linear mixing is set programmatically (ELECTRON_OVERRIDES): the
        # reference's input reader accepts only plain/TF/local-TF in text.
        electrons.update({"mixing_beta": 0.7})
        positions = _positions_block("alat", ["X", "X"], [[0, 0, 0], [0.25, 0.25, 0.25]])
        kpoints = "K_POINTS automatic\n 4 4 4 1 1 1\n"
    elif name == "scf-dia64":
        frac = supercell(DIAMOND_CUBIC, 2)
        # Unshifted 2x2x2 mesh: under the cubic group it reduces to the four
        # points Gamma, X, M, R (weights 1:3:3:1) whose plane-wave counts
        # differ slightly; the shifted mesh would collapse to one point.
        system = {"ibrav": 1, "celldm(1)": 20.52, "nat": len(frac), "ntyp": 1, "ecutwfc": 30.0,
                  "ecutrho": 180.0, "nbnd": 160, **SUPERCELL_SMEARING}
        electrons.update(SUPERCELL_MIXING)
        positions = _positions_block("crystal", ["X"] * len(frac), frac)
        kpoints = "K_POINTS automatic\n 2 2 2 0 0 0\n"
    elif name == "scf-dia8-disp":
        a = 10.26
        cart = DIAMOND_CUBIC * a + displacements(8, 0.05)
        system = {"ibrav": 1, "celldm(1)": a, "nat": 8, "ntyp": 1, "ecutwfc": 25.0, "nbnd": 24}
        control["tprnfor"] = True
        positions = _positions_block("bohr", ["X"] * 8, cart)
        kpoints = "K_POINTS automatic\n 3 3 3 0 0 0\n"
    elif name == "scf-dia216":
        a = 30.78
        frac = supercell(DIAMOND_CUBIC, 3)
        cart = frac * a + displacements(len(frac), 0.03)
        system = {"ibrav": 1, "celldm(1)": a, "nat": len(frac), "ntyp": 1, "ecutwfc": 30.0,
                  "ecutrho": 180.0, "nbnd": 480, **SUPERCELL_SMEARING}
        electrons.update(SUPERCELL_MIXING)
        control["tprnfor"] = True
        positions = _positions_block("bohr", ["X"] * len(frac), cart)
        kpoints = "K_POINTS gamma\n"
    else:
        raise KeyError(f"unknown benchmark cell {name!r}")
    text = _namelists({k: _value(v) for k, v in system.items()},
                      {k: _value(v) for k, v in electrons.items()},
                      {k: _value(v) for k, v in control.items()})
    text += f"ATOMIC_SPECIES\n  X 12.0 {pseudo_file}\n" + positions + kpoints
    return text


CONFIGS = ("scf-fcc2", "scf-fcc2-smear", "scf-dia64", "scf-dia8-disp", "scf-dia216")

# ELECTRONS entries applied after parsing (qepy_pw/pw/scf.py:3042 'linear').
ELECTRON_OVERRIDES = {"scf-fcc2": {"mixing_mode": "linear"}}
