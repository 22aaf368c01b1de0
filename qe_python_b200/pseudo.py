"""Synthetic norm-conserving pseudopotential (UPF v2) of the benchmark cells.

Z_val = 4 with
  V_loc(r) = -2 Z erf(r/0.8)/r - 3 exp(-(r/1.0)^2)        [Ry]
(the long-range tail -2Z/r in Ry, as the reference's V_loc(G) removes
-Z erf(r)/r in Hartree: qepy_pw/upf.py:162-222), and one s and one p
Kleinman-Bylander projector beta_l(r) = r^l exp(-r^2/1.2) with
D = diag(2.0, 1.0) Ry.  No PP_PSWFC and no PP_RHOATOM: the SCF starts from a
uniform density and random wavefunctions (qepy_pw/pw/scf.py:1004-1012,
853-870).  The file is read by the reference's ``read_upf``
(qepy_pw/upf.py:953-1094) and by ``read_synthetic_upf`` below.
"""

from __future__ import annotations

import math
import xml.etree.ElementTree as ET
from dataclasses import dataclass
from pathlib import Path

import numpy as np

Z_VALENCE = 4.0
ERF_WIDTH = 0.8
WELL_DEPTH_RY = 3.0
WELL_WIDTH = 1.0
BETA_WIDTH = 1.2
D_RY = (2.0, 1.0)
# QE-style logarithmic mesh r_i = exp(xmin + i dx) / Z
MESH_XMIN = -7.0
MESH_DX = 0.0125
MESH_SIZE = 1101


@dataclass(frozen=True)
class SyntheticPseudo:
    element: str
    z_valence: float
    r: np.ndarray
    rab: np.ndarray
    vloc_ry: np.ndarray
    betas: tuple[np.ndarray, ...]       # r * beta_l(r) as stored in PP_BETA
    angular_momenta: tuple[int, ...]
    cutoff_indices: tuple[int, ...]
    dij_ry: np.ndarray
    functional: str = "SLA PZ NOGX NOGC"


def radial_mesh() -> tuple[np.ndarray, np.ndarray]:
    i = np.arange(MESH_SIZE, dtype=float)
    r = np.exp(MESH_XMIN + i * MESH_DX) / Z_VALENCE
    return r, r * MESH_DX


def _erf(values: np.ndarray) -> np.ndarray:
    return np.array([math.erf(v) for v in values])


def synthetic_pseudo(element: str = "X") -> SyntheticPseudo:
    r, rab = radial_mesh()
    vloc = -2.0 * Z_VALENCE * _erf(r / ERF_WIDTH) / r - WELL_DEPTH_RY * np.exp(-(r / WELL_WIDTH) ** 2)
    betas, lvals, cutoffs = [], [], []
    for l in (0, 1):
        beta = r**l * np.exp(-(r**2) / BETA_WIDTH)
        stored = r * beta
        # first mesh index beyond which |r beta| < 1e-14
        significant = np.flatnonzero(np.abs(stored) > 1.0e-14)
        cutoff = int(significant[-1] + 2) if significant.size else MESH_SIZE
        cutoff = min(cutoff + (cutoff % 2 == 0), MESH_SIZE)
        stored = np.where(np.arange(MESH_SIZE) < cutoff, stored, 0.0)
        betas.append(stored)
        lvals.append(l)
        cutoffs.append(cutoff)
    return SyntheticPseudo(element, Z_VALENCE, r, rab, vloc, tuple(betas), tuple(lvals),
                           tuple(cutoffs), np.diag(D_RY))


def _fmt(values: np.ndarray) -> str:
    lines = []
    for start in range(0, len(values), 4):
        lines.append(" ".join(f"{v: .16E}" for v in values[start:start + 4]))
    return "\n" + "\n".join(lines) + "\n"


def write_synthetic_upf(path: str | Path, element: str = "X") -> Path:
    """Write the synthetic pseudopotential as a UPF v2 file."""
    pseudo = synthetic_pseudo(element)
    path = Path(path)
    n = len(pseudo.r)
    root = ET.Element("UPF", version="2.0.1")
    ET.SubElement(root, "PP_INFO").text = "synthetic benchmark pseudopotential (seed-free, analytic)"
    ET.SubElement(root, "PP_HEADER", {
        "generated": "qe_python_b200.pseudo", "element": element, "pseudo_type": "NC",
        "relativistic": "scalar", "is_ultrasoft": "F", "is_paw": "F", "is_coulomb": "F",
        "has_so": "F", "core_correction": "F", "functional": pseudo.functional,
        "z_valence": f"{pseudo.z_valence:.6f}", "l_max": "1", "mesh_size": str(n),
        "number_of_wfc": "0", "number_of_proj": str(len(pseudo.betas)),
    })
    mesh = ET.SubElement(root, "PP_MESH", {"mesh": str(n)})
    ET.SubElement(mesh, "PP_R", {"type": "real", "size": str(n)}).text = _fmt(pseudo.r)
    ET.SubElement(mesh, "PP_RAB", {"type": "real", "size": str(n)}).text = _fmt(pseudo.rab)
    ET.SubElement(root, "PP_LOCAL", {"type": "real", "size": str(n)}).text = _fmt(pseudo.vloc_ry)
    nonlocal_ = ET.SubElement(root, "PP_NONLOCAL")
    for index, (beta, l, cutoff) in enumerate(
            zip(pseudo.betas, pseudo.angular_momenta, pseudo.cutoff_indices), start=1):
        ET.SubElement(nonlocal_, f"PP_BETA.{index}", {
            "type": "real", "size": str(n), "index": str(index), "label": f"beta-{index}",
            "angular_momentum": str(l), "cutoff_radius_index": str(cutoff),
        }).text = _fmt(beta)
    ET.SubElement(nonlocal_, "PP_DIJ", {"type": "real", "size": str(pseudo.dij_ry.size)}).text = \
        _fmt(pseudo.dij_ry.reshape(-1))
    path.write_text(ET.tostring(root, encoding="unicode"))
    return path


def read_synthetic_upf(path: str | Path) -> SyntheticPseudo:
    """Parse the subset of UPF v2 the SCF driver uses (NC, no NLCC)."""
    root = ET.fromstring(Path(path).read_text())
    header = {k.lower(): v for k, v in root.find(".//PP_HEADER").attrib.items()}

    def numbers(node):
        return np.array(node.text.replace("D", "E").split(), dtype=float)

    r = numbers(root.find(".//PP_R"))
    rab = numbers(root.find(".//PP_RAB"))
    vloc = numbers(root.find(".//PP_LOCAL"))
    betas, lvals, cutoffs = [], [], []
    elements = [e for e in root.find(".//PP_NONLOCAL") if e.tag.upper().startswith("PP_BETA")]
    elements.sort(key=lambda e: int(e.attrib.get("index", "0")))
    for e in elements:
        betas.append(numbers(e))
        lvals.append(int(e.attrib["angular_momentum"]))
        cut = int(e.attrib.get("cutoff_radius_index", str(len(r))))
        cutoffs.append(len(r) if cut <= 1 or cut > len(r) else cut)
    nproj = len(betas)
    dij = numbers(root.find(".//PP_DIJ")).reshape(nproj, nproj) if nproj else np.zeros((0, 0))
    return SyntheticPseudo(header.get("element", "X"), float(header["z_valence"]), r, rab, vloc,
                           tuple(betas), tuple(lvals), tuple(cutoffs), dij,
                           header.get("functional", "unknown"))
