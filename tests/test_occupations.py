"""Broadened occupations against the reference's values (CPU only).

The fixture tests/golden/smearing.json holds the reference's wgauss, w1gauss
and smeared_occupations outputs (qepy_pw/occupations.py:610-908) for every
broadening order, generated by tests/golden/make_golden.py.
"""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from qe_python_b200.occupations import (
    fixed_occupations,
    smeared_occupations,
    smearing_order,
    w1gauss,
    wgauss,
)

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "smearing.json").read_text())


@pytest.mark.parametrize("order", [0, 1, 2, -1, -99])
def test_step_and_entropy_functions(order):
    x = np.asarray(GOLDEN["x"])
    ref = GOLDEN["functions"][str(order)]
    np.testing.assert_allclose(wgauss(x, order), ref["wgauss"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(w1gauss(x, order), ref["w1gauss"], rtol=0, atol=1e-15)


@pytest.mark.parametrize("case", range(len(GOLDEN["cases"])))
def test_fermi_level_occupations_and_demet(case):
    c = GOLDEN["cases"][case]
    eigenvalues = [np.asarray(e) for e in c["eigenvalues_ha"]]
    fermi, occ, demet = smeared_occupations(eigenvalues, np.asarray(c["weights"]), c["nelec"],
                                            c["degauss_ha"], c["order"])
    assert abs(fermi - c["fermi_ha"]) < 1e-11
    for mine, ref in zip(occ, c["occupations"]):
        np.testing.assert_allclose(mine, ref, rtol=0, atol=1e-10)
    assert abs(demet - c["demet_ha"]) < 1e-12
    total = sum(w * o.sum() for w, o in zip(np.asarray(c["weights"]) / np.sum(c["weights"]), occ))
    assert abs(total - c["nelec"]) < 1e-9


def test_names_and_fixed_filling():
    assert smearing_order("gaussian") == 0
    assert smearing_order("Marzari_Vanderbilt") == -1
    assert smearing_order("m-p") == 1
    assert smearing_order("fd") == -99
    with pytest.raises(ValueError):
        smearing_order("nonsense")
    occ = fixed_occupations(6, 4, 2)
    assert len(occ) == 2 and occ[1].tolist() == [2, 2, 2, 2, 0, 0]
    with pytest.raises(ValueError):
        smeared_occupations([np.zeros(2)], np.ones(1), 4.0, 0.01, 0)  # no empty states
