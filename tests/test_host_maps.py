"""Host index maps agree bit for bit with the reference (CPU only).

Golden data: tests/golden/index_maps.json (SHA-256 of every basis' Miller
array, FFT grids, k points of each benchmark cell, generated by the
reference's make_bases / fft_shape) and index_maps_fcc2.npz (full arrays and
serial slot maps of the 2-atom cell).
"""

from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from qe_python_b200.basis import (
    _next_fast_len_real,
    _qe_energy_order,
    fft_shape,
    grid_slots,
    make_bases,
)

GOLDEN = Path(__file__).resolve().parent / "golden"
MAPS = json.loads((GOLDEN / "index_maps.json").read_text())


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.int32).tobytes()).hexdigest()


@pytest.mark.parametrize("target,expected", [(0, 1), (1, 1), (7, 8), (11, 12), (17, 18), (31, 32),
                                             (133, 135), (89, 90)])
def test_fast_lengths(target, expected):
    assert _next_fast_len_real(target) == expected


@pytest.mark.parametrize("name", [n for n in MAPS if n != "scf-dia216"] + ["scf-dia216"])
def test_bases_and_grid_match_reference(name):
    ref = MAPS[name]
    reciprocal = np.asarray(ref["reciprocal"])
    bases = make_bases(reciprocal, np.asarray(ref["kpoints"]), ref["ecutwfc"])
    assert [len(b) for b in bases] == ref["npw"]
    assert [_sha(b.indices) for b in bases] == ref["miller_sha256"]
    assert _sha(bases[0].catalog.indices) == ref["catalog_sha256"]
    shape = fft_shape(bases, reciprocal, ref["ecutrho"], tuple(ref["fft_factors"]))
    assert list(shape) == ref["fft_shape"]


def test_fcc2_slot_maps_bit_exact():
    g = np.load(GOLDEN / "index_maps_fcc2.npz")
    ref = MAPS["scf-fcc2"]
    bases = make_bases(np.asarray(ref["reciprocal"]), np.asarray(ref["kpoints"]), ref["ecutwfc"])
    miller = np.concatenate([b.indices for b in bases])
    np.testing.assert_array_equal(miller, g["miller"])
    linear, zmajor, positions, sticks = grid_slots(bases[0].indices, tuple(ref["fft_shape"]))
    for mine, theirs in ((linear, g["linear_slots"]), (zmajor, g["z_major_slots"]),
                         (positions, g["stick_positions"]), (sticks, g["sticks"])):
        assert mine.dtype == theirs.dtype
        np.testing.assert_array_equal(mine, theirs)


def test_energy_order_keeps_degenerate_groups_in_input_order():
    values = np.array([1.0, 0.5, 0.5 + 4e-9, 0.5 - 4e-9, 2.0, 1.0 + 1e-9, 0.5 + 9e-9])
    order = _qe_energy_order(values)
    # group around 0.5 starts at 0.5-4e-9: members within 1e-8 of it keep index order
    assert list(order[:4]) == [1, 2, 3, 6]
    assert list(order[4:6]) == [0, 5]
    assert order[6] == 4


def test_energy_order_chain_longer_than_tolerance():
    # consecutive gaps below eps but the chain spans more than eps: a new
    # group starts once a value leaves eps of the group's first member
    values = np.array([0.0, 6e-9, 12e-9, 18e-9])[::-1].copy()
    order = _qe_energy_order(values)
    assert list(order) == [2, 3, 0, 1]


def test_empty_basis_raises():
    with pytest.raises(ValueError):
        # |k+G| >= 50 for every G at k = (1/2, 1/2, 1/2): nothing below 1e-3 Ry
        make_bases(np.eye(3) * 100.0, np.array([0.5, 0.5, 0.5]), 1e-3)


@pytest.mark.parametrize("length,ecutrho", [(10.26, 80.0), (15.8, 120.0), (7.3, 200.0)])
def test_charge_extent_equals_sorted_sphere(length, ecutrho):
    """fft_shape takes the extent of the k = 0 charge sphere without sorting
    it; the extent must equal that of the QE-ordered sphere make_bases builds."""
    from qe_python_b200.basis import _charge_extent, make_basis

    lattice = length / 2.0 * np.array([[-1.0, 0.0, 1.0], [0.0, 1.0, 1.0], [-1.0, 1.0, 0.0]])
    reciprocal = 2.0 * np.pi * np.linalg.inv(lattice).T
    sphere = make_basis(reciprocal, np.zeros(3), ecutrho)
    np.testing.assert_array_equal(_charge_extent(reciprocal, ecutrho),
                                  np.max(np.abs(sphere.indices), axis=0))


def _scan_energy_order(values, tolerance):
    """The ordering rule element by element (qepy_pw/basis.py:1588-1616): a
    stable ascending sort in which a group starts at the first value not
    within ``tolerance`` of the current group's first value, and each group
    keeps its incoming order."""
    keys = np.asarray(values, dtype=float)
    order = np.argsort(keys, kind="stable")
    ranked = keys[order]
    out, start = [], 0
    while start < len(order):
        stop = start + 1
        while stop < len(order) and abs(ranked[stop] - ranked[start]) < tolerance:
            stop += 1
        out.extend(sorted(order[start:stop]))
        start = stop
    return np.asarray(out, dtype=order.dtype)


def test_energy_order_groups_match_an_element_scan():
    from qe_python_b200.basis import _ORDER_EPS, _qe_energy_order

    rng = np.random.default_rng(5)
    for _ in range(300):
        n = int(rng.integers(1, 200))
        # chains of values whose gaps straddle the tolerance, so that a run
        # of near-equal neighbours splits into several groups
        values = (rng.integers(0, 12, n).astype(float)
                  + rng.choice([0.0, 0.4, 0.8, 1.2, 1.6, 3.0], n) * _ORDER_EPS)
        assert np.array_equal(_qe_energy_order(values), _scan_energy_order(values, _ORDER_EPS))
