"""Crystal symmetry for the SCF set-up: space group, k-point reduction,
FFT-grid factors and density symmetrisation.

Conventions follow the reference (qepy_pw/symmetry.py, pw/input.py):
fractional coordinates are row vectors, an operation (M, t) maps x to
x M + t, a k point (reciprocal crystal coordinates) maps to k M^{-T}.
  * space group: integer M with M G M^T = G (G = A A^T, rows of A the
    lattice vectors) that map the labelled basis onto itself for some t
  * Monkhorst-Pack mesh: ((i + s/2)/n) folded to [-1/2, 1/2)
    (qepy_pw/pw/input.py:953-985)
  * reduction: orbits under the mesh-compatible operations and time
    reversal, first mesh point of each orbit as representative, weights
    summed (qepy_pw/symmetry.py:856-925)
  * grid factors: lcm of the denominators of the fractional translations
    (qepy_pw/symmetry.py:623-645)
  * density: rho_sym(x) = mean over operations of rho(x M + t) on the FFT
    grid, then rescaled to the electron count.  rho(G) built from plane
    waves inside the wavefunction sphere lies inside the charge sphere, so
    this real-space average equals the reference's reciprocal star
    projection.
"""

from __future__ import annotations

import itertools
import math
from dataclasses import dataclass
from fractions import Fraction

import numpy as np


@dataclass(frozen=True)
class Operation:
    matrix: np.ndarray       # (3, 3) integer, row-vector convention
    translation: np.ndarray  # (3,) fractional


def _wrap(x: np.ndarray) -> np.ndarray:
    y = x - np.floor(x)
    y[np.isclose(y, 1.0, atol=1.0e-10)] = 0.0
    return y


def lattice_point_group(lattice: np.ndarray, tol: float = 1.0e-6) -> list[np.ndarray]:
    metric = lattice @ lattice.T
    found = []
    scale = max(1.0, float(np.max(np.abs(metric))))
    for entries in itertools.product((-1, 0, 1), repeat=9):
        m = np.array(entries, dtype=int).reshape(3, 3)
        if abs(round(np.linalg.det(m))) != 1:
            continue
        if np.max(np.abs(m @ metric @ m.T - metric)) <= tol * scale:
            found.append(m)
    # identity first, then the enumeration order
    found.sort(key=lambda m: 0 if np.array_equal(m, np.eye(3, dtype=int)) else 1)
    return found


def _crystallographic(t: np.ndarray, tol: float) -> bool:
    """QE accepts fractional translations whose components are 0 or
    +-1/2, 1/3, 1/4, 1/6 (qepy_pw/symmetry.py:672-691)."""
    for c in t - np.rint(t):
        mag = abs(float(c))
        if mag <= tol:
            continue
        inv = 1.0 / mag
        if round(inv) not in (2, 3, 4, 6) or abs(inv - round(inv)) > tol:
            return False
    return True


def space_group(lattice: np.ndarray, fractional: np.ndarray, labels: list[str],
                tol: float = 1.0e-5) -> list[Operation]:
    """Operations (M, t); for each lattice rotation the first atom (in input
    order) of the first atom's species that gives an admissible t is used."""
    fractional = np.asarray(fractional, dtype=float)
    labels = list(labels)
    ops = []
    for m in lattice_point_group(lattice):
        image = fractional @ m
        candidates = [np.array(fractional[j] - image[0])
                      for j in range(len(labels)) if labels[j] == labels[0]]
        for t in candidates:
            if not _crystallographic(t, tol):
                continue
            t = _wrap(t)
            moved = _wrap(image + t)
            ok = True
            for i, x in enumerate(moved):
                delta = fractional - x
                delta -= np.round(delta)
                hit = np.flatnonzero((np.abs(delta).max(axis=1) < tol)
                                     & (np.array(labels) == labels[i]))
                if hit.size != 1:
                    ok = False
                    break
            if ok:
                t = t.copy()
                t[np.abs(t) < tol] = 0.0
                ops.append(Operation(m, t))
                break
    return ops


def fft_factors(ops: list[Operation], tol: float = 1.0e-7) -> tuple[int, int, int]:
    factors = [1, 1, 1]
    for op in ops:
        for axis, value in enumerate(op.translation):
            reduced = float(value) % 1.0
            fraction = Fraction(reduced).limit_denominator(48)
            if abs(float(fraction) - reduced) <= tol:
                factors[axis] = math.lcm(factors[axis], fraction.denominator)
    return tuple(factors)


def monkhorst_pack(grid, shift) -> tuple[np.ndarray, np.ndarray]:
    points = []
    for i in range(grid[0]):
        for j in range(grid[1]):
            for k in range(grid[2]):
                f = np.array([(i + 0.5 * shift[0]) / grid[0], (j + 0.5 * shift[1]) / grid[1],
                              (k + 0.5 * shift[2]) / grid[2]])
                f -= np.floor(f + 0.5)
                points.append(f)
    points = np.array(points)
    return points, np.full(len(points), 1.0 / len(points))


def _keys(points: np.ndarray) -> list[tuple]:
    return [tuple(row) for row in np.round(_wrap(np.asarray(points, dtype=float)), 10)]


def mesh_compatible(points: np.ndarray, ops: list[Operation]) -> list[Operation]:
    keys = set(_keys(points))
    return [op for op in ops
            if all(k in keys for k in _keys(points @ np.linalg.inv(op.matrix).T))]


def reduce_kpoints(points: np.ndarray, weights: np.ndarray, ops: list[Operation],
                   time_reversal: bool = True):
    keys = _keys(points)
    lookup = {k: i for i, k in enumerate(keys)}
    if time_reversal:
        time_reversal = all(k in lookup for k in _keys(-points))
    maps = []
    for op in ops:
        moved = points @ np.linalg.inv(op.matrix).T
        for sign in ((1.0, -1.0) if time_reversal else (1.0,)):
            index = np.array([lookup.get(k, -1) for k in _keys(sign * moved)])
            if np.all(index >= 0):
                maps.append(index)
    assigned = np.zeros(len(points), dtype=bool)
    reps, wts = [], []
    mapping = np.full(len(points), -1, dtype=np.int32)
    for i in range(len(points)):
        if assigned[i]:
            continue
        orbit = {int(m[i]) for m in maps} or {i}
        orbit = sorted(orbit)
        assigned[orbit] = True
        mapping[orbit] = len(reps)
        reps.append(points[i].copy())
        wts.append(float(np.sum(weights[orbit])))
    return np.array(reps), np.array(wts), mapping


class DensitySymmetrizer:
    """Average a real-space density over the space-group operations.

    ``apply`` (host, NumPy) is the CPU restatement; ``apply_device`` runs the
    same average on the GPU (qeb_symmetrize_density, operations summed in
    the reference's order: qepy_pw/symmetry.py:178-238)."""

    def __init__(self, ops: list[Operation], shape) -> None:
        self.shape = tuple(int(v) for v in shape)
        n = np.array(self.shape)
        self.operations = list(ops)
        # integer terms of the transformed coordinates: axis b of op(i) is
        # (offset_b + sum_a coeff_ab i_a) mod n_b
        self.offsets = np.zeros((len(ops), 3), dtype=np.int32)
        self.coefficients = np.zeros((len(ops), 3, 3), dtype=np.int32)
        for index, op in enumerate(ops):
            offset = np.asarray(op.translation, dtype=float) * n
            scaled = np.asarray(op.matrix, dtype=float) * n[None, :] / n[:, None]
            if np.max(np.abs(offset - np.rint(offset))) > 1.0e-7 or \
                    np.max(np.abs(scaled - np.rint(scaled))) > 1.0e-7:
                raise ValueError("operation is not commensurate with the FFT grid")
            self.offsets[index] = np.rint(offset).astype(np.int32)
            self.coefficients[index] = np.rint(scaled).astype(np.int32)
        self.maps = None
        self.count = len(ops) if len(ops) > 1 else 1

    def _host_maps(self) -> list:
        if self.maps is not None:
            return self.maps
        n = np.array(self.shape)
        grid = np.indices(self.shape).reshape(3, -1).T  # integer grid coordinates
        self.maps = []
        for op in self.operations:
            if np.array_equal(op.matrix, np.eye(3, dtype=int)) and not np.any(op.translation):
                continue
            # x = i / n ; x' = x M + t ; i' = n * x'
            shifted = (grid / n) @ op.matrix + op.translation
            target = shifted * n
            rounded = np.round(target)
            if np.max(np.abs(target - rounded)) > 1.0e-6:
                raise ValueError("operation is not commensurate with the FFT grid")
            rounded = np.mod(rounded.astype(np.int64), n)
            self.maps.append(np.ravel_multi_index(rounded.T, self.shape))
        return self.maps

    def apply(self, density: np.ndarray) -> np.ndarray:
        """Host restatement: the identity adds the density itself, every
        other operation its permuted copy, in the operations' order."""
        if self.count == 1:
            return density
        flat = np.asarray(density, dtype=float).reshape(-1)
        total = np.zeros_like(flat)
        maps = iter(self._host_maps())
        for op in self.operations:
            if np.array_equal(op.matrix, np.eye(3, dtype=int)) and not np.any(op.translation):
                total += flat
            else:
                total += flat[next(maps)]
        return (total / self.count).reshape(self.shape)

    def apply_device(self, density):
        """The same average of a float64 CUDA tensor (C-order grid) on the GPU."""
        import torch

        from . import _lib
        from .device import stream_handle

        if self.count == 1:
            return density
        if tuple(density.shape) != self.shape or density.dtype != torch.float64:
            raise ValueError("density must be a float64 grid of the symmetrizer's shape")
        source = density.contiguous()
        out = torch.empty_like(source)
        offsets = np.ascontiguousarray(self.offsets)
        coefficients = np.ascontiguousarray(self.coefficients)
        _lib.check("qeb_symmetrize_density", _lib.load().qeb_symmetrize_density(
            *self.shape, len(self.operations), offsets.ctypes.data, coefficients.ctypes.data,
            source.data_ptr(), out.data_ptr(), stream_handle()))
        return out
