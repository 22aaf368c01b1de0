"""Seeded synthetic workloads for the H|psi> microbenchmark and parity tests.

The H|psi> microbenchmark cell: cubic L = 15.8 bohr, one k point (Gamma,
complex coefficients), ecutwfc 30 Ry (11 019 plane waves), ecutrho 150 Ry
(64^3 grid by the reference's grid rule), 256 bands.
  psi(G)  = (N(0,1) + i N(0,1)) exp(-|k+G|^2 / 20)
  V(r)    = sum over 64 seeded centres of a_i exp(-|r - R_i|^2 / 1 bohr^2),
            minimum image, a_i ~ U[-1, 1] Ha
  beta    = 64 atoms x 8 channels (s, p, p, s) with Gaussian radial form
            r^l exp(-r^2/1.2); per-atom real symmetric D ~ U[-2, 2] Ry,
            coupling = D/2 in Hartree (qepy_pw/upf.py:541-551).
The nonlocal operator is one materialised (beta, coupling) term with
P = 512 channels (qepy_pw/diagonalization.py:195-202, 312-326).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .basis import fft_shape, make_bases

SEED = 20261203


@dataclass
class HpsiWorkload:
    lattice: np.ndarray
    reciprocal: np.ndarray
    volume: float
    shape: tuple[int, int, int]
    miller: np.ndarray        # (npw, 3) int32
    vectors: np.ndarray       # (npw, 3) k+G, bohr^-1
    kinetic: np.ndarray       # (npw,) Hartree
    psi: np.ndarray           # (npw, nbands) complex128, F-order
    potential: np.ndarray     # (nx, ny, nz) float64, C-order, Hartree
    beta: np.ndarray          # (npw, P) complex128, F-order
    coupling: np.ndarray      # (P, P) float64, Hartree

    @property
    def npw(self) -> int:
        return self.miller.shape[0]

    @property
    def nbands(self) -> int:
        return self.psi.shape[1]


def _gaussian_radial(l: int, q: np.ndarray, a: float = 1.2) -> np.ndarray:
    """int_0^inf r^2 j_l(q r) r^l exp(-r^2/a) dr in closed form:
    sqrt(pi)/2^(l+2) a^(l+3/2) q^l exp(-q^2 a / 4)."""
    return np.sqrt(np.pi) / 2 ** (l + 2) * a ** (l + 1.5) * q**l * np.exp(-(q**2) * a / 4.0)


def _real_harmonics(l: int, unit: np.ndarray) -> np.ndarray:
    """QE ylmr2 ordering for l <= 1 (qepy_pw/_native_fft.pyx:1603-1661)."""
    if l == 0:
        return np.full((unit.shape[0], 1), 1.0 / np.sqrt(4.0 * np.pi))
    c = np.sqrt(3.0 / (4.0 * np.pi))
    return np.stack((c * unit[:, 2], -c * unit[:, 0], -c * unit[:, 1]), axis=1)


def _projectors(vectors, volume, positions, rng):
    q = np.sqrt(np.einsum("ij,ij->i", vectors, vectors))
    unit = np.zeros_like(vectors)
    nz = q > 1.0e-14
    unit[nz] = vectors[nz] / q[nz, None]
    unit[~nz] = (0.0, 0.0, 1.0)
    channels = []
    for l in (0, 1, 1, 0):
        radial = 4.0 * np.pi / np.sqrt(volume) * _gaussian_radial(l, q)
        angular = _real_harmonics(l, unit)
        channels.append(((-1j) ** l) * angular * radial[:, None])
    species_beta = np.concatenate(channels, axis=1)  # (npw, 8)
    per_atom = species_beta.shape[1]
    natoms = positions.shape[0]
    beta = np.empty((vectors.shape[0], natoms * per_atom), dtype=np.complex128, order="F")
    coupling = np.zeros((natoms * per_atom, natoms * per_atom))
    phases = np.exp(-1j * (vectors @ positions.T))
    for atom in range(natoms):
        block = slice(atom * per_atom, (atom + 1) * per_atom)
        beta[:, block] = species_beta * phases[:, atom, None]
        d = rng.uniform(-2.0, 2.0, (per_atom, per_atom))
        coupling[block, block] = 0.5 * 0.5 * (d + d.T)
    return beta, coupling


def hpsi_microbench(nbands: int = 256, seed: int = SEED, length: float = 15.8,
                    ecutwfc: float = 30.0, ecutrho: float = 150.0, natoms: int = 64,
                    ncentres: int = 64) -> HpsiWorkload:
    lattice = np.eye(3) * length
    reciprocal = 2.0 * np.pi * np.linalg.inv(lattice).T
    volume = float(abs(np.linalg.det(lattice)))
    basis = make_bases(reciprocal, np.zeros(3), ecutwfc)[0]
    shape = fft_shape([basis], reciprocal, ecutrho)
    miller = np.ascontiguousarray(basis.indices, dtype=np.int32)
    vectors = basis.vectors
    kinetic = basis.kinetic
    rng = np.random.default_rng(seed)
    g2 = np.einsum("ij,ij->i", vectors, vectors)
    psi = (rng.standard_normal((miller.shape[0], nbands))
           + 1j * rng.standard_normal((miller.shape[0], nbands)))
    psi = np.asfortranarray(psi * np.exp(-g2 / 20.0)[:, None])
    # smooth real potential from Gaussians of width 1 bohr (minimum image)
    centres = rng.uniform(0.0, length, (ncentres, 3))
    amplitudes = rng.uniform(-1.0, 1.0, ncentres)
    axes = [np.arange(n) * (length / n) for n in shape]
    gx, gy, gz = np.meshgrid(*axes, indexing="ij")
    potential = np.zeros(shape)
    for centre, amplitude in zip(centres, amplitudes):
        d2 = np.zeros(shape)
        for grid, c in zip((gx, gy, gz), centre):
            delta = grid - c
            delta -= length * np.round(delta / length)
            d2 += delta * delta
        potential += amplitude * np.exp(-d2)
    positions = rng.uniform(0.0, length, (natoms, 3))
    beta, coupling = _projectors(vectors, volume, positions, rng)
    return HpsiWorkload(lattice, reciprocal, volume, tuple(shape), miller, vectors, kinetic,
                        psi, np.ascontiguousarray(potential), beta, coupling)
