"""Radial tables, structure-dependent set-up terms and the LDA functional.

Host-side set-up of the SCF (once per run or per k point), restated from the
reference so that the GPU Hamiltonian sees the same operator:
  * V_loc(|G|): dq = 0.01 table of the short-range part with the analytic
    -Z erf(r)/r tail restored, G = 0 "alpha Z" term (qepy_pw/upf.py:107-222)
  * beta_l(|k+G|): dq = 0.01 radial transform table, 4-point Lagrange
    interpolation, 4 pi / sqrt(Omega) normalisation (qepy_pw/upf.py:270-326)
  * projector columns (-i)^l Y_lm beta_l (qepy_pw/upf.py:483-556,
    _native_fft.pyx:1702-1791)
  * Ewald energy (qepy_pw/ewald.py:49-143, QE ewald.f90)
  * PZ81 LDA (Perdew-Zunger 1981 parametrisation of Ceperley-Alder,
    unpolarised; the reference's qepy_pw/xc.py:862-929).
Energies are in Hartree internally.
"""

from __future__ import annotations

import math

import numpy as np
import torch
from scipy.special import erf, erfc

DQ = 0.01


def qe_simpson(values: np.ndarray, rab: np.ndarray) -> np.ndarray:
    """QE simpsn on a radial mesh (qepy_pw/upf.py:917-943): weights 1,4,2,...,4,1
    times rab/3 along the last axis; an even-length mesh corrects the last
    three weights."""
    n = rab.size
    if n < 3 or values.shape[-1] != n:
        raise ValueError("Simpson integration needs matching arrays of length >= 3")
    w = np.zeros(n)
    w[0] = w[-1] = 1.0
    w[1:-1:2] = 4.0
    w[2:-1:2] = 2.0
    if n % 2 == 0:
        w[-3] -= 0.25
        w[-2] += 1.0
        w[-1] = 1.25
    return np.tensordot(values, rab * w / 3.0, axes=([-1], [0]))


def spherical_jn(l: int, x: np.ndarray) -> np.ndarray:
    """j_l(x) for l <= 1: power series for |x| < l + 1 (at least 1), closed
    form above, as the reference's special.spherical_jn does for these orders."""
    x = np.asarray(x, dtype=float)
    out = np.empty_like(x)
    small = np.abs(x) < max(1.0, float(l + 1))
    if np.any(small):
        xs = x[small]
        odd = 1.0
        for k in range(1, 2 * l + 2, 2):
            odd *= k
        term = xs**l / odd
        total = term.copy()
        for i in range(1, 80):
            term = term * (-xs * xs / (2.0 * i * (2.0 * l + 2.0 * i + 1.0)))
            total += term
            if np.all(np.abs(term) <= 2.0e-16 * (1.0 + np.abs(total))):
                break
        out[small] = total
    if np.any(~small):
        xl = x[~small]
        j0 = np.sin(xl) / xl
        out[~small] = j0 if l == 0 else j0 / xl - np.cos(xl) / xl
    if l > 1:
        raise ValueError("only l <= 1 projectors are used by the benchmark cells")
    return out


def lagrange4(table: np.ndarray, q: np.ndarray) -> np.ndarray:
    """QE four-point interpolation of a dq table (_native_fft.pyx:1556-1600)."""
    scaled = q / DQ
    lower = np.floor(scaled).astype(np.int64)
    f = scaled - lower
    u, v, w = 1.0 - f, 2.0 - f, 3.0 - f
    if table.ndim == 1:
        return (table[lower] * u * v * w / 6.0 + table[lower + 1] * f * v * w / 2.0
                - table[lower + 2] * f * u * w / 2.0 + table[lower + 3] * f * u * v / 6.0)
    return (table[lower] * (u * v * w / 6.0)[:, None] + table[lower + 1] * (f * v * w / 2.0)[:, None]
            - table[lower + 2] * (f * u * w / 2.0)[:, None]
            + table[lower + 3] * (f * u * v / 6.0)[:, None])


def lagrange4_derivative(table: np.ndarray, q: np.ndarray) -> np.ndarray:
    """d/dq of ``lagrange4``: the derivatives of the four Lagrange weights
    in the fraction f = q/dq - floor(q/dq), divided by dq
    (qepy_pw/upf.py:880-914)."""
    scaled = q / DQ
    lower = np.floor(scaled).astype(np.int64)
    f = scaled - lower
    u, v, w = 1.0 - f, 2.0 - f, 3.0 - f
    weights = (-(v * w + u * w + u * v) / 6.0, (v * w - f * (v + w)) / 2.0,
               -(u * w - f * (u + w)) / 2.0, (u * v - f * (u + v)) / 6.0)
    out = 0.0
    for offset, weight in enumerate(weights):
        sample = table[lower + offset]
        out = out + (sample * (weight / DQ) if table.ndim == 1
                     else sample * (weight / DQ)[:, None])
    return out


class SpeciesTables:
    """V_loc(q) and beta_l(q) of one pseudopotential in one cell volume."""

    def __init__(self, pseudo, volume: float) -> None:
        self.pseudo = pseudo
        self.volume = float(volume)
        self._vloc = None
        self._vloc_qmax = -1.0
        self._beta = None
        self._beta_qmax = -1.0

    # -- local potential ------------------------------------------------------
    def _vloc_table(self, qmax: float) -> np.ndarray:
        if self._vloc is not None and self._vloc_qmax + 1.0e-14 >= qmax:
            return self._vloc
        p = self.pseudo
        beyond = np.flatnonzero(p.r > 10.0)
        count = int(beyond[0] + 1) if len(beyond) else len(p.r)
        if count % 2 == 0:
            count -= 1
        r, rab = p.r[:count], p.rab[:count]
        short = r * (0.5 * p.vloc_ry[:count]) + p.z_valence * erf(r)
        size = int(qmax / DQ + 4)
        q = np.arange(size) * DQ
        table = np.empty(size)
        pref = 4.0 * np.pi / self.volume
        for b in range(0, size, 128):
            qb = q[b:b + 128]
            qr = np.multiply.outer(qb, r)
            sinc = np.ones_like(qr)
            np.divide(np.sin(qr), qb[:, None], out=sinc, where=qb[:, None] != 0.0)
            if b == 0:
                sinc[0] = r
            table[b:b + 128] = pref * qe_simpson(sinc * short[None, :], rab)
        self._vloc, self._vloc_qmax = table, qmax
        return table

    def vloc(self, q: np.ndarray) -> np.ndarray:
        """Periodic V_loc(|G|) in Hartree including the 1/Omega factor."""
        q = np.asarray(q, dtype=float)
        p = self.pseudo
        out = np.zeros_like(q)
        positive = q > 1.0e-12
        if np.any(~positive):
            beyond = np.flatnonzero(p.r > 10.0)
            count = int(beyond[0] + 1) if len(beyond) else len(p.r)
            if count % 2 == 0:
                count -= 1
            r, rab = p.r[:count], p.rab[:count]
            out[~positive] = 4.0 * np.pi / self.volume * qe_simpson(
                r * (r * 0.5 * p.vloc_ry[:count] + p.z_valence), rab)
        if np.any(positive):
            qp = q[positive]
            table = self._vloc_table(float(qp.max()))
            out[positive] = lagrange4(table, qp) - (4.0 * np.pi / self.volume) * p.z_valence \
                * np.exp(-0.25 * qp**2) / qp**2
        return out

    def vloc_with_derivative(self, q: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        """V_loc(|G|) and dV_loc/d|G| (zero at G = 0): the table's
        interpolation derivative plus that of the analytic -Z erf(r)/r tail
        (qepy_pw/upf.py:224-261)."""
        q = np.asarray(q, dtype=float)
        values = self.vloc(q)
        derivative = np.zeros_like(q)
        positive = q > 1.0e-12
        if np.any(positive):
            qp = q[positive]
            table = self._vloc_table(float(qp.max()))
            tail = -(4.0 * np.pi / self.volume) * self.pseudo.z_valence \
                * np.exp(-0.25 * qp**2) / qp**2
            derivative[positive] = lagrange4_derivative(table, qp) + tail * (-0.5 * qp - 2.0 / qp)
        return values, derivative

    # -- projectors -----------------------------------------------------------
    def _beta_table(self, qmax: float) -> np.ndarray:
        if self._beta is not None and self._beta_qmax + 1.0e-14 >= qmax:
            return self._beta
        p = self.pseudo
        size = int(np.floor(qmax / DQ + 4.0 + 0.5))
        q = np.arange(size) * DQ
        table = np.empty((size, len(p.betas)))
        pref = 4.0 * np.pi / np.sqrt(self.volume)
        for column, (rbeta, l, cutoff) in enumerate(zip(p.betas, p.angular_momenta, p.cutoff_indices)):
            count = min(cutoff, len(p.r), len(rbeta))
            r = p.r[:count]
            radial = rbeta[:count] * r
            for b in range(0, size, 128):
                bessel = spherical_jn(l, np.multiply.outer(q[b:b + 128], r)) * radial[None, :]
                table[b:b + 128, column] = pref * qe_simpson(bessel, p.rab[:count])
        self._beta, self._beta_qmax = table, qmax
        return table

    @property
    def channels(self) -> int:
        return sum(2 * l + 1 for l in self.pseudo.angular_momenta)

    def projectors(self, kg: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        """Species beta columns (npw, channels) and the channel coupling
        0.5 D_Ry (qepy_pw/upf.py:483-556)."""
        p = self.pseudo
        q = np.sqrt(kg[:, 0] ** 2 + kg[:, 1] ** 2 + kg[:, 2] ** 2)
        radial = lagrange4(self._beta_table(float(q.max()) if q.size else 0.0), q)
        safe = q > 1.0e-14
        inv = np.where(safe, 1.0 / np.where(safe, q, 1.0), 0.0)
        x = np.where(safe, kg[:, 0] * inv, 0.0)
        y = np.where(safe, kg[:, 1] * inv, 0.0)
        z = np.where(safe, kg[:, 2] * inv, 1.0)
        s0 = 1.0 / math.sqrt(4.0 * math.pi)
        s1 = math.sqrt(3.0 / (4.0 * math.pi))
        columns, ident = [], []
        for index, l in enumerate(p.angular_momenta):
            if l == 0:
                harmonics = (np.full_like(q, s0),)
            elif l == 1:
                harmonics = (s1 * z, -s1 * x, -s1 * y)
            else:
                raise ValueError("only l <= 1 projectors are supported")
            for m, h in enumerate(harmonics):
                columns.append(((-1j) ** l) * radial[:, index] * h)
                ident.append((index, l, m))
        beta = np.asfortranarray(np.stack(columns, axis=1))
        coupling = np.zeros((len(ident), len(ident)))
        for i, (ri, li, mi) in enumerate(ident):
            for j, (rj, lj, mj) in enumerate(ident):
                if li == lj and mi == mj:
                    coupling[i, j] = 0.5 * p.dij_ry[ri, rj]
        return beta, coupling

    def projectors_with_gradient(self, kg: np.ndarray):
        """``projectors`` and the Cartesian gradient of every column with
        respect to k+G, (npw, channels, 3): (-i)^l (dbeta/dq Y_lm khat +
        beta grad Y_lm), zero at k+G = 0 (qepy_pw/upf.py:558-597).  The l = 1
        harmonics are s1 (z, -x, -y)/q, whose gradients are
        s1 (e_a - khat_a khat)/q."""
        p = self.pseudo
        beta, coupling = self.projectors(kg)
        q = np.sqrt(kg[:, 0] ** 2 + kg[:, 1] ** 2 + kg[:, 2] ** 2)
        table = self._beta_table(float(q.max()) if q.size else 0.0)
        radial = lagrange4(table, q)
        radial_d = lagrange4_derivative(table, q)
        safe = q > 1.0e-14
        inv = np.where(safe, 1.0 / np.where(safe, q, 1.0), 0.0)
        khat = kg * inv[:, None]
        s0 = 1.0 / math.sqrt(4.0 * math.pi)
        s1 = math.sqrt(3.0 / (4.0 * math.pi))
        gradient = np.zeros((len(q), beta.shape[1], 3), dtype=np.complex128)
        column = 0
        for index, l in enumerate(p.angular_momenta):
            phase = (-1j) ** l
            if l == 0:
                harmonics = [(np.full_like(q, s0), np.zeros((len(q), 3)))]
            elif l == 1:
                harmonics = []
                for axis, sign in ((2, 1.0), (0, -1.0), (1, -1.0)):
                    unit = np.zeros(3)
                    unit[axis] = 1.0
                    value = sign * s1 * khat[:, axis]
                    grad = sign * s1 * (unit[None, :] - khat[:, axis:axis + 1] * khat) \
                        * inv[:, None]
                    harmonics.append((value, grad))
            else:
                raise ValueError("only l <= 1 projectors are supported")
            for value, grad in harmonics:
                gradient[:, column, :] = phase * (radial_d[:, index, None] * khat * value[:, None]
                                                  + radial[:, index, None] * grad)
                column += 1
        gradient[~safe] = 0.0
        return beta, coupling, gradient


def channel_list(angular_momenta) -> list[tuple[int, int, int]]:
    """(radial column, l, m) of every projector channel in QE's order."""
    return [(index, l, m) for index, l in enumerate(angular_momenta) for m in range(2 * l + 1)]


def device_projectors(tables: "SpeciesTables", kg) -> tuple:
    """``SpeciesTables.projectors`` on the GPU: the radial table (host, once
    per species and cell) interpolated and combined with the real harmonics
    by qeb_projector_basis for every plane wave.  ``kg`` is the (npw, 3)
    k+G array (host or device); returns (beta, coupling) with beta a
    column-major complex128 CUDA tensor."""
    from . import _lib
    from .device import empty_f, leading_dimension, require_cuda, stream_handle

    device = require_cuda()
    p = tables.pseudo
    if any(l > 2 for l in p.angular_momenta):
        raise ValueError("only l <= 2 projectors are supported")
    kg_dev = kg if isinstance(kg, torch.Tensor) else torch.from_numpy(np.asarray(kg, dtype=float))
    kg_dev = kg_dev.to(device=device, dtype=torch.float64)
    npw = kg_dev.shape[0]
    kg_cols = kg_dev.T.contiguous()  # (3, npw): column-major (npw, 3)
    qmax = float(torch.sqrt((kg_dev * kg_dev).sum(dim=1)).max()) if npw else 0.0
    table = torch.from_numpy(np.ascontiguousarray(tables._beta_table(qmax))).to(device)
    channels = channel_list(p.angular_momenta)
    radial = np.array([c[0] for c in channels], dtype=np.int32)
    ls = np.array([c[1] for c in channels], dtype=np.int32)
    ms = np.array([c[2] for c in channels], dtype=np.int32)
    beta = empty_f(npw, len(channels), torch.complex128, device)
    _lib.check("qeb_projector_basis", _lib.load().qeb_projector_basis(
        npw, kg_cols.data_ptr(), table.data_ptr(), table.shape[0], table.shape[1], DQ,
        len(channels), radial.ctypes.data, ls.ctypes.data, ms.ctypes.data, beta.data_ptr(),
        leading_dimension(beta), stream_handle()))
    coupling = np.zeros((len(channels), len(channels)))
    for i, (ri, li, mi) in enumerate(channels):
        for j, (rj, lj, mj) in enumerate(channels):
            if li == lj and mi == mj:
                coupling[i, j] = 0.5 * p.dij_ry[ri, rj]
    return beta, coupling


def structure_factor(vectors: np.ndarray, positions: np.ndarray, weights: np.ndarray) -> np.ndarray:
    """S(G) = sum_a w_a exp(-i G.tau_a), chunked over atoms (host)."""
    out = np.zeros(len(vectors), dtype=np.complex128)
    for a0 in range(0, len(positions), 16):
        out += np.exp(-1j * (vectors @ positions[a0:a0 + 16].T)) @ weights[a0:a0 + 16]
    return out


def ewald_energy(lattice: np.ndarray, positions: np.ndarray, charges: np.ndarray,
                 ecutrho_ry: float, structure=structure_factor) -> float:
    """Ion-ion Ewald energy in Hartree (qepy_pw/ewald.py:49-143).

    ``structure(vectors, positions, charges)`` evaluates the structure factor
    (host by default; the SCF passes a GPU evaluation for large cells)."""
    lattice = np.asarray(lattice, dtype=float)
    positions = np.asarray(positions, dtype=float)
    charges = np.asarray(charges, dtype=float)
    volume = abs(float(np.linalg.det(lattice)))
    reciprocal = 2.0 * np.pi * np.linalg.inv(lattice).T
    total = float(np.sum(charges))
    alpha = 2.9
    while True:
        alpha -= 0.1
        bound = 2.0 * total**2 * np.sqrt(alpha / np.pi) * erfc(np.sqrt(ecutrho_ry / (4.0 * alpha)))
        if bound <= 1.0e-7:
            break
        if alpha <= 0.0:
            raise RuntimeError("optimal Ewald alpha not found")
    # reciprocal-space sum over |G|^2 <= ecutrho (lexicographic Miller order)
    smin = float(np.linalg.svd(reciprocal, compute_uv=False)[-1])
    nmax = int(np.ceil(np.sqrt(ecutrho_ry) / smin)) + 1
    axis = np.arange(-nmax, nmax + 1)
    recip_sum = -total**2 / (4.0 * alpha)
    acc = 0.0
    yz = np.stack(np.meshgrid(axis, axis, indexing="ij"), -1).reshape(-1, 2)
    gs, g2s = [], []
    for i in axis:
        miller = np.column_stack((np.full(len(yz), i), yz))
        g = miller @ reciprocal
        g2 = np.einsum("ij,ij->i", g, g)
        keep = (g2 <= ecutrho_ry) & (g2 > 1.0e-14)
        gs.append(g[keep])
        g2s.append(g2[keep])
    g, g2 = np.concatenate(gs), np.concatenate(g2s)
    if g2.size:
        s = structure(g, positions, charges)
        acc = float(np.sum(np.abs(s) ** 2 * np.exp(-g2 / (4.0 * alpha)) / g2))
    recip_sum = (recip_sum + acc) * 4.0 * np.pi / volume
    recip_sum -= float(np.sum(charges**2) * 2.0 * np.sqrt(alpha / np.pi))
    # real-space sum within 4/sqrt(alpha)
    radius = 4.0 / np.sqrt(alpha)
    real_sum = 0.0
    sqa = float(np.sqrt(alpha))
    q = None
    for first, d in _real_space_blocks(lattice, positions, radius):
        # d: (block atoms, nat, images, 3) separations a - b + image (torch)
        if q is None:
            q = torch.as_tensor(charges, dtype=torch.float64, device=d.device)
        dist = torch.linalg.vector_norm(d, dim=3)
        mask = (dist >= 1.0e-14) & (dist <= radius)
        safe = torch.where(mask, dist, torch.ones_like(dist))
        contrib = torch.where(mask, torch.special.erfc(sqa * safe) / safe, torch.zeros_like(dist))
        block_q = q[first:first + d.shape[0]]
        real_sum += float(torch.sum(block_q * (contrib.sum(dim=2) @ q)))
    return 0.5 * (recip_sum + 0.5 * real_sum)


def _real_space_blocks(lattice: np.ndarray, positions: np.ndarray, radius: float, block: int = 16):
    """(first atom, separations) for blocks of atoms a: the vectors
    a - b + R (float64 torch tensors, on the GPU when there is one) over all
    atoms b and the lattice translations R of one common image cube, large
    enough that every pair within ``radius`` is in it for every a (images
    beyond ``radius`` are masked by the callers)."""
    device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() \
        else torch.device("cpu")
    lmin = float(np.linalg.svd(lattice, compute_uv=False)[-1])
    reach = max(float(np.max(np.linalg.norm(a - positions, axis=1))) for a in positions)
    nb = int(np.ceil((radius + reach) / lmin)) + 1
    rng = np.arange(-nb, nb + 1)
    images = torch.as_tensor(
        np.stack(np.meshgrid(rng, rng, rng, indexing="ij"), -1).reshape(-1, 3) @ lattice,
        dtype=torch.float64, device=device)
    pos = torch.as_tensor(np.ascontiguousarray(positions), dtype=torch.float64, device=device)
    for first in range(0, len(positions), block):
        d0 = pos[first:first + block, None, :] - pos[None, :, :]
        yield first, d0[:, :, None, :] + images[None, None, :, :]


def pz81(rho: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """(eps_xc, v_xc) in Hartree of the unpolarised PZ81 LDA.

    Slater exchange eps_x = -(3/4)(3/pi)^(1/3) rho^(1/3) = -0.458165/r_s and
    the Perdew-Zunger (1981) correlation: for r_s >= 1
    eps_c = gamma/(1 + beta1 sqrt(r_s) + beta2 r_s), otherwise
    eps_c = A ln r_s + B + C r_s ln r_s + D r_s, with gamma = -0.1423,
    beta1 = 1.0529, beta2 = 0.3334, A = 0.0311, B = -0.048, C = 0.0020,
    D = -0.0116; v = eps - (r_s/3) d eps/d r_s.  Densities at or below 1e-10
    give zero, as the reference's LDA driver does.
    """
    d = np.abs(np.asarray(rho, dtype=np.float64))
    active = d > 1.0e-10
    d = np.maximum(d, 1.0e-10)
    rs = 0.6203504908994 / np.cbrt(d)
    eps = -0.687247939924714 * (2.0 / 3.0) / rs
    v = (4.0 / 3.0) * eps
    high = rs < 1.0
    lnrs = np.log(rs)
    ec_high = 0.0311 * lnrs - 0.048 + 0.0020 * rs * lnrs - 0.0116 * rs
    vc_high = ec_high - (0.0311 + (0.0020 * (lnrs + 1.0) - 0.0116) * rs) / 3.0
    sq = np.sqrt(rs)
    den = 1.0 + 1.0529 * sq + 0.3334 * rs
    ec_low = -0.1423 / den
    vc_low = ec_low + (-0.1423 / 3.0) * rs * (0.5 * 1.0529 / sq + 0.3334) / den**2
    eps = eps + np.where(high, ec_high, ec_low)
    v = v + np.where(high, vc_high, vc_low)
    eps[~active] = 0.0
    v[~active] = 0.0
    return eps, v
