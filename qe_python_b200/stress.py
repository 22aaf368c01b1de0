"""Analytic (Hellmann-Feynman) stress at SCF convergence, on the GPU.

The seven terms of the reference's stress (qepy_pw/pw/scf.py:1676-1931),
compressive positive, Hartree/bohr^3:
  kinetic   sum_k w_k sum_G (sum_b f_b |c_Gb|^2) (k+G)_i (k+G)_j / Omega
  local     sum_G Re(conj rho(G) dV_loc/d|G| S(G)) G_i G_j / |G| + E_loc/Omega 1
  nonlocal  (T + T^T)/2 + E_nl/Omega 1, T from the projector gradients
  Hartree   -4 pi sum_G |rho(G)|^2 G_i G_j / G^4 + E_H/Omega 1
  xc        -(E_xc - int rho v_xc)/Omega 1                   (LDA)
  core      0 (no core correction in the supported pseudopotentials)
  Ewald     qepy_pw/ewald.py:261-365
each symmetrised over the point group (qepy_pw/symmetry.py:1006-1027).

The nonlocal tensor of the reference sums, per atom a,
  T_lr = 2/Omega sum_k w_k Re sum_{p,b} f_b conj(dO_a[p,l,r,b]) (D O_a)[p,b],
  dO_a[p,l,r,b] = sum_g conj(d beta_p/d(k+G)_l) (k+G)_r conj(e_a) psi_b,
with e_a = exp(-i (k+G).tau_a).  Moving the band sum inside,
  T_lr = 2/Omega sum_k w_k Re sum_g (k+G)_r sum_p d beta_p/d(k+G)_l U[g,p],
  U[g,p] = sum_a e_a(g) sum_b conj(psi_b(g)) f_b (D O_a)[p,b],
which is one (npw x bands) x (bands x P) product per k point and species
instead of nine (npw x P) x (npw x bands) ones.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch
from scipy.special import erfc

from . import kernels as K
from .device import to_device_f
from .pseudo_tables import _real_space_blocks


@dataclass
class StressTerms:
    """Symmetrised stress terms, Hartree/bohr^3 (the reference's
    SCFStressTerms, qepy_pw/pw/scf.py:175-184)."""

    kinetic: np.ndarray
    local: np.ndarray
    nonlocal_: np.ndarray
    hartree: np.ndarray
    xc: np.ndarray
    core_correction: np.ndarray
    ewald: np.ndarray

    def as_tuple(self) -> tuple:
        return (self.kinetic, self.local, self.nonlocal_, self.hartree, self.xc,
                self.core_correction, self.ewald)


def symmetrize_stress(tensor: np.ndarray, lattice: np.ndarray, operations) -> np.ndarray:
    """Average R^T T R over the point group, R = L^-1 M L the Cartesian
    form of each operation's fractional matrix M (row-vector convention),
    then symmetrise the result (qepy_pw/symmetry.py:1006-1027)."""
    tensor = np.asarray(tensor, dtype=float)
    if len(operations) <= 1:
        return 0.5 * (tensor + tensor.T)
    lattice = np.asarray(lattice, dtype=float)
    inverse = np.linalg.inv(lattice)
    out = np.zeros((3, 3))
    for op in operations:
        rotation = inverse @ np.asarray(op.matrix, dtype=float) @ lattice
        out += rotation.T @ tensor @ rotation
    out /= len(operations)
    return 0.5 * (out + out.T)


def _outer_sum(weight: torch.Tensor, left: torch.Tensor, right: torch.Tensor) -> np.ndarray:
    """sum_g weight[g] left[g, i] right[g, j] as a host (3, 3) array."""
    return torch.einsum("g,gi,gj->ij", weight, left, right).cpu().numpy()


def kinetic_stress(states, occupations, weights, volume: float) -> np.ndarray:
    out = np.zeros((3, 3))
    for state, occ, weight in zip(states, occupations, weights):
        occ = np.asarray(occ, dtype=float)
        if occ.size == 0:
            continue
        psi = state.vectors[:, :occ.size]
        device = psi.device
        density = (psi.real.double() ** 2 + psi.imag.double() ** 2) @ \
            torch.as_tensor(occ, dtype=torch.float64, device=device)
        gk = torch.from_numpy(np.ascontiguousarray(state.basis.vectors)).to(device)
        out += float(weight) * _outer_sum(density, gk, gk) / volume
    return out


def _species_structure(system, label: str, g: torch.Tensor) -> torch.Tensor:
    """S(G) = sum over the species' atoms of exp(-i G.tau), FP64 on the device."""
    pos = np.array([p for p, l in zip(system.positions, system.labels) if l == label])
    out = torch.zeros(g.shape[0], dtype=torch.complex128, device=g.device)
    for a0 in range(0, len(pos), 64):
        tau = torch.from_numpy(np.ascontiguousarray(pos[a0:a0 + 64])).to(g.device)
        angle = g @ tau.T
        out += torch.polar(torch.ones_like(angle), -angle).sum(dim=1)
    return out


def local_and_hartree_stress(system, tables, grid, cgrid, rho: torch.Tensor):
    """(local, Hartree) terms from rho(G) on the charge sphere."""
    device = rho.device
    volume = system.volume
    rho_g = cgrid.to_g(rho)
    g = torch.from_numpy(np.ascontiguousarray(grid.vectors)).to(device)
    g2_host = np.asarray(grid.g2, dtype=float)
    q_host = np.sqrt(g2_host)
    g2 = torch.from_numpy(g2_host).to(device)
    q = torch.from_numpy(q_host).to(device)
    radial = q > 1.0e-14
    safe_q = torch.where(radial, q, torch.ones_like(q))
    local_energy = 0.0
    local_tensor = np.zeros((3, 3))
    for label, table in tables.items():
        if label not in system.labels:
            continue
        values, derivative = table.vloc_with_derivative(q_host)
        values = torch.from_numpy(values).to(device)
        derivative = torch.from_numpy(derivative).to(device)
        structure = _species_structure(system, label, g)
        local_energy += volume * float(torch.real(torch.sum(torch.conj(rho_g) * values
                                                             * structure)))
        weight = torch.where(radial, torch.real(torch.conj(rho_g) * derivative * structure)
                             / safe_q, torch.zeros_like(q))
        local_tensor += _outer_sum(weight, g, g)
    local = local_tensor + local_energy / volume * np.eye(3)
    nonzero = g2 > 1.0e-14
    safe_g2 = torch.where(nonzero, g2, torch.ones_like(g2))
    density2 = torch.where(nonzero, torch.abs(rho_g) ** 2 / safe_g2, torch.zeros_like(g2))
    hartree_energy = 2.0 * np.pi * volume * float(torch.sum(density2))
    hartree_tensor = -4.0 * np.pi * _outer_sum(density2 / safe_g2, g, g)
    hartree = hartree_tensor + hartree_energy / volume * np.eye(3)
    return local, hartree


def xc_stress(system, rho: torch.Tensor) -> np.ndarray:
    """-(E_xc - int rho v_xc)/Omega on the diagonal (PZ81 LDA, no core)."""
    from .charge import pz81

    epsilon, potential = pz81(rho)
    scale = system.volume / rho.numel()
    energy = scale * float(torch.sum(rho * epsilon))
    potential_energy = scale * float(torch.sum(rho * potential))
    return -(energy - potential_energy) / system.volume * np.eye(3)


def nonlocal_stress(system, states, tables, occupations, weights) -> np.ndarray:
    """(T + T^T)/2 + E_nl/Omega 1 with T of the module docstring."""
    volume = system.volume
    tensor = np.zeros((3, 3))
    energy = 0.0
    for state, occ, weight in zip(states, occupations, weights):
        occ = np.asarray(occ, dtype=float)
        active = np.flatnonzero(np.abs(occ) > 1.0e-15)
        if active.size == 0:
            continue
        count = int(active[-1]) + 1
        device = state.vectors.device
        psi = state.vectors[:, :count]
        if psi.dtype != torch.complex128:
            psi = psi.to(torch.complex128)
        psi = psi.T.contiguous().T
        f_b = torch.as_tensor(occ[:count], dtype=torch.float64, device=device)
        kg_host = np.ascontiguousarray(state.basis.vectors)
        kg = torch.from_numpy(kg_host).to(device)
        for label, table in tables.items():
            atom_index = [i for i, l in enumerate(system.labels) if l == label]
            if not atom_index or table.channels == 0:
                continue
            species, coupling1, gradient = table.projectors_with_gradient(kg_host)
            tau = torch.as_tensor(np.ascontiguousarray(system.positions[atom_index].T),
                                  dtype=torch.float64, device=device)
            angle = kg @ tau
            phases = torch.polar(torch.ones_like(angle), -angle)      # (npw, natoms)
            del angle
            natoms, c = phases.shape[1], species.shape[1]
            species_d = torch.from_numpy(np.ascontiguousarray(species)).to(device)
            beta = to_device_f((species_d[:, None, :] * phases[:, :, None]).reshape(-1, natoms * c),
                               torch.complex128, device)
            becp = K.gemm(K.OP_C, beta, psi)                            # (natoms c, bands)
            coupling = torch.from_numpy(coupling1.astype(np.complex128)).to(device)
            coupled = torch.einsum("pq,aqb->apb", coupling,
                                   becp.reshape(natoms, c, count))       # D O_a
            energy += float(weight) * float(torch.real(
                torch.sum(torch.conj(becp.reshape(natoms, c, count)) * coupled * f_b)))
            # U[g, p] = sum_a e_a(g) sum_b conj(psi_b(g)) f_b (D O_a)[p, b]
            y = (coupled * f_b).reshape(natoms * c, count).T.conj()      # (bands, natoms c)
            m = torch.conj(psi @ y.contiguous())                          # (npw, natoms c)
            u = (m.reshape(-1, natoms, c) * phases[:, :, None]).sum(dim=1)  # (npw, c)
            grad = torch.from_numpy(gradient).to(device)                  # (npw, c, 3)
            tensor += 2.0 * float(weight) / volume * torch.real(
                torch.einsum("gpl,gp,gr->lr", grad, u, kg.to(torch.complex128))).cpu().numpy()
    return 0.5 * (tensor + tensor.T) + energy / volume * np.eye(3)


def ewald_stress(lattice, positions, charges, ecutrho_ry: float, g_vectors) -> np.ndarray:
    """Ewald stress with the energy's alpha and G set (qepy_pw/ewald.py:261-365):
    reciprocal sums on the G sphere and the real-space pair sum over the
    images within 4/sqrt(alpha), both in FP64 on the device."""
    lattice = np.asarray(lattice, dtype=float)
    positions = np.asarray(positions, dtype=float)
    charges = np.asarray(charges, dtype=float)
    volume = abs(float(np.linalg.det(lattice)))
    total = float(np.sum(charges))
    alpha = 2.9
    while True:
        alpha -= 0.1
        if 2.0 * total**2 * np.sqrt(alpha / np.pi) * erfc(np.sqrt(ecutrho_ry / (4.0 * alpha))) <= 1.0e-7:
            break
        if alpha <= 0.0:
            raise RuntimeError("optimal Ewald alpha not found")
    device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() \
        else torch.device("cpu")
    g = torch.from_numpy(np.ascontiguousarray(g_vectors, dtype=float)).to(device)
    g2 = torch.einsum("ij,ij->i", g, g)
    keep = g2 > 1.0e-14
    g, g2 = g[keep], g2[keep]
    q = torch.from_numpy(charges).to(device)
    pos = torch.from_numpy(np.ascontiguousarray(positions)).to(device)
    structure = torch.zeros(g.shape[0], dtype=torch.complex128, device=device)
    for a0 in range(0, len(positions), 64):
        angle = pos[a0:a0 + 64] @ g.T
        structure += q[a0:a0 + 64].to(torch.complex128) @ torch.polar(torch.ones_like(angle), -angle)
    terms = torch.abs(structure) ** 2 * torch.exp(-g2 / (4.0 * alpha)) / g2
    reciprocal_sum = float(torch.sum(terms))
    reciprocal_tensor = _outer_sum(terms * (1.0 / (4.0 * alpha) + 1.0 / g2), g, g)
    scalar = -total**2 / (4.0 * alpha) + reciprocal_sum
    stress = 2.0 * np.pi / volume**2 * (scalar * np.eye(3) - 2.0 * reciprocal_tensor)
    radius = 4.0 / np.sqrt(alpha)
    ra = float(np.sqrt(alpha))
    real = None
    for first, d in _real_space_blocks(lattice, positions, radius):
        # d: (block atoms i, atoms j, images, 3) separations tau_i - tau_j + image
        dist = torch.linalg.vector_norm(d, dim=3)
        mask = (dist >= 1.0e-14) & (dist <= radius)
        safe = torch.where(mask, dist, torch.ones_like(dist))
        radial = (-torch.special.erfc(ra * safe) / safe**2
                  - 2.0 * ra / np.sqrt(np.pi) * torch.exp(-alpha * safe**2) / safe)
        qd = q.to(d.device)
        qi = qd[first:first + d.shape[0]]
        weight = 0.25 * qi[:, None, None] * qd[None, :, None] * radial / (volume * safe)
        weight = torch.where(mask, weight, torch.zeros_like(weight))
        block = torch.einsum("ijn,ijna,ijnb->ab", weight, d, d)
        real = block if real is None else real + block
    if real is not None:
        stress = stress - real.cpu().numpy()
    return 0.5 * (stress + stress.T)


def scf_stress(system, states, tables, grid, cgrid, rho: torch.Tensor, occupations,
               weights, pools=None) -> tuple[np.ndarray, StressTerms]:
    """Total stress and its symmetrised terms (Ha/bohr^3) at convergence;
    with k-point pools ``states``/``occupations``/``weights`` are this
    rank's k points and the k sums are combined over the pools."""
    charges = np.array([system.pseudos[l].z_valence for l in system.labels])
    kinetic = kinetic_stress(states, occupations, weights, system.volume)
    nonlocal_ = nonlocal_stress(system, states, tables, occupations, weights)
    if pools is not None:
        device = states[0].vectors.device if states else None
        kinetic = pools.sum_array(kinetic, device)
        nonlocal_ = pools.sum_array(nonlocal_, device)
    local, hartree = local_and_hartree_stress(system, tables, grid, cgrid, rho)
    xc = xc_stress(system, rho)
    core = np.zeros((3, 3))
    ewald = ewald_stress(system.lattice, system.positions, charges, system.ecutrho,
                         grid.vectors)
    raw = (kinetic, local, nonlocal_, hartree, xc, core, ewald)
    terms = StressTerms(*(symmetrize_stress(0.5 * (t + t.T), system.lattice, system.operations)
                          for t in raw))
    total_raw = sum(raw)
    total = symmetrize_stress(0.5 * (total_raw + total_raw.T), system.lattice, system.operations)
    return total, terms
