"""Hellmann-Feynman forces at SCF convergence.

F = F_nonlocal + F_local + F_ewald (symmetrised when the space group is
non-trivial), minus the mean force, as qepy_pw/pw/scf.py:4143-4227 assembles
them (no core correction in the supported pseudopotentials).
  F_nonlocal[atom] = -2 sum_k w_k Re sum_{p in atom, b} f_b
                     conj(d becp_a[p, b]) (D becp)[p, b],
                     d becp_a = beta_atom^H (i (k+G)_a psi)     (scf.py:1521-1631)
  F_local[atom]    = Omega Re sum_G conj(rho(G)) i G V_loc(|G|) e^{-i G tau}
                                                                 (scf.py:1634-1673)
  F_ewald          = -dE_ewald/dtau with E_ewald's alpha and G set
                                                                 (ewald.py:144-260)
The three d becp products per k point are complex GEMMs on the GPU
(libqeb200.so); the per-atom reductions are small host sums.  Hartree/bohr.
"""

from __future__ import annotations

import numpy as np
import torch
from scipy.special import erfc

from . import kernels as K
from .device import empty_f, to_device_f
from .pseudo_tables import _real_space_blocks


def ewald_forces(lattice, positions, charges, ecutrho_ry, g_vectors) -> np.ndarray:
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
    g = np.asarray(g_vectors, dtype=float)
    g2 = np.einsum("ij,ij->i", g, g)
    keep = g2 > 1.0e-14
    g, g2 = g[keep], g2[keep]
    weight = 2.0 * np.pi / volume * np.exp(-g2 / (4.0 * alpha)) / g2
    forces = _ewald_reciprocal_forces(positions, charges, g, weight)
    radius = 4.0 / np.sqrt(alpha)
    ra = float(np.sqrt(alpha))
    q = None
    total_grad = None
    for first, d in _real_space_blocks(lattice, positions, radius):
        # d: (block atoms i, nat j, images, 3) separations i - j + image (torch)
        if q is None:
            q = torch.as_tensor(charges, dtype=torch.float64, device=d.device)
            total_grad = torch.zeros((len(positions), 3), dtype=torch.float64, device=d.device)
        dist = torch.linalg.vector_norm(d, dim=3)
        mask = (dist >= 1.0e-14) & (dist <= radius)
        safe = torch.where(mask, dist, torch.ones_like(dist))
        radial = (-torch.special.erfc(ra * safe) / safe**2
                  - 2.0 * ra / np.sqrt(np.pi) * torch.exp(-alpha * safe**2) / safe)
        qi = q[first:first + d.shape[0]]
        grad = (0.25 * qi[:, None, None, None] * q[None, :, None, None]
                * (radial / safe)[:, :, :, None] * d)
        grad = torch.where(mask[:, :, :, None], grad, torch.zeros_like(grad)).sum(dim=2)
        total_grad[first:first + d.shape[0]] -= grad.sum(dim=1)
        total_grad += grad.sum(dim=0)
    if total_grad is not None:
        forces = forces + total_grad.cpu().numpy()
    return forces


def _ewald_reciprocal_forces(positions, charges, g, weight) -> np.ndarray:
    """-d/dtau of sum_G w(G) |S(G)|^2, S(G) = sum_a Z_a e^{-i G tau_a}, in
    FP64 on the GPU when one is present (216 atoms x 1.2M G vectors are
    2.6e8 phase factors), else on the host."""
    device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() \
        else torch.device("cpu")
    gt = torch.from_numpy(np.ascontiguousarray(g)).to(device)
    wt = torch.from_numpy(weight).to(device)
    pos = torch.from_numpy(np.ascontiguousarray(positions)).to(device)
    q = torch.from_numpy(np.ascontiguousarray(charges, dtype=float)).to(device)
    chunk = 64
    structure = torch.zeros(len(weight), dtype=torch.complex128, device=device)
    for a0 in range(0, len(positions), chunk):
        ph = torch.exp(-1j * (pos[a0:a0 + chunk] @ gt.T))
        structure += q[a0:a0 + chunk].to(torch.complex128) @ ph
    conj_s = torch.conj(structure)
    forces = torch.zeros_like(pos)
    for a0 in range(0, len(positions), chunk):
        ph = torch.exp(-1j * (pos[a0:a0 + chunk] @ gt.T))
        deriv = 2.0 * torch.real(conj_s[None, :] * (-1j * q[a0:a0 + chunk, None] * ph))
        forces[a0:a0 + chunk] -= (wt[None, :] * deriv) @ gt
    return forces.cpu().numpy()


def local_forces(system, tables, grid, rho) -> np.ndarray:
    """Omega Re sum_G conj(rho(G)) i G V_loc(|G|) exp(-i G tau), on the GPU."""
    device = torch.device("cuda", torch.cuda.current_device())
    rho_g = torch.from_numpy(grid.to_g(rho)).to(device)
    gvec = torch.from_numpy(grid.vectors).to(device)
    q = np.sqrt(grid.g2)
    out = np.zeros((len(system.positions), 3))
    for label, table in tables.items():
        vloc = torch.from_numpy(table.vloc(q)).to(device)
        weight = torch.conj(rho_g) * vloc  # (nG,)
        idx = [i for i, l in enumerate(system.labels) if l == label]
        for a0 in range(0, len(idx), 32):
            atoms = idx[a0:a0 + 32]
            pos = torch.from_numpy(system.positions[atoms]).to(device)
            phase = torch.exp(-1j * (pos @ gvec.T))               # (na, nG)
            term = (1j * weight)[None, :] * phase                   # (na, nG)
            f = torch.real(term @ gvec.to(torch.complex128))        # (na, 3)
            out[atoms] = system.volume * f.cpu().numpy()
    return out


def _band_occupations(occupations, nk: int) -> list[np.ndarray]:
    """Per-k occupation arrays; an int means two electrons in that many bands."""
    if isinstance(occupations, (int, np.integer)):
        return [np.full(int(occupations), 2.0) for _ in range(nk)]
    return [np.asarray(f, dtype=float) for f in occupations]


def nonlocal_forces(system, states, tables, occupations, weights=None) -> np.ndarray:
    """F_nl = -2 sum_k w_k sum_b f_b Re[conj(d becp/d tau) D becp]
    (qepy_pw/pw/scf.py:1521-1631); ``occupations`` is a band count (two
    electrons each) or one occupation array per k point; ``weights`` the k
    weights of ``states`` (default: all of the system's k points)."""
    out = np.zeros((len(system.positions), 3))
    band_occ = _band_occupations(occupations, len(states))
    weights = system.weights if weights is None else weights
    for state, weight, occ in zip(states, weights, band_occ):
        active = np.flatnonzero(np.abs(occ) > 1.0e-15)
        if active.size == 0:
            continue
        count = int(active[-1]) + 1
        f_b = occ[:count][None, :]
        basis = state.basis
        device = state.vectors.device
        psi = state.vectors[:, :count]
        if psi.dtype != torch.complex128:
            psi = psi.to(torch.complex128)
        psi = psi.T.contiguous().T
        vectors = basis.vectors
        kg = torch.from_numpy(vectors).to(device)
        for label, table in tables.items():
            atom_index = [i for i, l in enumerate(system.labels) if l == label]
            if not atom_index or table.channels == 0:
                continue
            species, coupling1 = table.projectors(vectors)
            # structure phases exp(-i (k+G).tau) on the device
            tau = torch.as_tensor(np.ascontiguousarray(system.positions[atom_index].T),
                                  dtype=torch.float64, device=device)
            angle = kg @ tau
            phases = to_device_f(torch.polar(torch.ones_like(angle), -angle), torch.complex128,
                                 device)
            del angle
            species = to_device_f(species, torch.complex128, device)
            natoms, c = phases.shape[1], species.shape[1]
            beta = empty_f(len(basis), natoms * c, torch.complex128, device)
            for a in range(natoms):
                beta[:, a * c:(a + 1) * c] = species * phases[:, a:a + 1]
            coupling = to_device_f(np.kron(np.eye(natoms), coupling1).astype(np.complex128),
                                   torch.complex128, device)
            becp = K.gemm(K.OP_C, beta, psi)
            coupled = K.gemm(K.OP_N, coupling, becp).cpu().numpy()
            for axis in range(3):
                scaled = (psi * (1j * kg[:, axis:axis + 1])).T.contiguous().T
                dbecp = K.gemm(K.OP_C, beta, scaled).cpu().numpy()
                contrib = (np.real(np.conj(dbecp) * coupled) * f_b).sum(axis=1)  # per channel
                out[atom_index, axis] -= 2.0 * float(weight) * contrib.reshape(natoms, c).sum(axis=1)
    return out


def hellmann_feynman_forces(system, states, tables, grid, rho, occupations, weights=None,
                            pools=None) -> np.ndarray:
    """Total forces; with k-point pools, ``states``/``occupations``/``weights``
    are this rank's k points and the nonlocal part is summed over the pools."""
    charges = np.array([system.pseudos[l].z_valence for l in system.labels])
    nonlocal_part = nonlocal_forces(system, states, tables, occupations, weights)
    if pools is not None:
        device = states[0].vectors.device if states else None
        nonlocal_part = pools.sum_array(nonlocal_part, device)
    components = [
        nonlocal_part,
        ewald_forces(system.lattice, system.positions, charges, system.ecutrho, grid.vectors),
        local_forces(system, tables, grid, rho),
    ]
    total = sum(symmetrize_forces(c, system) for c in components)
    return total - total.mean(axis=0, keepdims=True)


def symmetrize_forces(forces: np.ndarray, system) -> np.ndarray:
    """Average F over the space group: F'(op(atom)) = F(atom) R (cartesian)."""
    ops = system.operations
    if len(ops) <= 1:
        return forces
    lattice = system.lattice
    frac = system.positions @ np.linalg.inv(lattice)
    out = np.zeros_like(forces)
    for op in ops:
        rot = np.linalg.inv(lattice) @ op.matrix @ lattice  # cartesian row convention
        moved = frac @ op.matrix + op.translation
        for i, x in enumerate(moved):
            delta = frac - x
            delta -= np.round(delta)
            j = int(np.argmin(np.abs(delta).max(axis=1)))
            out[j] += forces[i] @ rot
    return out / len(ops)
