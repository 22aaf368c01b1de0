"""Band energy as a differentiable function of the potential and the ions.

E_band(V_Hxc, tau) = sum_k w_k sum_b f_b eps_b(k), the eigenvalues of
H = T + V_ion(tau) + V_Hxc + V_NL(tau) solved by the GPU Davidson.  By
Hellmann-Feynman (eigenpairs converged):
  dE/dV(r)   = sum_k w_k sum_b f_b |psi_b(r)|^2 / N_r
               (psi_b(r) the unnormalised inverse FFT of the coefficients;
               the GPU density kernel with weights w f / N_r)
  dE/dtau_a  = local:    Re sum_G conj(rho_N(G)) (-i G) V_loc(|G|) e^{-i G tau_a} N_r
               nonlocal: 2 sum_k w_k Re sum_b f_b conj(d becp_a) (D becp)
               (the same derivative contractions as the Hellmann-Feynman
               forces, qepy_pw/pw/scf.py:1521-1673, with the opposite sign)
``BandEnergy.apply(v_hxc, positions)`` returns E_band (Hartree) and, through
torch.autograd, d E_band / d v_hxc and d E_band / d positions.
"""

from __future__ import annotations

import numpy as np
import torch

from .diagonalization import PlaneWaveHamiltonian, davidson
from .forces import nonlocal_forces
from .scf import ChargeGrid, KPointState, QERandom, projector_terms, random_starting_subspace


class BandProblem:
    """Fixed cell, bases and tables; positions and V_Hxc vary."""

    def __init__(self, system, precision: str = "f64", tolerance: float = 1.0e-11) -> None:
        """precision: 'f64' (plain), or 'mixed' (chosen form: an FP32/split-TF32
        Davidson to 1e-6 Ha, then FP64 Davidson iterations from its vectors).

        Hellmann-Feynman gradients are first order in the eigenvector error,
        while the Davidson stopping rule on eigenvalue changes only bounds a
        second-order quantity, so the final solve also requires residual norms
        below ``tolerance``."""
        from .basis import fft_shape, make_bases
        from .pseudo_tables import SpeciesTables
        from .symmetry import fft_factors

        if precision not in ("f64", "mixed"):
            raise ValueError("precision must be 'f64' or 'mixed'")
        self.system = system
        self.precision = precision
        self.tolerance = tolerance
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.bases = make_bases(system.reciprocal, system.kpoints, system.ecutwfc)
        self.shape = fft_shape(self.bases, system.reciprocal, system.ecutrho,
                               fft_factors(system.operations))
        self.grid = ChargeGrid(self.shape, system.reciprocal, system.ecutrho)
        self.tables = {l: SpeciesTables(p, system.volume) for l, p in system.pseudos.items()}
        self.occupied = int(round(system.nelec / 2.0))
        self.q = np.sqrt(self.grid.g2)

    def v_ion(self, positions: np.ndarray) -> tuple[np.ndarray, float]:
        coeff = np.zeros(len(self.grid.g2), dtype=np.complex128)
        for label, table in self.tables.items():
            pos = positions[[i for i, l in enumerate(self.system.labels) if l == label]]
            coeff += table.vloc(self.q) * np.exp(-1j * (self.grid.vectors @ pos.T)).sum(axis=1)
        return np.ascontiguousarray(self.grid.to_r(coeff)), float(np.real(coeff[self.grid.g2 < 1e-14].sum()))

    def solve(self, v_hxc: np.ndarray, positions: np.ndarray):
        """Eigenpairs of every k for the given potential and positions."""
        import copy

        system = copy.copy(self.system)
        system.positions = positions
        v_ion, v0 = self.v_ion(positions)
        v_dev = torch.from_numpy(v_ion + v_hxc).to(self.device)
        rng = QERandom()
        states, energy = [], 0.0
        for basis, weight in zip(self.bases, system.weights):
            state = KPointState(basis, self.shape, self.device)
            state.terms = projector_terms(system, self.tables, state.basis)
            stages = [("f64", self.tolerance)] if self.precision == "f64" else \
                [("f32", max(self.tolerance, 1.0e-6)), ("f64", self.tolerance)]
            sol = None
            for stage, (precision, tolerance) in enumerate(stages):
                ws = state.workspace(precision)
                ham = PlaneWaveHamiltonian(state.basis, None, state.terms, local_workspace=ws,
                                           real_potential=v_dev, potential_average=v0)
                final = stage == len(stages) - 1
                if sol is None:
                    start, eigs, applied = random_starting_subspace(ham, state.basis, rng,
                                                                    system.nbnd)
                else:
                    start, eigs, applied = sol.eigenvectors.to(ham.dtype), None, None
                sol = davidson(ham.apply, ham.diagonal, system.nbnd, initial_vectors=start,
                               tolerance=tolerance, max_iterations=300, subspace_multiplier=4,
                               residual_factor=1.0 if final else None,
                               initial_is_ritz=eigs is not None,
                               initial_is_orthonormal=eigs is not None, initial_eigenvalues=eigs,
                               initial_applied=applied, operator_into=ham.apply_into,
                               dtype=ham.dtype)
            state.vectors = sol.eigenvectors.to(torch.complex128).T.contiguous().T
            state.eigenvalues = np.asarray(sol.eigenvalues)
            energy += float(weight) * 2.0 * float(np.sum(state.eigenvalues[:self.occupied]))
            states.append(state)
        return energy, states, system

    def potential_gradient(self, states) -> np.ndarray:
        """dE/dV(r) = sum w f |psi(r)|^2 / N_r on the (nx, ny, nz) grid."""
        rho = torch.zeros(self.shape, dtype=torch.float64, device=self.device)
        n_r = float(np.prod(self.shape))
        for state, weight in zip(states, self.system.weights):
            ws = state.workspace("f64")
            w = torch.full((self.occupied,), float(weight) * 2.0 / n_r, dtype=torch.float64,
                           device=self.device)
            ws.accumulate_density(rho, state.vectors[:, :self.occupied], w)
        return rho.cpu().numpy()

    def position_gradient(self, states, system, dedv: np.ndarray) -> np.ndarray:
        """dE/dtau: local part from dE/dV, nonlocal part from the projectors."""
        # local: E depends on V_ion(r) = sum_G c(G) e^{iGr} with
        # c(G) = sum_a v(G) e^{-iG tau_a}; dE/dc(G) = sum_r dE/dV(r) e^{iGr}
        n_r = float(np.prod(self.shape))
        dedv_g = self.grid.to_g(dedv) * n_r  # sum_r f(r) e^{-iGr}
        grad = np.zeros((len(system.positions), 3))
        for label, table in self.tables.items():
            vloc = table.vloc(self.q)
            for a in [i for i, l in enumerate(system.labels) if l == label]:
                phase = np.exp(-1j * (self.grid.vectors @ system.positions[a]))
                # dE/dtau = Re sum_G conj(dedv_g) (-i G) v(G) e^{-iG tau}
                grad[a] = np.real((np.conj(dedv_g) * (-1j) * vloc * phase) @ self.grid.vectors)
        grad -= nonlocal_forces(system, states, self.tables, self.occupied)
        return grad


class BandEnergy(torch.autograd.Function):
    """E_band(v_hxc, positions) with a Hellmann-Feynman backward."""

    @staticmethod
    def forward(ctx, v_hxc: torch.Tensor, positions: torch.Tensor, problem: BandProblem):
        energy, states, system = problem.solve(v_hxc.detach().cpu().numpy(),
                                               positions.detach().cpu().numpy())
        ctx.problem, ctx.states, ctx.system = problem, states, system
        ctx.v_shape, ctx.v_dtype, ctx.v_device = v_hxc.shape, v_hxc.dtype, v_hxc.device
        return torch.tensor(energy, dtype=torch.float64, device=v_hxc.device)

    @staticmethod
    def backward(ctx, grad_output: torch.Tensor):
        problem = ctx.problem
        dedv = problem.potential_gradient(ctx.states)
        dedtau = problem.position_gradient(ctx.states, ctx.system, dedv)
        g = float(grad_output)
        grad_v = torch.from_numpy(g * dedv).to(device=ctx.v_device, dtype=ctx.v_dtype)
        grad_tau = torch.from_numpy(g * dedtau).to(device=ctx.v_device, dtype=torch.float64)
        return grad_v, grad_tau, None
