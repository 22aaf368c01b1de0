"""Charge-density grid work of the SCF loop, resident on the GPU.

The per-iteration steps between two Davidson passes -- rho(r) -> rho(G),
the Hartree potential 4 pi rho(G)/G^2, the PZ81 LDA potential, the density
residual metric, plain-Broyden or linear mixing and the energy sums -- run
on the device in FP64 so that neither rho nor V_eff crosses PCIe inside an
iteration (the reference does them on the host: qepy_pw/pw/scf.py:3174-3288,
3830-4020; qepy_pw/mixing.py:413-421, 621-759; _native_fft.pyx:1882-1970).
The 3-D FFTs of the density grid use torch.fft (cuFFT); the pointwise steps
are FP64 tensor arithmetic.
"""

from __future__ import annotations

import math

import numpy as np
import torch


class DeviceChargeGrid:
    """The charge sphere |G|^2 <= ecutrho of an FFT grid, on the device."""

    def __init__(self, host_grid, device) -> None:
        self.shape = host_grid.shape
        self.size = host_grid.size
        self.device = device
        nx, ny, nz = self.shape
        slots = host_grid.slots.astype(np.int64)
        flat = (slots[:, 0] * ny + slots[:, 1]) * nz + slots[:, 2]
        self.flat = torch.from_numpy(flat).to(device)
        self.g2 = torch.from_numpy(np.ascontiguousarray(host_grid.g2)).to(device)
        self.nonzero = self.g2 > 1.0e-14
        self.inv_g2 = torch.where(self.nonzero, 1.0 / torch.where(self.nonzero, self.g2, 1.0),
                                  torch.zeros_like(self.g2))

    def to_g(self, grid: torch.Tensor) -> torch.Tensor:
        """Forward FFT divided by N_r, gathered on the sphere."""
        full = torch.fft.fftn(grid.to(torch.complex128), norm="forward")
        return full.reshape(-1)[self.flat]

    def to_r(self, coefficients: torch.Tensor) -> torch.Tensor:
        """Unnormalised inverse FFT of sphere coefficients (real part)."""
        full = torch.zeros(self.size, dtype=torch.complex128, device=self.device)
        full[self.flat] = coefficients
        return torch.fft.ifftn(full.reshape(self.shape), norm="forward").real.contiguous()

    def hartree(self, rho_g: torch.Tensor) -> torch.Tensor:
        return (4.0 * math.pi) * rho_g * self.inv_g2

    def residual_metric(self, residual_g: torch.Tensor) -> float:
        """sum 4 pi |drho(G)|^2 / G^2 over G != 0 (FP64 tree sum)."""
        terms = (residual_g.real ** 2 + residual_g.imag ** 2) * self.inv_g2
        return 4.0 * math.pi * float(torch.sum(terms))


def pz81(rho: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
    """(eps_xc, v_xc) in Hartree of the unpolarised PZ81 LDA on the device.

    Same formulas and constants as the host version in pseudo_tables.pz81:
    Slater exchange plus Perdew-Zunger (1981) correlation, zero at densities
    at or below 1e-10.
    """
    d = torch.abs(rho)
    active = d > 1.0e-10
    d = torch.clamp(d, min=1.0e-10)
    rs = 0.6203504908994 / torch.pow(d, 1.0 / 3.0)
    eps = -0.687247939924714 * (2.0 / 3.0) / rs
    v = (4.0 / 3.0) * eps
    lnrs = torch.log(rs)
    ec_high = 0.0311 * lnrs - 0.048 + 0.0020 * rs * lnrs - 0.0116 * rs
    vc_high = ec_high - (0.0311 + (0.0020 * (lnrs + 1.0) - 0.0116) * rs) / 3.0
    sq = torch.sqrt(rs)
    den = 1.0 + 1.0529 * sq + 0.3334 * rs
    ec_low = -0.1423 / den
    vc_low = ec_low + (-0.1423 / 3.0) * rs * (0.5 * 1.0529 / sq + 0.3334) / den ** 2
    high = rs < 1.0
    eps = torch.where(active, eps + torch.where(high, ec_high, ec_low), 0.0)
    v = torch.where(active, v + torch.where(high, vc_high, vc_low), 0.0)
    return eps, v


class DeviceBroydenMixer:
    """Broyden mixing of rho(G) in the Coulomb metric, modes 'plain' and 'TF'
    (qepy_pw/mixing.py:262-413, 621-759); history on the device."""

    def __init__(self, grid: DeviceChargeGrid, beta: float, ndim: int, mode: str = "plain",
                 nelec: float | None = None, volume: float | None = None) -> None:
        self.grid = grid
        self.beta = float(beta)
        self.ndim = int(ndim)
        self.active = torch.nonzero(grid.nonzero).reshape(-1)
        self.inv_g2 = grid.inv_g2[self.active]
        self.tf_factor = None
        if mode.lower() == "tf":
            from .scf import thomas_fermi_g2

            g2 = grid.g2[self.active]
            self.tf_factor = g2 / (g2 + thomas_fermi_g2(nelec, volume))
        elif mode.lower() != "plain":
            raise ValueError(f"mixing_mode {mode!r} is not supported")
        self.dx: list[torch.Tensor] = []
        self.df: list[torch.Tensor] = []
        self._next = 0
        self.prev_in = None
        self.prev_res = None

    def reset(self) -> None:
        """Forget the secant history (the next step is linear mixing)."""
        self.dx, self.df = [], []
        self._next = 0
        self.prev_in = self.prev_res = None

    def mix(self, rho_in: torch.Tensor, residual_g: torch.Tensor) -> torch.Tensor:
        current = self.grid.to_g(rho_in)
        cur = current[self.active]
        res = residual_g[self.active]
        saved_in, saved_res = cur.clone(), res.clone()
        if self.prev_in is not None:
            dx, df = self.prev_in - cur, self.prev_res - res
            if len(self.dx) < self.ndim:
                self.dx.append(dx)
                self.df.append(df)
            else:  # cyclic overwrite of one history slot
                self.dx[self._next] = dx
                self.df[self._next] = df
                self._next = (self._next + 1) % self.ndim
        if self.dx:
            dfs = torch.stack(self.df)
            dxs = torch.stack(self.dx)
            weighted = torch.conj(dfs) * self.inv_g2[None, :]
            projection = torch.real(weighted @ res).cpu().numpy()
            gram = torch.real(weighted @ dfs.T).cpu().numpy()
            try:
                gamma = np.linalg.solve(gram, projection)
            except np.linalg.LinAlgError:
                gamma = np.linalg.lstsq(gram, projection, rcond=1.0e-14)[0]
            g = torch.from_numpy(gamma.astype(np.complex128)).to(cur.device)
            cur = cur - g @ dxs
            res = res - g @ dfs
        if self.tf_factor is not None:
            res = res * self.tf_factor
        mixed = current + self.beta * residual_g
        mixed[self.active] = cur + self.beta * res
        zero = ~self.grid.nonzero
        mixed[zero] = current[zero]
        self.prev_in, self.prev_res = saved_in, saved_res
        return self.grid.to_r(mixed)


class DeviceLinearMixer:
    """(1 - beta) rho_in + beta rho_out (qepy_pw/mixing.py:413-421)."""

    def __init__(self, beta: float) -> None:
        self.beta = float(beta)

    def mix(self, rho_in: torch.Tensor, rho_out: torch.Tensor) -> torch.Tensor:
        return (1.0 - self.beta) * rho_in + self.beta * rho_out
