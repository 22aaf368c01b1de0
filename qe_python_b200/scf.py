"""Self-consistent field driver on the B200 H|psi> / Davidson path.

Restates the reference's SCF loop (qepy_pw/pw/scf.py:_run_scf, :1997-4375)
for the benchmark cells' feature set: norm-conserving pseudopotentials
without core correction, LDA (PZ81), no spin, fixed or broadened
(smeared) occupations, Davidson,
linear or plain-Broyden density mixing, symmetry-reduced k points.  Each
k point's Hamiltonian and Davidson solve run on the GPU (PlaneWaveHamiltonian,
davidson); the density is accumulated by the GPU FFT kernels; the charge-grid
steps (Hartree, XC, mixing, energies) stay on the device in FP64
(qe_python_b200.charge), where the reference runs them on the host.

Precision schedules:
  'f64'    plain FP64 everywhere on the GPU;
  'mixed'  chosen form: FP32 FFT passes and split-TF32 projector GEMMs
           until the density residual falls below ``switch_ry``, then FP64
           H|psi> for the remaining iterations (eigenvalues, energies and the
           density accumulation are always FP64).
Energies are Hartree internally; SCFResult reports both units.
"""

from __future__ import annotations

import ctypes
import threading
import time
from dataclasses import dataclass, field

import numpy as np
import scipy.fft
import torch

from . import _lib
from . import kernels as K
from .basis import LocalPotentialWorkspace, fft_shape, make_bases
from .configs import DIAMOND_CUBIC, displacements, supercell
from .device import empty_f, leading_dimension, require_cuda, stream_handle, to_device_f
from .diagonalization import (
    OVERLAP,
    PlaneWaveHamiltonian,
    apply_hamiltonians,
    davidson,
    davidson_steps,
    lowest_generalized_eigh,
    refined_davidson_steps,
    run_lockstep,
    RoundGraphs,
)
from .pseudo import SyntheticPseudo, synthetic_pseudo
from .charge import DeviceBroydenMixer, DeviceChargeGrid, DeviceLinearMixer
from .charge import pz81 as device_pz81
from .occupations import fixed_occupations, smeared_occupations, smearing_order
from .pseudo_tables import SpeciesTables, device_projectors, ewald_energy, pz81
from .symmetry import (
    DensitySymmetrizer,
    Operation,
    fft_factors,
    mesh_compatible,
    monkhorst_pack,
    reduce_kpoints,
    space_group,
)


@dataclass
class System:
    """A periodic cell and the SCF controls (Hartree internally)."""

    lattice: np.ndarray          # rows = lattice vectors (bohr)
    positions: np.ndarray        # cartesian atom positions (bohr)
    labels: list[str]
    pseudos: dict[str, SyntheticPseudo]
    ecutwfc: float               # Ry
    ecutrho: float               # Ry
    nbnd: int
    kpoints: np.ndarray          # crystal coordinates
    weights: np.ndarray          # sum to 1
    operations: list[Operation]
    conv_thr: float = 1.0e-8     # Ry
    mixing_mode: str = "plain"
    mixing_beta: float = 0.7
    mixing_ndim: int = 8
    diago_david_ndim: int = 2
    maxiter: int = 100
    forces: bool = False
    stress: bool = False         # analytic stress at convergence (tstress)
    name: str = ""
    occupations: str = "fixed"   # or "smearing"
    smearing: str = "gaussian"
    degauss: float = 0.0         # Ry

    @property
    def volume(self) -> float:
        return abs(float(np.linalg.det(self.lattice)))

    @property
    def reciprocal(self) -> np.ndarray:
        return 2.0 * np.pi * np.linalg.inv(self.lattice).T

    @property
    def nelec(self) -> float:
        return float(sum(self.pseudos[l].z_valence for l in self.labels))


def benchmark_system(name: str) -> System:
    """The benchmark cells of qe_python_b200.configs as System objects."""
    pseudo = synthetic_pseudo("X")
    smear = ("fixed", "gaussian", 0.0)
    if name in ("scf-fcc2", "scf-fcc2-smear"):
        a = 10.26
        lattice = a / 2.0 * np.array([[-1.0, 0.0, 1.0], [0.0, 1.0, 1.0], [-1.0, 1.0, 0.0]])
        positions = np.array([[0.0, 0.0, 0.0], [0.25, 0.25, 0.25]]) * a
        grid, shift, ecut, ecutrho, nbnd = (4, 4, 4), (1, 1, 1), 20.0, 80.0, 8
        mixing, forces = "linear", False
        if name == "scf-fcc2-smear":
            mixing, smear = "plain", ("smearing", "marzari-vanderbilt", 0.02)
    elif name == "scf-dia64":
        lattice = np.eye(3) * 20.52
        positions = supercell(DIAMOND_CUBIC, 2) * 20.52
        grid, shift, ecut, ecutrho, nbnd = (2, 2, 2), (0, 0, 0), 30.0, 180.0, 160
        mixing, forces = "TF", False
        smear = _supercell_smearing()
    elif name == "scf-dia8-disp":
        a = 10.26
        lattice = np.eye(3) * a
        positions = DIAMOND_CUBIC * a + displacements(8, 0.05)
        grid, shift, ecut, ecutrho, nbnd = (3, 3, 3), (0, 0, 0), 25.0, 100.0, 24
        mixing, forces = "plain", True
    elif name == "scf-dia216":
        a = 30.78
        lattice = np.eye(3) * a
        positions = supercell(DIAMOND_CUBIC, 3) * a + displacements(216, 0.03)
        grid, shift, ecut, ecutrho, nbnd = None, None, 30.0, 180.0, 480
        mixing, forces = "TF", True
        smear = _supercell_smearing()
    else:
        raise KeyError(name)
    labels = ["X"] * len(positions)
    frac = positions @ np.linalg.inv(lattice)
    ops = space_group(lattice, frac, labels)
    if grid is None:  # Gamma only: the space group is used as found
        kpoints, weights = np.zeros((1, 3)), np.ones(1)
    else:
        points, w = monkhorst_pack(grid, shift)
        ops = mesh_compatible(points, ops)
        kpoints, weights, _ = reduce_kpoints(points, w, ops)
    return System(lattice, positions, labels, {"X": pseudo}, ecut, ecutrho, nbnd, kpoints, weights,
                  ops, mixing_mode=mixing, forces=forces, name=name, occupations=smear[0],
                  smearing=smear[1], degauss=smear[2])


def _supercell_smearing() -> tuple[str, str, float]:
    from .configs import SUPERCELL_SMEARING as s

    return s["occupations"], s["smearing"], float(s["degauss"])


# ---------------------------------------------------------------------------
# host pieces of the loop

class QERandom:
    """QE randy stream (qepy_pw/pw/scf.py:452-538); pairs drawn by the host
    routine qeb_qe_random_pairs of libqeb200.so."""

    M, A, C, NT = 714025, 1366, 150889, 97

    def __init__(self, seed: int = 0) -> None:
        s = min(abs(int(seed)), self.C)
        s = (self.C - s) % self.M
        self.table = np.empty(self.NT, dtype=np.int64)
        for i in range(self.NT):
            s = (self.A * s + self.C) % self.M
            self.table[i] = s
        s = (self.A * s + self.C) % self.M
        self.seed = s
        self.current = s

    def pairs(self, plane_waves: int, bands: int) -> tuple[np.ndarray, np.ndarray]:
        first = np.empty((plane_waves, bands), order="F")
        second = np.empty((plane_waves, bands), order="F")
        cur = ctypes.c_int64(self.current)
        seed = ctypes.c_int64(self.seed)
        _lib.check("qeb_qe_random_pairs", _lib.load().qeb_qe_random_pairs(
            plane_waves, bands, self.table.ctypes.data, ctypes.byref(cur), ctypes.byref(seed),
            first.ctypes.data, second.ctypes.data))
        self.current, self.seed = int(cur.value), int(seed.value)
        return first, second

    def draws(self, plane_waves: int, bands: int) -> tuple[np.ndarray, np.ndarray]:
        """The next pairs as the stream's integer values (each draw times
        714025; int32, column-major): ``pairs`` divided on the device."""
        first = np.empty((plane_waves, bands), dtype=np.int32, order="F")
        second = np.empty((plane_waves, bands), dtype=np.int32, order="F")
        cur = ctypes.c_int64(self.current)
        seed = ctypes.c_int64(self.seed)
        _lib.check("qeb_qe_random_draws", _lib.load().qeb_qe_random_draws(
            plane_waves, bands, self.table.ctypes.data, ctypes.byref(cur), ctypes.byref(seed),
            first.ctypes.data, second.ctypes.data))
        self.current, self.seed = int(cur.value), int(seed.value)
        return first, second


class StartingDraws:
    """The random pairs of every k point's starting wavefunctions, drawn in
    k-point order from one QE stream on a host thread while the SCF set-up
    runs.  The stream is sequential (each draw picks the shuffle-table
    entry of the previous one): the 2 x 504 x 80 725 draws of the 216-atom
    cell take 0.5-0.7 s of one core, which the thread hides behind the
    set-up; the ctypes call releases the GIL.  ``take(k)`` waits for k's
    draws; those of k points outside ``keep`` (another pool's) only advance
    the stream."""

    def __init__(self, rng: QERandom, sizes, bands: int, keep=None) -> None:
        sizes = [int(v) for v in sizes]
        keep = set(range(len(sizes))) if keep is None else set(keep)
        self._ready = [threading.Event() for _ in sizes]
        self._draws: list = [None] * len(sizes)
        self._error: BaseException | None = None
        _lib.load()

        def run() -> None:
            try:
                for k, npw in enumerate(sizes):
                    pair = rng.draws(npw, bands)
                    self._draws[k] = pair if k in keep else None
                    self._ready[k].set()
            except BaseException as exc:  # re-raised by take()
                self._error = exc
                for event in self._ready:
                    event.set()

        self._thread = threading.Thread(target=run, name="qe-random-draws", daemon=True)
        self._thread.start()

    def take(self, k: int) -> tuple[np.ndarray, np.ndarray]:
        self._ready[k].wait()
        if self._error is not None:
            raise RuntimeError("random starting draws failed") from self._error
        pair, self._draws[k] = self._draws[k], None
        if pair is None:
            raise RuntimeError(f"the draws of k point {k} were not kept or were already taken")
        return pair


class ChargeGrid:
    """Charge-density sphere on the FFT grid (qepy_pw/pw/scf.py:268-321)."""

    def __init__(self, shape, reciprocal: np.ndarray, cutoff_ry: float) -> None:
        self.shape = tuple(int(v) for v in shape)
        axes = [np.rint(np.fft.fftfreq(n) * n).astype(np.int32) for n in self.shape]
        metric = reciprocal @ reciprocal.T
        x, y, z = axes[0][:, None, None], axes[1][None, :, None], axes[2][None, None, :]
        # |G|^2 summed term by term in place (the same additions in the same
        # order as one expression, without its full-grid temporaries)
        g2 = np.empty(self.shape)
        np.add(metric[0, 0] * x * x + metric[1, 1] * y * y, metric[2, 2] * z * z, out=g2)
        g2 += 2.0 * metric[0, 1] * x * y
        g2 += 2.0 * metric[0, 2] * x * z
        g2 += 2.0 * metric[1, 2] * y * z
        # C-order grid points inside the sphere (argwhere's order)
        inside = g2 <= cutoff_ry + 1.0e-12
        i0, i1, i2 = np.nonzero(inside)
        self.slots = np.empty((i0.size, 3), dtype=np.int32)
        self.slots[:, 0], self.slots[:, 1], self.slots[:, 2] = i0, i1, i2
        self.index = tuple(self.slots.T)
        self.miller = np.empty((i0.size, 3), dtype=np.int32)
        self.miller[:, 0], self.miller[:, 1], self.miller[:, 2] = axes[0][i0], axes[1][i1], axes[2][i2]
        self.vectors = self.miller @ reciprocal
        self.g2 = g2[inside]
        self.size = int(np.prod(self.shape))

    def to_g(self, grid: np.ndarray) -> np.ndarray:
        """Forward FFT divided by N_r, gathered on the sphere."""
        return scipy.fft.fftn(grid, workers=-1)[self.index] / self.size

    def to_r(self, coefficients: np.ndarray) -> np.ndarray:
        """Unnormalised inverse FFT of sphere coefficients (real part)."""
        full = np.zeros(self.shape, dtype=np.complex128)
        full[self.index] = coefficients
        return np.real(scipy.fft.ifftn(full, norm="forward", workers=-1))


def hartree(rho_g: np.ndarray, g2: np.ndarray) -> np.ndarray:
    out = np.zeros_like(rho_g)
    mask = g2 > 1.0e-14
    out[mask] = 4.0 * np.pi * rho_g[mask] / g2[mask]
    return out


def neumaier_metric(residual: np.ndarray, g2: np.ndarray) -> float:
    """sum 4 pi |drho(G)|^2 / G^2 with Neumaier compensation (_native_fft.pyx:1922-1970)."""
    mask = g2 > 1.0e-14
    terms = 4.0 * np.pi * (residual[mask].real ** 2 + residual[mask].imag ** 2) / g2[mask]
    total = 0.0
    correction = 0.0
    for t in terms.tolist():
        u = total + t
        correction += (total - u) + t if total >= t else (t - u) + total
        total = u
    return total + correction


def thomas_fermi_g2(nelec: float, volume: float) -> float:
    """Thomas-Fermi screening wavevector squared (bohr^-2) of the uniform
    electron gas of the cell's mean density (qepy_pw/mixing.py:51-59)."""
    if not nelec or nelec <= 0.0 or not volume or volume <= 0.0:
        raise ValueError("Thomas-Fermi mixing needs a positive nelec and volume")
    rs = (3.0 * volume / (4.0 * np.pi * nelec)) ** (1.0 / 3.0)
    return float((12.0 / np.pi) ** (2.0 / 3.0) / rs)


class BroydenMixer:
    """Broyden mixing of rho(G) in the Coulomb metric (qepy_pw/mixing.py:
    262-413, modes 'plain' and 'TF'; 'TF' scales the updated residual by
    G^2 / (G^2 + k_TF^2) before the linear step)."""

    def __init__(self, grid: ChargeGrid, beta: float, ndim: int, cutoff_ry: float,
                 mode: str = "plain", nelec: float | None = None,
                 volume: float | None = None) -> None:
        self.grid = grid
        self.beta = float(beta)
        self.ndim = int(ndim)
        active = grid.g2 > 1.0e-14
        active &= grid.g2 <= cutoff_ry + 1.0e-12
        self.active = np.flatnonzero(active)
        self.g2 = grid.g2[self.active]
        self.tf_factor = None
        if mode.lower() == "tf":
            ks2 = thomas_fermi_g2(nelec, volume)
            self.tf_factor = self.g2 / (self.g2 + ks2)
        elif mode.lower() != "plain":
            raise ValueError(f"mixing_mode {mode!r} is not supported")
        self.dx: list[np.ndarray] = []
        self.df: list[np.ndarray] = []
        self._next = 0
        self.prev_in = None
        self.prev_res = None

    def _push(self, store: list, value: np.ndarray) -> None:
        if len(store) < self.ndim:
            store.append(value)

    def mix(self, rho_in: np.ndarray, residual_g: np.ndarray) -> np.ndarray:
        current = self.grid.to_g(rho_in)
        cur = current[self.active].copy()
        res = residual_g[self.active].copy()
        saved_in, saved_res = cur.copy(), res.copy()
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
            dfs = np.array(self.df)
            dxs = np.array(self.dx)
            weighted = np.conj(dfs) / self.g2[None, :]
            projection = np.real(weighted @ res)
            gram = np.real(weighted @ dfs.T)
            try:
                gamma = np.linalg.solve(gram, projection)
            except np.linalg.LinAlgError:
                gamma = np.linalg.lstsq(gram, projection, rcond=1.0e-14)[0]
            cur -= gamma @ dxs
            res -= gamma @ dfs
        if self.tf_factor is not None:
            res *= self.tf_factor
        mixed = current + self.beta * residual_g
        mixed[self.active] = cur + self.beta * res
        zero = np.flatnonzero(self.grid.g2 <= 1.0e-14)
        mixed[zero] = current[zero]
        self.prev_in, self.prev_res = saved_in, saved_res
        return self.grid.to_r(mixed)


class LinearMixer:
    def __init__(self, beta: float) -> None:
        self.beta = float(beta)

    def mix(self, rho_in: np.ndarray, rho_out: np.ndarray) -> np.ndarray:
        return (1.0 - self.beta) * rho_in + self.beta * rho_out


@dataclass
class SCFResult:
    converged: bool
    total_energy_ha: float
    iterations: int
    energies_ha: list[float]
    accuracies_ha: list[float]
    eigenvalues_ha: list[np.ndarray]
    energy_terms_ha: dict[str, float]
    density: np.ndarray
    forces_ha_per_bohr: np.ndarray | None
    wall_seconds: float
    precision_log: list[str] = field(default_factory=list)
    davidson_iterations: list[float] = field(default_factory=list)
    timings: dict[str, float] = field(default_factory=dict)
    occupations: list[np.ndarray] = field(default_factory=list)
    fermi_energy_ha: float | None = None
    # the last iteration's input V_eff(r) (device, C-order) and each local k
    # point's eigenvectors (device, complex128, nbnd + guard columns)
    potential: "torch.Tensor | None" = None
    eigenvectors: list = field(default_factory=list)
    # analytic stress and its symmetrised terms (Ha/bohr^3) when asked for
    stress_ha_per_bohr3: np.ndarray | None = None
    stress_terms: "object | None" = None

    @property
    def total_energy_ry(self) -> float:
        return 2.0 * self.total_energy_ha


class KPointState:
    """Per-k device objects reused across SCF iterations."""

    def __init__(self, basis, shape, device) -> None:
        self.basis = basis.materialize() if basis.catalog is not None else basis
        self.workspaces: dict[str, LocalPotentialWorkspace] = {}
        self.shape = shape
        self.device = device
        self.vectors: torch.Tensor | None = None
        self.eigenvalues: np.ndarray | None = None
        self.terms = None
        # projector operands on the device per precision (fixed ions)
        self.device_projectors: dict = {}
        # refined Davidson: (lam, R, V) with H(V) X = X lam + R for X = vectors
        self.refined = None

    def workspace(self, precision: str) -> LocalPotentialWorkspace:
        if precision not in self.workspaces:
            self.workspaces[precision] = LocalPotentialWorkspace(
                self.basis, self.shape, precision=precision, device=self.device)
        return self.workspaces[precision]


def gpu_structure_factor(vectors: np.ndarray, positions: np.ndarray,
                         weights: np.ndarray) -> np.ndarray:
    """S(G) = sum_a w_a exp(-i G.tau_a) in FP64 on the device (set-up of large
    cells: one complex exponential per G vector and atom)."""
    device = torch.device("cuda", torch.cuda.current_device())
    g = torch.from_numpy(np.ascontiguousarray(vectors)).to(device)
    pos = torch.from_numpy(np.ascontiguousarray(positions)).to(device)
    w = torch.from_numpy(np.asarray(weights, dtype=np.float64)).to(device).to(torch.complex128)
    out = torch.zeros(len(vectors), dtype=torch.complex128, device=device)
    for a0 in range(0, len(positions), 32):
        out += torch.exp(-1j * (g @ pos[a0:a0 + 32].T)) @ w[a0:a0 + 32]
    return out.cpu().numpy()


def _as128(t: torch.Tensor) -> torch.Tensor:
    return t if t.dtype == torch.complex128 else t.to(torch.complex128).T.contiguous().T


def random_starting_subspace(ham: PlaneWaveHamiltonian, basis, source, nbnd: int):
    """Random trial vectors amp e^(2 pi i phase) / (1 + |k+G|^2) rotated by a
    Rayleigh-Ritz step in their span (qepy_pw/pw/scf.py:853-870, 923-953).
    ``source`` is a QERandom (drawn now) or the (first, second) integer
    draws of this k point (QERandom.draws, StartingDraws.take).  Returns
    (vectors, eigenvalues, H vectors) in the Hamiltonian's dtype."""
    if isinstance(source, QERandom):
        source = source.draws(len(basis), nbnd)
    first, second = source
    npw = len(basis)
    if first.shape != (npw, nbnd) or second.shape != (npw, nbnd):
        raise ValueError("the random draws do not match the basis and the band count")
    # the trial vectors are formed on the device (qeb_random_trials): the
    # host sends the 32-bit draws, a quarter of the complex128 trial bytes
    device = ham.device
    first_d = torch.from_numpy(first.ravel(order="F")).to(device)
    second_d = torch.from_numpy(second.ravel(order="F")).to(device)
    kinetic = torch.from_numpy(np.ascontiguousarray(basis.kinetic, dtype=np.float64)).to(device)
    trials_dev = empty_f(npw, nbnd, ham.dtype, device)
    _lib.check("qeb_random_trials", _lib.load().qeb_random_trials(
        npw, nbnd, first_d.data_ptr(), second_d.data_ptr(), kinetic.data_ptr(),
        trials_dev.data_ptr(), leading_dimension(trials_dev),
        1 if ham.dtype == torch.complex64 else 0, stream_handle()))
    del first_d, second_d, kinetic
    applied = ham.apply(trials_dev)
    t128, a128 = _as128(trials_dev), _as128(applied)
    proj = K.gemm(K.OP_C, t128, a128)
    over = K.gemm(K.OP_C, t128, t128)
    values, rot = lowest_generalized_eigh(0.5 * (proj + proj.conj().T),
                                          0.5 * (over + over.conj().T), nbnd)
    vectors = K.gemm(K.OP_N, t128, rot.T.contiguous().T)
    hvectors = K.gemm(K.OP_N, a128, rot.T.contiguous().T)
    if ham.dtype != torch.complex128:
        vectors = vectors.to(ham.dtype).T.contiguous().T
        hvectors = hvectors.to(ham.dtype).T.contiguous().T
    return vectors, values.cpu().numpy(), hvectors


def projector_terms(system: System, tables: dict, basis) -> tuple:
    """(beta, coupling) per species with atom phases packed
    (qepy_pw/pw/scf.py:596-718)."""
    from .diagonalization import FactorizedProjectorTerm

    vectors = basis.vectors
    terms = []
    for label, table in tables.items():
        pos = np.array([p for p, l in zip(system.positions, system.labels) if l == label])
        if not len(pos) or table.channels == 0:
            continue
        # init_us_2 on the device: radial interpolation, Y_lm and (-i)^l
        # (qeb_projector_basis), then exp(-i (k+G).tau) for every atom
        device = require_cuda()
        vectors_dev = torch.from_numpy(np.ascontiguousarray(vectors)).to(device)
        beta, coupling = device_projectors(table, vectors_dev)
        angle = vectors_dev @ torch.from_numpy(np.ascontiguousarray(pos.T)).to(device)
        phases = to_device_f(torch.polar(torch.ones_like(angle), -angle), torch.complex128,
                             device)
        del angle, vectors_dev
        terms.append(FactorizedProjectorTerm(beta, phases, coupling))
    return tuple(terms)


@dataclass
class SCFSetup:
    """Fixed-ion pieces of an SCF: bases, FFT grid, charge sphere, species
    tables and the ionic local potential (qepy_pw/pw/scf.py:2193-2330)."""

    bases: list
    shape: tuple
    grid: ChargeGrid
    cgrid: DeviceChargeGrid
    tables: dict
    v_ion: torch.Tensor          # V_ion(r), C-order (nx, ny, nz) float64 on the device
    v_ion_average: float         # its G = 0 component (QE v_of_0)


def scf_setup(system: System, device, on_bases=None) -> SCFSetup:
    """Bases of every k point, the FFT grid by the reference's rule, the
    charge sphere and V_ion(r) = sum_species V_loc(|G|) S(G).
    ``on_bases(bases)``, when given, runs as soon as the bases exist (the
    SCF starts its random draws there)."""
    reciprocal = system.reciprocal
    bases = make_bases(reciprocal, system.kpoints, system.ecutwfc)
    if on_bases is not None:
        on_bases(bases)
    shape = fft_shape(bases, reciprocal, system.ecutrho, fft_factors(system.operations))
    grid = ChargeGrid(shape, reciprocal, system.ecutrho)
    tables = {label: SpeciesTables(p, system.volume) for label, p in system.pseudos.items()}
    q = np.sqrt(grid.g2)
    v_ion_g = np.zeros(len(grid.g2), dtype=np.complex128)
    for label, table in tables.items():
        pos = np.array([p for p, l in zip(system.positions, system.labels) if l == label])
        structure = gpu_structure_factor(grid.vectors, pos, np.ones(len(pos)))
        v_ion_g += table.vloc(q) * structure
    cgrid = DeviceChargeGrid(grid, device)
    v_ion = cgrid.to_r(torch.from_numpy(v_ion_g).to(device))
    v_ion_average = float(np.real(np.sum(v_ion_g[grid.g2 < 1.0e-14])))
    return SCFSetup(bases, tuple(shape), grid, cgrid, tables, v_ion, v_ion_average)


def starting_density(system: System, setup: SCFSetup) -> torch.Tensor:
    """Uniform starting density rho = nelec / Omega (no PP_RHOATOM,
    qepy_pw/pw/scf.py:1004-1012)."""
    return torch.full(setup.shape, system.nelec / system.volume, dtype=torch.float64,
                      device=setup.v_ion.device)


def hxc_potential(setup: SCFSetup, rho: torch.Tensor) -> torch.Tensor:
    """V_H(r) + V_xc(r) of a density (Hartree 4 pi rho(G)/G^2, PZ81 LDA)."""
    cgrid = setup.cgrid
    vh = cgrid.to_r(cgrid.hartree(cgrid.to_g(rho)))
    _eps, vxc = device_pz81(rho)
    return vh + vxc


def starting_hamiltonians(system: System, precision: str = "f64", setup: SCFSetup | None = None):
    """The first SCF iteration's Hamiltonian of every k point: V_eff =
    V_ion + V_H + V_xc of the uniform starting density and the projector
    terms of the fixed ions (the operator the reference hands to Davidson at
    qepy_pw/pw/scf.py:3396-3411, 3510 in its first iteration).  Returns
    (hamiltonians, V_eff(r) on the device, setup)."""
    device = require_cuda()
    setup = setup if setup is not None else scf_setup(system, device)
    v_eff = setup.v_ion + hxc_potential(setup, starting_density(system, setup))
    hams = []
    for basis in setup.bases:
        state = KPointState(basis, setup.shape, device)
        terms = projector_terms(system, setup.tables, state.basis)
        hams.append(PlaneWaveHamiltonian(state.basis, None, terms,
                                         local_workspace=state.workspace(precision),
                                         real_potential=v_eff,
                                         potential_average=setup.v_ion_average))
    return hams, v_eff, setup


MIN_FP64_ITERATIONS = 3  # mixed form: FP64 iterations before convergence is accepted
GRAPH_ROUNDS_DEFAULT = False  # mixed form: batched k-point rounds from CUDA graphs
MIXED_GUARD_BANDS = 24  # mixed form: extra Davidson roots beyond nbnd (run_scf guard_bands)
REFINED_FLOOR_RATIO = 1.0e-3  # refined iterations: Davidson threshold >= ratio x conv_thr (Ry -> Ha)


def _k_point_solve(ham, system, start_vectors, initial_eigs, initial_applied, tol, occ_roots,
                   is_ritz, timers, lock=False, nroots=None, refined=False, carried=None,
                   overlap=False):
    """One k point's diagonalisation as a generator of H applications: the
    Davidson of qepy_pw/pw/scf.py:3496-3556 (20 iterations), repeated up to
    five more times from its last vectors while more than five roots remain
    unconverged.  ``refined``: the chosen form's FP64-accurate Davidson
    (``refined_davidson_steps``: FP64 block, FP32 corrections), started
    from ``carried`` = (lam, R) when given; the final (lam, R) are left in
    ``carried_out``.  ``overlap``: the solves yield OVERLAP around their
    reduced eigensolves (lockstep k points).  Returns (DavidsonResult,
    Davidson iterations, carried_out)."""
    attempt, total_its = 0, 0.0
    vectors, eigs, applied = start_vectors, initial_eigs, initial_applied
    carried_out: dict = {}
    while True:
        if refined:
            sol = yield from refined_davidson_steps(
                ham.diagonal, nroots or system.nbnd, initial_vectors=vectors, tolerance=tol,
                max_iterations=20, subspace_multiplier=system.diago_david_ndim,
                occupied_roots=occ_roots, timers=timers, initial_state=carried,
                state_out=carried_out, overlap_solves=overlap)
            carried = (None if carried_out["residual"] is None
                       else (carried_out["lam"], carried_out["residual"], carried_out["error"]))
        else:
            sol = yield from davidson_steps(
                ham.diagonal, nroots or system.nbnd, initial_vectors=vectors, tolerance=tol,
                max_iterations=20,
                subspace_multiplier=system.diago_david_ndim, residual_factor=None,
                residual_energy_scale=None, occupied_roots=occ_roots, initial_is_ritz=is_ritz,
                initial_is_orthonormal=True, initial_eigenvalues=eigs, initial_applied=applied,
                timers=timers, dtype=ham.dtype, lock_converged=lock, overlap_solves=overlap)
        attempt += 1
        total_its += sol.iterations
        if sol.converged or sol.number_unconverged <= 5 or attempt >= 6:
            return sol, total_its, carried_out
        vectors, eigs, applied = sol.eigenvectors, sol.eigenvalues, None


def _drive(steps, ham, ham32=None):
    """Run a generator of H applications with one Hamiltonian (complex64
    requests go to ``ham32`` when given: the refined Davidson's FP32
    corrections)."""
    try:
        request = next(steps)
        while True:
            if request is not OVERLAP:
                target = ham32 if ham32 is not None and request[0].dtype == torch.complex64 else ham
                target.apply_into(*request)
            request = steps.send(None)
    except StopIteration as done:
        return done.value


def _apply_by_dtype(hams, hams32, requests, graphs=None) -> None:
    """Batched H applications of a lockstep round: complex128 requests with
    ``hams`` and complex64 ones with ``hams32`` (when given), each group in
    one launch per FFT pass; the complex64 group through ``graphs`` (a
    RoundGraphs) when given."""
    groups: dict = {}
    for request in requests:
        groups.setdefault(request[1].dtype, []).append(request)
    for dtype, group in groups.items():
        if graphs is not None and dtype == torch.complex64:
            graphs(group)
            continue
        table = hams32 if hams32 is not None and dtype == torch.complex64 else hams
        apply_hamiltonians(table, group)


def run_scf(system: System, precision: str = "f64", switch_ry: float = 1.0e-5,
            progress=None, timers=None, pools=None, fp32_floor: float = 5.0e-7,
            batch_kpoints: bool | None = None, lock_converged: bool | None = None,
            guard_bands: int | None = None, restart_mixer_at_switch: bool = False,
            fp64_phase: str = "refined", eigenvalue_change_ry: float = 1.0e-6,
            graph_rounds: bool | None = None, refined_floor: float | None = None) -> SCFResult:
    """Converge the Kohn-Sham density to ``system.conv_thr`` (Ry) on the GPU.

    ``timers``: optional object with a ``measure(name)`` context manager,
    handed to the Hamiltonian and Davidson (the reference's timer names).
    ``pools``: optional qe_python_b200.pools.KPointPools; each rank then
    solves its own k points and the density, eigenvalues and nonlocal
    forces are combined over the pools.  ``batch_kpoints`` (default: on for
    the mixed form) runs the k points' Davidson solves in lockstep with one
    launch per FFT pass for all of them; the results are those of the
    k-by-k loop.  ``lock_converged`` (off unless asked for) locks the
    converged roots at each Davidson restart (``davidson_steps``; the
    reference never locks).  On the 216-atom cell it made each Davidson
    iteration cheaper, but the locked vectors, frozen at the Davidson
    threshold, held the FP32 iterations near dr2 = 5e-5 Ry and the SCF took
    more iterations overall.

    Mixed form: ``fp32_floor`` (Ha) bounds the Davidson threshold of the
    FP32 iterations from below; ``restart_mixer_at_switch`` drops the
    Broyden history when H|psi> turns FP64.  ``fp64_phase`` picks the
    iterations after the switch: 'refined' (default) solves with
    ``refined_davidson_steps`` (FP64 Ritz block, chosen-form H and GEMMs
    for the corrections) and accepts convergence once 2 dr2 < conv_thr in a
    refined iteration whose eigenvalues moved less than
    ``eigenvalue_change_ry`` from the previous iteration's, with its
    Davidson threshold held at or above ``refined_floor`` Ha (default
    REFINED_FLOOR_RATIO x conv_thr: measured on the 216- and 64-atom cells,
    1e-11 Ha changed no SCF iteration count and no eigenvalue at the fixed
    potential by more than 1e-11 Ry, and took the 216-atom SCF from 5.23 to
    4.78 s; 1e-10 Ha cost the 64-atom cell three more iterations); 'f64' runs the
    plain FP64 Davidson there and accepts convergence after
    MIN_FP64_ITERATIONS such iterations.  ``graph_rounds`` replays the
    chosen-form H applications of the batched k-point rounds from CUDA
    graphs (diagonalization.RoundGraphs; off when ``timers`` are given, as
    their synchronisation cannot be captured).  Measured on the 216-atom Gamma
    cell and the 64-atom 4-k cell (SCF to 1e-8 Ry): a 5e-7 Ha floor with
    the history kept took 19 and 13 iterations (6.7 s, 4.0 s) where a
    2e-6 Ha floor with the restart took 20 and 17 (8.2-8.7 s, 4.6 s); the
    energies, eigenvalues and forces differed from the plain form's by the
    same amounts.  Floors of 3e-7, 2e-7 and 1e-7 Ha took 20-23 iterations
    on the 216-atom cell."""
    if batch_kpoints is None:
        batch_kpoints = precision == "mixed"
    if graph_rounds is None:
        graph_rounds = GRAPH_ROUNDS_DEFAULT and precision == "mixed"
    graph_rounds = bool(graph_rounds) and timers is None
    round_graphs = None
    lock_converged = bool(lock_converged)
    # ``guard_bands`` (chosen form): Davidson solves nbnd + guard roots, the
    # guard roots at the loose threshold of empty bands; only the nbnd
    # requested bands enter occupations, density and energies.  Under
    # smearing every requested band converges to the tight threshold, and a
    # multiplet cut by the last one converges slowly; with fixed occupations
    # the empty requested bands already play that part.  Default: on for the
    # mixed form with smearing.  The plain form solves exactly nbnd roots, as
    # the reference does.
    if guard_bands is None:
        guard_bands = MIXED_GUARD_BANDS if (precision == "mixed"
                                            and system.occupations == "smearing") else 0
    guard_bands = max(0, int(guard_bands))
    if precision not in ("f64", "mixed"):
        raise ValueError("precision must be 'f64' or 'mixed'")
    if fp64_phase not in ("refined", "f64"):
        raise ValueError("fp64_phase must be 'refined' or 'f64'")
    device = require_cuda()
    started = time.perf_counter()
    timings: dict[str, float] = {}

    def tick(name, t0):
        timings[name] = timings.get(name, 0.0) + time.perf_counter() - t0

    t0 = time.perf_counter()
    volume = system.volume
    nelec = system.nelec
    occupied = int(round(nelec / 2.0))
    smeared = system.occupations == "smearing"
    if smeared:
        if system.degauss <= 0.0:
            raise ValueError("smearing requires a positive degauss")
        order = smearing_order(system.smearing)
    elif system.occupations != "fixed":
        raise ValueError(f"occupations {system.occupations!r} are not supported")
    elif system.nbnd < occupied:
        raise ValueError("nbnd is smaller than the number of occupied states")
    fermi = None
    draws = {}

    def start_draws(bases) -> None:
        # the first iteration's random pairs of every k point, drawn on a
        # host thread during the rest of the set-up
        nk_all = len(bases)
        keep = list(pools.local_kpoints(nk_all)) if pools is not None else None
        bands = min(system.nbnd + guard_bands, min(len(b) for b in bases))
        draws["all"] = StartingDraws(QERandom(), [len(b) for b in bases], bands, keep)

    setup = scf_setup(system, device, on_bases=start_draws)
    bases, shape, grid, cgrid = setup.bases, setup.shape, setup.grid, setup.cgrid
    tables, v_ion, v_ion_average = setup.tables, setup.v_ion, setup.v_ion_average
    if min(len(b) for b in bases) < system.nbnd:
        raise ValueError("nbnd exceeds the smallest plane-wave basis")
    nsolve = min(system.nbnd + guard_bands, min(len(b) for b in bases))
    charges = np.array([system.pseudos[l].z_valence for l in system.labels])
    e_ion = ewald_energy(system.lattice, system.positions, charges, system.ecutrho,
                         structure=gpu_structure_factor)
    rho = starting_density(system, setup)
    symmetrizer = DensitySymmetrizer(system.operations, shape) if len(system.operations) > 1 else None
    mixer = (DeviceLinearMixer(system.mixing_beta) if system.mixing_mode == "linear"
             else DeviceBroydenMixer(cgrid, system.mixing_beta, system.mixing_ndim,
                                     system.mixing_mode, nelec, volume))
    states = [KPointState(b, shape, device) for b in bases]
    nk = len(states)
    local_k = list(pools.local_kpoints(nk)) if pools is not None else list(range(nk))
    davidson_tolerance = 0.5 * 1.0e-2  # diago_thr_init 1e-2 Ry -> Ha
    previous_accuracy = np.inf
    first_diagonalization = True
    input_hxc = None
    energies, accuracies, precision_log, david_its = [], [], [], []
    previous_eigenvalues = None
    energy_terms: dict[str, float] = {}
    total = 0.0
    converged = False
    current_precision = "f32" if precision == "mixed" else "f64"
    rho_device = torch.zeros(shape, dtype=torch.float64, device=device)
    tick("setup", t0)
    iteration = 1
    while iteration <= system.maxiter:
        t0 = time.perf_counter()
        if input_hxc is None:
            input_hxc = hxc_potential(setup, rho)
        v_dev = v_ion + input_hxc
        if iteration > 1 and np.isfinite(previous_accuracy):
            if iteration == 2:
                davidson_tolerance = 5.0e-3
            davidson_tolerance = max(5.0e-14, min(davidson_tolerance,
                                                  0.1 * previous_accuracy / max(1.0, nelec)))
        if precision == "mixed" and current_precision == "f32" and np.isfinite(previous_accuracy) \
                and 2.0 * previous_accuracy < switch_ry:
            # FP64 from here on.  The Davidson threshold was held at the
            # FP32 floor: restart it from the current residual.  The Broyden
            # secant pairs of the FP32 iterations are kept unless asked
            # otherwise (their fixed point differs from the FP64 one by less
            # than the residual at the switch, and keeping them saved
            # iterations on both benchmark cells).
            current_precision = fp64_phase
            if restart_mixer_at_switch and isinstance(mixer, DeviceBroydenMixer):
                mixer.reset()
            davidson_tolerance = max(5.0e-14, 0.1 * previous_accuracy / max(1.0, nelec))
        # FP32 eigenvalues stall near 1e-7 relative: never ask more of them
        # than ``fp32_floor`` (Ha)
        tol = davidson_tolerance if current_precision != "f32" else max(davidson_tolerance, fp32_floor)
        refined = current_precision == "refined"
        if refined:
            # the refined iterations need not resolve eigenvalues finer than
            # a thousandth of the SCF threshold (the reference's schedule,
            # 0.1 dr2 / nelec, reaches 5e-13 Ha in the last iteration at
            # conv_thr 1e-8 Ry)
            floor = REFINED_FLOOR_RATIO * system.conv_thr if refined_floor is None else refined_floor
            tol = max(tol, floor)
        precision_log.append(current_precision)
        tick("v_of_rho", t0)
        t0 = time.perf_counter()
        local_eigenvalues = {}
        its = []
        hams, hams32, solves = {}, {}, {}
        # lockstep k points: their reduced eigensolves run side by side
        lockstep = bool(batch_kpoints) and len(local_k) > 1
        for k, state in enumerate(states):
            if k not in local_k:
                # (the shared random stream stays in step with one rank:
                # StartingDraws draws every k point's pairs in order)
                continue
            if state.terms is None:
                state.terms = projector_terms(system, tables, state.basis)

            def hamiltonian(form):
                made = PlaneWaveHamiltonian(state.basis, None, state.terms,
                                            local_workspace=state.workspace(form),
                                            real_potential=v_dev,
                                            potential_average=v_ion_average, timers=timers,
                                            device_projectors=state.device_projectors.get(form))
                state.device_projectors[form] = made.projectors
                return made

            ham = hamiltonian("f64" if refined else current_precision)
            carried = None
            if refined:
                hams32[k] = hamiltonian("f32")
                if state.refined is not None and state.vectors is not None and \
                        state.vectors.shape[1] == nsolve:
                    # H X = X lam + R for the previous potential; the new one
                    # adds (V_new - V_old) X, an FP32 local apply of the
                    # (small) potential change
                    lam_prev, r_prev, v_prev, error_prev = state.refined
                    x32 = to_device_f(state.vectors, torch.complex64, device)
                    dvx = hams32[k].local_workspace.apply(v_dev - v_prev, x32)
                    carried = (lam_prev, r_prev + dvx, error_prev)
                    del x32, dvx
            initial_applied = None
            initial_eigs = None
            if state.vectors is None:
                start_vectors, initial_eigs, initial_applied = random_starting_subspace(
                    ham, state.basis, draws["all"].take(k), nsolve)
            else:
                start_vectors = state.vectors.to(ham.dtype).T.contiguous().T
            # first SCF iteration: rotate_wfc Ritz vectors (or the first
            # pass's eigenvectors when the iteration is repeated); later
            # iterations restart from the converged eigenvectors
            # (qepy_pw/pw/scf.py:3503-3556)
            occ_roots = occupied if iteration > 1 and not smeared else system.nbnd
            hams[k] = ham
            solves[k] = _k_point_solve(ham, system, start_vectors, initial_eigs, initial_applied,
                                       tol, occ_roots, iteration == 1, timers,
                                       lock=lock_converged, nroots=nsolve, refined=refined,
                                       carried=carried, overlap=lockstep)
        k_order = sorted(solves)
        if lockstep:
            # chosen form: the k points' Davidson solves advance together and
            # each round's H applications share one launch per FFT pass
            table = [hams[k] for k in k_order]
            table32 = [hams32[k] for k in k_order] if refined else None
            chosen = table32 if refined else (table if current_precision == "f32" else None)
            graphs = None
            if graph_rounds and chosen is not None:
                if round_graphs is None:
                    round_graphs = RoundGraphs(chosen, max_width=nsolve)
                round_graphs.set_potential(chosen[0]._potential)
                graphs = round_graphs
            outcomes = run_lockstep([solves[k] for k in k_order],
                                    lambda requests: _apply_by_dtype(table, table32, requests,
                                                                     graphs))
        else:
            outcomes = [_drive(solves[k], hams[k], hams32.get(k)) for k in k_order]
        for k, (sol, total_its, carried_out) in zip(k_order, outcomes):
            state = states[k]
            its.append(total_its)
            state.vectors = sol.eigenvectors.to(torch.complex128).T.contiguous().T
            state.refined = ((carried_out["lam"], carried_out["residual"], v_dev,
                              carried_out["error"])
                             if refined and carried_out.get("residual") is not None else None)
            state.eigenvalues = np.asarray(sol.eigenvalues)[:system.nbnd]
            local_eigenvalues[k] = state.eigenvalues
        david_its.append(float(np.mean(its)))
        if pools is not None:
            eigenvalues = pools.gather_eigenvalues(nk, local_eigenvalues, system.nbnd, device)
            for k, values in enumerate(eigenvalues):
                states[k].eigenvalues = values
        else:
            eigenvalues = [local_eigenvalues[k] for k in range(nk)]
        torch.cuda.synchronize()
        tick("c_bands", t0)
        t0 = time.perf_counter()
        if smeared:
            # qepy_pw/pw/scf.py:3685-3695 (degauss halved to Hartree)
            fermi, band_occ, demet = smeared_occupations(eigenvalues, system.weights, nelec,
                                                         0.5 * system.degauss, order)
        else:
            band_occ, demet = fixed_occupations(system.nbnd, occupied, len(states)), 0.0
        # density from the occupied states (FP64 accumulation on the GPU),
        # bands up to the last one with a nonzero occupation (scf.py:1406-1431)
        rho_device.zero_()
        for k in local_k:
            state, weight, occ = states[k], system.weights[k], band_occ[k]
            active = np.flatnonzero(np.abs(occ) > 1.0e-15)
            if active.size == 0:
                continue
            count = int(active[-1]) + 1
            ws = state.workspace("f64")
            w = torch.from_numpy(float(weight) * occ[:count] / volume).to(device)
            ws.accumulate_density(rho_device, state.vectors[:, :count], w)
        if pools is not None:
            pools.sum_(rho_device)
        rho_out = rho_device * (nelec * grid.size / (float(torch.sum(rho_device)) * volume))
        if symmetrizer is not None:
            # on the device (qeb_symmetrize_density), then renormalised
            sym = symmetrizer.apply_device(rho_out)
            rho_out = sym * (nelec * grid.size / (float(torch.sum(sym)) * volume))
        band_energy = sum(w * float(np.sum(e * f)) for w, e, f in zip(system.weights, eigenvalues, band_occ))
        scale = volume / grid.size
        deband = -scale * float(torch.sum(rho_out * input_hxc))
        residual_g = cgrid.to_g(rho_out - rho)
        accuracy = 0.5 * volume * cgrid.residual_metric(residual_g)
        previous_accuracy = accuracy
        tick("sum_band", t0)
        if iteration == 1 and first_diagonalization and accuracy < davidson_tolerance * max(1.0, nelec):
            davidson_tolerance = max(5.0e-14, 0.1 * accuracy / max(1.0, nelec))
            first_diagonalization = False
            continue
        first_diagonalization = False
        t0 = time.perf_counter()
        # The mixed form finishes in FP64, with at least MIN_FP64_ITERATIONS
        # FP64 iterations: the residual metric weights |drho(G)|^2 by 1/G^2
        # and hardly sees the high-G density noise of the FP32 iterations,
        # which mixing removes only a factor (1 - beta) per iteration, while
        # V_xc passes it on to the eigenvalues.
        fp64_done = sum(1 for p in precision_log if p == "f64")
        if current_precision == "refined":
            # measured criterion: the eigenvalues of this FP64-accurate
            # iteration moved less than eigenvalue_change_ry from those of
            # the previous one, itself refined (the FP32 iterations'
            # eigenvalues carry their 5e-7 Ha floor)
            change = np.inf
            if previous_eigenvalues is not None and len(precision_log) > 1 and \
                    precision_log[-2] == "refined":
                change = max(float(np.max(np.abs(a - b)))
                             for a, b in zip(eigenvalues, previous_eigenvalues))
            converged = 2.0 * accuracy < system.conv_thr and 2.0 * change < eigenvalue_change_ry
        else:
            converged = 2.0 * accuracy < system.conv_thr and current_precision == "f64" and \
                (precision == "f64" or fp64_done >= MIN_FP64_ITERATIONS)
        previous_eigenvalues = [np.array(e, copy=True) for e in eigenvalues]
        if converged:
            rho_energy = rho_out
        elif isinstance(mixer, DeviceBroydenMixer):
            rho_energy = mixer.mix(rho, residual_g)
        else:
            rho_energy = mixer.mix(rho, rho_out)
        rho_energy_g = cgrid.to_g(rho_energy)
        vh_g = cgrid.hartree(rho_energy_g)
        e_h = volume * 0.5 * float(torch.real(torch.vdot(rho_energy_g, vh_g)))
        eps_xc, vxc = device_pz81(rho_energy)
        e_xc = scale * float(torch.sum(rho_energy * eps_xc))
        vh = cgrid.to_r(vh_g)
        hxc = vh + vxc
        descf = -scale * float(torch.sum(rho_energy * hxc) - torch.sum(rho_out * hxc))
        input_hxc = hxc
        energy_terms = {"one_electron": band_energy + deband, "hartree": e_h, "xc": e_xc,
                        "ewald": e_ion, "descf": descf, "smearing": demet}
        total = sum(energy_terms.values())
        energies.append(total)
        accuracies.append(accuracy)
        tick("mix_energy", t0)
        if progress is not None:
            progress(iteration, total, accuracy, current_precision)
        rho = rho_energy
        if converged:
            break
        iteration += 1
    rho_device = rho
    rho = rho.cpu().numpy()
    forces = None
    stress = stress_terms = None
    if system.stress and converged:
        from .stress import scf_stress

        t0 = time.perf_counter()
        stress, stress_terms = scf_stress(system, [states[k] for k in local_k], tables, grid, cgrid,
                                          rho_device, [band_occ[k] for k in local_k],
                                          [system.weights[k] for k in local_k], pools=pools)
        tick("stress", t0)
    del rho_device
    if system.forces and converged:
        from .forces import hellmann_feynman_forces

        t0 = time.perf_counter()
        forces = hellmann_feynman_forces(system, [states[k] for k in local_k], tables, grid, rho,
                                         [band_occ[k] for k in local_k],
                                         weights=[system.weights[k] for k in local_k],
                                         pools=pools)
        tick("forces", t0)
    return SCFResult(converged, total, iteration, energies, accuracies,
                     [s.eigenvalues for s in states], energy_terms, rho, forces,
                     time.perf_counter() - started, precision_log, david_its, timings,
                     [np.asarray(f) for f in band_occ], fermi, v_dev,
                     [states[k].vectors for k in local_k], stress, stress_terms)
