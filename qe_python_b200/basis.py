"""Plane-wave bases, FFT grids and the GPU local-potential workspace.

Host index maps (built once per k point, uploaded as int32):
  * ``make_bases``      - QE-ordered G catalog and per-k bases
                          (reference: qepy_pw/basis.py:1483-1577, 1588-1616);
  * ``fft_shape``       - the FFT grid rule (qepy_pw/basis.py:1619-1682);
  * workspace maps      - linear / z-major slots and sticks
                          (qepy_pw/basis.py:510-555).
These must agree bit for bit with the reference.

``LocalPotentialWorkspace`` keeps the reference's constructor and
``apply`` / ``accumulate_density`` signatures (qepy_pw/basis.py:460-471,
1210-1215, 1354-1362) but runs the stick/plane FFT passes of
``libqeb200.so`` on torch CUDA tensors.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from math import prod

import numpy as np
import torch

from . import _lib
from .autotune import TUNER, bucket
from .device import (
    REAL_OF,
    as_numpy,
    empty_f,
    is_column_major,
    leading_dimension,
    require_cuda,
    stream_handle,
    to_device_f,
)

# Energies closer than this are one degenerate group whose members keep
# their incoming order (QE hpsort_eps; qepy_pw/basis.py:1588-1616).
_ORDER_EPS = 1.0e-8
# Cutoff slack of the per-k selection (qepy_pw/basis.py:1540).
_CUTOFF_SLACK = 1.0e-12


def _next_fast_len_real(target: int) -> int:
    """Smallest 2-3-5 smooth integer >= target (qepy_pw/basis.py:27-37)."""
    n = max(1, int(target))
    while True:
        m = n
        for p in (2, 3, 5):
            while m % p == 0:
                m //= p
        if m == 1:
            return n
        n += 1


def _compact_unsigned(values: np.ndarray, upper_bound: int) -> np.ndarray:
    """uint16 when every index fits, else uint32 (qepy_pw/basis.py:77-80)."""
    return np.asarray(values, dtype=np.uint16 if upper_bound <= 65536 else np.uint32)


def _qe_energy_order(values: np.ndarray, tolerance: float = _ORDER_EPS) -> np.ndarray:
    """Stable ascending order in which values closer than ``tolerance`` to the
    first member of their group keep their incoming order.

    Same ordering as qepy_pw/basis.py:1588-1616: a group starts at the first
    value not within ``tolerance`` of the current group's first value.  Only
    runs of near-equal neighbours need the sequential scan.
    """
    keys = np.asarray(values, dtype=float)
    order = np.argsort(keys, kind="stable")
    if order.size < 2:
        return order
    ranked = keys[order]
    close = np.diff(ranked) < tolerance
    if not close.any():
        return order
    # maximal runs [a, b] of indices linked by consecutive near-equal gaps
    edges = np.flatnonzero(np.diff(np.concatenate(([False], close, [False])).astype(np.int8)))
    for a, b in zip(edges[0::2], edges[1::2]):
        start = a
        stop_run = b + 1  # run covers ranked[a..b], inclusive
        while start < stop_run:
            # the group of ranked[start]: the members after it up to the first
            # one not within tolerance of it (the same test as a scan)
            within = np.abs(ranked[start + 1:stop_run] - ranked[start]) < tolerance
            outside = np.flatnonzero(~within)
            stop = start + 1 + (int(outside[0]) if outside.size else within.size)
            if stop - start > 1:
                order[start:stop] = np.sort(order[start:stop])
            start = stop
    return order


@dataclass(frozen=True)
class PlaneWaveCatalog:
    """Global QE-ordered Miller catalog shared by all k (basis.py:84-106)."""

    indices: np.ndarray
    reciprocal: np.ndarray
    vectors: np.ndarray = field(repr=False, default=None)

    def __post_init__(self) -> None:
        if self.vectors is None:
            object.__setattr__(self, "vectors", np.asarray(self.indices @ self.reciprocal, dtype=float))


class PlaneWaveBasis:
    """One k point: rows ``global_indices`` of a shared catalog (basis.py:108-199).

    Also accepts the explicit ``(indices, vectors, kinetic)`` constructor of
    the reference.
    """

    def __init__(self, catalog_or_indices, mapping_or_vectors, kpoint_or_kinetic) -> None:
        if isinstance(catalog_or_indices, PlaneWaveCatalog):
            mapping = np.asarray(mapping_or_vectors)
            if mapping.size and (mapping.min() < 0 or mapping.max() >= len(catalog_or_indices.indices)):
                raise ValueError("global plane-wave mapping is out of range")
            self.catalog = catalog_or_indices
            self.global_indices = _compact_unsigned(mapping, len(catalog_or_indices.indices))
            self.k_crystal = np.asarray(kpoint_or_kinetic, dtype=float)
            self._indices = self._vectors = self._kinetic = None
        else:
            self.catalog = None
            self.global_indices = None
            self.k_crystal = None
            self._indices = np.asarray(catalog_or_indices, dtype=np.int32)
            self._vectors = np.asarray(mapping_or_vectors, dtype=float)
            self._kinetic = np.asarray(kpoint_or_kinetic, dtype=float)

    @property
    def indices(self) -> np.ndarray:
        if self.catalog is None:
            return self._indices
        return self.catalog.indices[self.global_indices]

    @property
    def vectors(self) -> np.ndarray:
        if self.catalog is None:
            return self._vectors
        return self.catalog.vectors[self.global_indices] + self.k_crystal @ self.catalog.reciprocal

    @property
    def kinetic(self) -> np.ndarray:
        """Hartree kinetic energies 1/2 |k+G|^2 (basis.py:187)."""
        if self.catalog is None:
            return self._kinetic
        v = self.vectors
        return 0.5 * np.einsum("ij,ij->i", v, v)

    def __len__(self) -> int:
        return len(self.global_indices) if self.catalog is not None else len(self._indices)

    def materialize(self) -> "PlaneWaveBasis":
        if self.catalog is None:
            return self
        v = self.vectors
        return PlaneWaveBasis(self.indices, v, 0.5 * np.einsum("ij,ij->i", v, v))


def _search_bound(reciprocal: np.ndarray, k: np.ndarray, ecut_ha: float, sigma_min: float) -> int:
    # ||n B|| >= sigma_min ||n|| bounds every Miller index inside the sphere
    # (basis.py:1458-1472, 1501-1507).
    radius = np.sqrt(2.0 * ecut_ha) + np.linalg.norm(k @ reciprocal)
    return int(np.ceil(radius / sigma_min)) + 1


def _miller_cube(bound: int) -> np.ndarray:
    """All integer triples in [-bound, bound]^3, lexicographic (basis.py:1475-1480)."""
    axis = np.arange(-bound, bound + 1, dtype=np.int32)
    a, b, c = np.meshgrid(axis, axis, axis, indexing="ij")
    return np.stack((a.ravel(), b.ravel(), c.ravel()), axis=1)


def make_bases(reciprocal, k_crystal, ecut_ry: float, *, mpi=None) -> list[PlaneWaveBasis]:
    """Per-k plane-wave bases sharing one global catalog.

    Same selection and order as qepy_pw/basis.py:1483-1577: the Miller cube
    ordered by |G|^2 (hpsort_eps groups keep Miller order), then per k the
    rows with 1/2|k+G|^2 <= ecut + 1e-12 ordered by |k+G|^2 with the same
    rule; the catalog keeps only rows some k uses, in global order.
    """
    reciprocal = np.asarray(reciprocal, dtype=float)
    kpoints = np.atleast_2d(np.asarray(k_crystal, dtype=float))
    if kpoints.ndim != 2 or kpoints.shape[1] != 3:
        raise ValueError("k_crystal must have shape (3,) or (nk, 3)")
    if kpoints.shape[0] == 0:
        raise ValueError("at least one k point is required")
    ecut_ha = 0.5 * float(ecut_ry)
    sigma_min = float(np.linalg.svd(reciprocal, compute_uv=False)[-1])
    bounds = np.array([_search_bound(reciprocal, k, ecut_ha, sigma_min) for k in kpoints])
    top = int(bounds.max())
    cube = _miller_cube(top)
    g = cube @ reciprocal
    cube = cube[_qe_energy_order(np.einsum("ij,ij->i", g, g))]
    del g
    selections = []
    for k, bound in zip(kpoints, bounds):
        if bound == top:
            rows = np.arange(len(cube), dtype=np.int32)
        else:
            rows = np.flatnonzero(np.all(np.abs(cube) <= bound, axis=1)).astype(np.int32)
        kg = (cube[rows] + k) @ reciprocal
        energy = 0.5 * np.einsum("ij,ij->i", kg, kg)
        inside = energy <= ecut_ha + _CUTOFF_SLACK
        rows, energy = rows[inside], energy[inside]
        if rows.size == 0:
            raise ValueError("ecutwfc produces an empty plane-wave basis")
        selections.append(rows[_qe_energy_order(energy)].astype(np.int32))
    used = np.zeros(len(cube), dtype=bool)
    for rows in selections:
        used[rows] = True
    kept = np.flatnonzero(used).astype(np.int32)
    renumber = np.full(len(cube), -1, dtype=np.int32)
    renumber[kept] = np.arange(kept.size, dtype=np.int32)
    catalog = PlaneWaveCatalog(np.ascontiguousarray(cube[kept], dtype=np.int32), reciprocal.copy())
    return [
        PlaneWaveBasis(catalog, renumber[rows].astype(np.int32), np.asarray(k, dtype=float))
        for k, rows in zip(kpoints, selections)
    ]


def _charge_extent(reciprocal: np.ndarray, ecut_ry: float) -> np.ndarray:
    """Largest |Miller index| per axis over the k = 0 sphere 1/2 |G|^2 <=
    ecut + 1e-12: the rows make_bases would select at k = 0, without their
    (order-only) energy sort."""
    ecut_ha = 0.5 * float(ecut_ry)
    sigma_min = float(np.linalg.svd(reciprocal, compute_uv=False)[-1])
    bound = int(_search_bound(reciprocal, np.zeros(3), ecut_ha, sigma_min))
    # Along axis a the sphere reaches |m_a| <= sqrt(2 ecut) |column a of
    # reciprocal^-1|; the planes m_a = +-m are checked from that bound down
    # with the same row test as the whole Miller cube (2-D slices of it
    # instead of the cube itself: the 216-atom cell's charge sphere spans a
    # 137^3 cube).
    inverse_norms = np.linalg.norm(np.linalg.inv(reciprocal), axis=0)
    axis = np.arange(-bound, bound + 1, dtype=np.int32)
    u, v = np.meshgrid(axis, axis, indexing="ij")
    u, v = u.ravel(), v.ravel()
    extent = np.zeros(3, dtype=np.int64)
    for a in range(3):
        top = min(bound, int(np.floor(np.sqrt(2.0 * (ecut_ha + _CUTOFF_SLACK))
                                      * inverse_norms[a])) + 1)
        others = [b for b in range(3) if b != a]
        found = -1
        for m in range(top, -1, -1):
            for sign in ((1, -1) if m else (1,)):
                rows = np.empty((u.size, 3), dtype=np.int32)
                rows[:, a] = sign * m
                rows[:, others[0]] = u
                rows[:, others[1]] = v
                g = rows @ reciprocal
                if np.any(0.5 * np.einsum("ij,ij->i", g, g) <= ecut_ha + _CUTOFF_SLACK):
                    found = m
                    break
            if found >= 0:
                break
        if found < 0:
            raise ValueError("ecutrho produces an empty charge sphere")
        extent[a] = found
    return extent


def make_basis(reciprocal, k_crystal, ecut_ry: float) -> PlaneWaveBasis:
    return make_bases(reciprocal, k_crystal, ecut_ry)[0]


def fft_shape(bases, reciprocal=None, ecutrho_ry=None, fft_factors=(1, 1, 1)) -> tuple[int, int, int]:
    """FFT grid of the reference (qepy_pw/basis.py:1619-1682).

    With ``ecutrho``: per axis, the largest |Miller| of the k=0 charge sphere
    n gives 2n+1, raised to the next 2-3-5 smooth length divisible by the
    symmetry factor.  Without: twice the per-k wavefunction span plus 2,
    raised to an even 2-3-5 smooth length.
    """
    if not bases:
        raise ValueError("at least one plane-wave basis is required")
    if (reciprocal is None) != (ecutrho_ry is None):
        raise ValueError("reciprocal and ecutrho_ry must be supplied together")
    if reciprocal is not None:
        extent = _charge_extent(np.asarray(reciprocal, dtype=float), float(ecutrho_ry))
        shape = []
        for n, factor in zip(extent, fft_factors):
            length = int(2 * n + 1)
            while True:
                candidate = _next_fast_len_real(length)
                if candidate % factor == 0:
                    shape.append(candidate)
                    break
                length = candidate + 1
        return tuple(shape)
    span = np.max(
        np.stack([b.indices.max(axis=0) - b.indices.min(axis=0) for b in bases]), axis=0
    )
    shape = []
    for n in span:
        length = _next_fast_len_real(int(2 * n + 2))
        if length % 2:
            length = _next_fast_len_real(length + 1)
        shape.append(length)
    return tuple(shape)


def grid_slots(miller: np.ndarray, shape) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
    """(linear_slots, z_major_slots, stick_positions, sticks) of basis.py:521-546.

    linear: C-order slot of (m mod n); z-major: z*nx*ny + x*ny + y; stick
    positions: sorted unique x*ny + y; sticks: unique (x, y) pairs.
    """
    nx, ny, nz = (int(v) for v in shape)
    sx = np.asarray(miller[:, 0] % nx, dtype=np.int32)
    sy = np.asarray(miller[:, 1] % ny, dtype=np.int32)
    sz = np.asarray(miller[:, 2] % nz, dtype=np.int32)
    linear = np.asarray(np.ravel_multi_index((sx, sy, sz), (nx, ny, nz)), dtype=np.int32)
    xy = sx * ny + sy
    size = nx * ny * nz
    z_major = _compact_unsigned(sz * (nx * ny) + xy, size)
    positions = _compact_unsigned(np.unique(xy), nx * ny)
    sticks = np.unique(np.column_stack((sx, sy)), axis=0).astype(np.int32, copy=False)
    return linear, z_major, positions, sticks


class FFTScratchPool:
    """Grow-only named device scratch shared by workspaces (basis.py:407-454)."""

    def __init__(self) -> None:
        self._buffers: dict[tuple[str, torch.device], torch.Tensor] = {}

    def buffer(self, name: str, nbytes: int, device: torch.device) -> torch.Tensor:
        key = (name, device)
        current = self._buffers.get(key)
        if current is None or current.numel() < nbytes:
            # 256-byte aligned by the CUDA caching allocator.
            current = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
            self._buffers[key] = current
        return current

    @property
    def nbytes(self) -> int:
        return sum(t.numel() for t in self._buffers.values())


_PRECISIONS = {"f64": (_lib.QEB_F64, torch.complex128), "f32": (_lib.QEB_F32, torch.complex64)}


class LocalPotentialWorkspace:
    """Reusable device maps and scratch for repeated local H|psi> calls.

    Constructor and methods follow qepy_pw/basis.py:460-471, 1210-1215 and
    1354-1362.  ``precision`` ('f64' plain, 'f32' chosen form) selects the
    kernel arithmetic; inputs of the other precision are converted.
    """

    def __init__(self, indices, shape, *, mpi=None, timers=None, scratch_pool=None,
                 descriptor=None, serial_fft_batch_size=None, retain_serial_sticks=True,
                 precision: str = "f64", device=None) -> None:
        if mpi is not None and getattr(mpi, "size", 1) != 1:
            raise ValueError("the B200 workspace is single-rank (one GPU per k-point pool)")
        if isinstance(indices, PlaneWaveBasis):
            miller = indices.indices
        else:
            miller = np.asarray(indices, dtype=np.int32)
        if miller.ndim != 2 or miller.shape[1] != 3:
            raise ValueError("indices must have shape (nplane, 3)")
        if serial_fft_batch_size is not None and int(serial_fft_batch_size) < 1:
            raise ValueError("serial_fft_batch_size must be at least 1")
        if precision not in _PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}")
        self.shape = tuple(int(v) for v in shape)
        self.size = prod(self.shape)
        self.plane_waves = len(miller)
        self.timers = timers
        self.precision = precision
        self._code, self.complex_dtype = _PRECISIONS[precision]
        self.real_dtype = REAL_OF[self.complex_dtype]
        self.device = device if device is not None else require_cuda()
        self.scratch_pool = scratch_pool if scratch_pool is not None else FFTScratchPool()
        self.serial_fft_batch_size = serial_fft_batch_size
        (self.linear_slots, self.z_major_slots, self.serial_stick_positions, sticks) = grid_slots(
            miller, self.shape
        )
        self.sticks = sticks if retain_serial_sticks else np.empty((0, 2), dtype=np.int32)
        self.local_plane_wave_indices = np.arange(self.plane_waves, dtype=np.int32)
        self.mpi = mpi
        self._plan = ctypes.c_void_p()
        slots64 = np.ascontiguousarray(self.z_major_slots, dtype=np.int64)
        lib = _lib.load()
        with torch.cuda.device(self.device):
            status = lib.qeb_local_plan_create(
                ctypes.byref(self._plan), self.shape[0], self.shape[1], self.shape[2],
                self.plane_waves, slots64.ctypes.data, self._code,
            )
        _lib.check("qeb_local_plan_create", status)
        info = np.zeros(9, dtype=np.int64)
        _lib.check("qeb_local_plan_info",
                   lib.qeb_local_plan_info(self._plan, info.ctypes.data, 9))
        self.stick_count = int(info[4])
        self.active_rows = int(info[5])
        # K of the pruned plane pass (every stick within the 2 K N2 kept rows
        # and columns of a 64-point plane), 0 for the active-row plane
        self.pruned_plane = int(info[8])
        self._potential_cache: tuple | None = None
        self._kinetic_cache: tuple | None = None
        # When a list, each apply batch appends its (A, B, C) pass times in ms.
        self.pass_times: list | None = None

    def __del__(self) -> None:
        plan = getattr(self, "_plan", None)
        if plan is not None and plan.value:
            try:
                _lib.load().qeb_local_plan_destroy(plan)
            except Exception:
                pass
            self._plan = None

    # -- operand preparation -------------------------------------------------
    def native_potential(self, real_potential, native_potential_layout: bool = False) -> torch.Tensor:
        """Device (nz, nx, ny) copy of V(r) in kernel precision, cached per tensor."""
        key = None
        if isinstance(real_potential, torch.Tensor):
            key = (id(real_potential), real_potential._version, native_potential_layout)
            if self._potential_cache is not None and self._potential_cache[0] == key:
                return self._potential_cache[1]
        v = real_potential
        if not isinstance(v, torch.Tensor):
            v = torch.from_numpy(np.ascontiguousarray(np.asarray(v, dtype=np.float64)))
        v = v.to(device=self.device, dtype=torch.float64)
        nx, ny, nz = self.shape
        if native_potential_layout:
            if tuple(v.shape) != (nz, nx, ny):
                raise ValueError("native potential must have shape (nz, nx, ny)")
        else:
            if tuple(v.shape) != (nx, ny, nz):
                raise ValueError("real potential must have shape (nx, ny, nz)")
            v = v.permute(2, 0, 1)
        v = v.to(self.real_dtype).contiguous()
        if key is not None:
            self._potential_cache = (key, v, real_potential)
        return v

    def _kinetic(self, diagonal) -> torch.Tensor | None:
        if diagonal is None:
            return None
        if isinstance(diagonal, torch.Tensor):
            key = (id(diagonal), diagonal._version)
            if self._kinetic_cache is not None and self._kinetic_cache[0] == key:
                return self._kinetic_cache[1]
        d = to_device_f(diagonal, torch.float64, self.device).to(self.real_dtype).contiguous()
        if d.numel() != self.plane_waves:
            raise ValueError("kinetic diagonal must have one entry per plane wave")
        if isinstance(diagonal, torch.Tensor):
            self._kinetic_cache = ((id(diagonal), diagonal._version), d, diagonal)
        return d

    def _scratch(self, nbands: int) -> tuple[torch.Tensor, int]:
        nbytes = int(_lib.load().qeb_local_scratch_bytes(self._plan, nbands))
        return self.scratch_pool.buffer("sticks", nbytes, self.device), nbytes

    # -- operator ------------------------------------------------------------
    def apply(self, real_potential, coefficients, *, native_potential_layout: bool = False,
              out=None, diagonal=None):
        """out[:, b] = (V psi_b)(G)/N + diagonal * psi_b on the GPU.

        ``coefficients`` / ``out`` are column-major (npw, nb) torch CUDA tensors
        (numpy input is copied to the device and the result returned as numpy).
        """
        host_result = not isinstance(coefficients, torch.Tensor)
        vectors = to_device_f(coefficients, self.complex_dtype, self.device)
        was_vector = vectors.dim() == 1
        if was_vector:
            vectors = vectors[:, None]
        if vectors.dim() != 2 or vectors.shape[0] != self.plane_waves:
            raise ValueError("coefficients must have shape (nplane,) or (nplane, nvec)")
        nb = vectors.shape[1]
        potential = self.native_potential(real_potential, native_potential_layout)
        kinetic = self._kinetic(diagonal)
        if out is None or host_result and not isinstance(out, torch.Tensor):
            target = empty_f(self.plane_waves, nb, self.complex_dtype, self.device)
        else:
            target = out if not was_vector or out.dim() == 2 else out[:, None]
            if (tuple(target.shape) != (self.plane_waves, nb) or target.dtype != self.complex_dtype
                    or not is_column_major(target) or target.device != self.device):
                raise ValueError("local-potential output has the wrong shape, dtype or layout")
        self._launch_apply(potential, vectors, kinetic, target)
        if host_result:
            result = as_numpy(target)
            if out is not None and not isinstance(out, torch.Tensor):
                out[...] = result.reshape(out.shape)
                result = out
            return result[:, 0] if was_vector and result.ndim == 2 else result
        return target[:, 0] if was_vector else target

    def _launch_apply(self, potential: torch.Tensor, vectors: torch.Tensor,
                      kinetic: torch.Tensor | None, target: torch.Tensor) -> None:
        nb = vectors.shape[1]
        if nb == 0:
            return
        if self.serial_fft_batch_size is not None:
            batch = max(1, int(self.serial_fft_batch_size))
        elif self.pass_times is not None or nb < 128:
            batch = nb
        else:
            # bands per launch, by measurement: a batch whose stick buffer
            # stays in L2 between the passes can beat one launch of all bands
            top = bucket(nb)
            candidates = [top] + [b for b in (128, 64) if b < top]
            key = f"local_apply/{self.precision}/{self.shape}/{self.plane_waves}/{top}"
            batch = TUNER.choose(key, candidates, lambda b: self._run_apply(
                potential, vectors, kinetic, target, min(b, nb)))
        self._run_apply(potential, vectors, kinetic, target, min(batch, nb, 65535))

    def _run_apply(self, potential, vectors, kinetic, target, batch: int) -> None:
        nb = vectors.shape[1]
        lib = _lib.load()
        stream = stream_handle()
        ld_in, ld_out = leading_dimension(vectors), leading_dimension(target)
        elem = vectors.element_size()
        for start in range(0, nb, batch):
            count = min(batch, nb - start)
            scratch, nbytes = self._scratch(count)
            args = (
                self._plan, scratch.data_ptr(), nbytes,
                vectors.data_ptr() + start * ld_in * elem, ld_in, count,
                potential.data_ptr(), 0 if kinetic is None else kinetic.data_ptr(),
                target.data_ptr() + start * ld_out * elem, ld_out, stream,
            )
            if self.pass_times is None:
                _lib.check("qeb_apply_local", lib.qeb_apply_local(*args))
            else:
                ms = (ctypes.c_float * 3)()
                _lib.check("qeb_apply_local_profiled", lib.qeb_apply_local_profiled(*args, ms))
                self.pass_times.append(tuple(float(v) for v in ms))

    def accumulate_density(self, density, coefficients, band_weights) -> None:
        """density[x, y, z] += sum_b w_b |psi_b(r)|^2 (float64, C-order grid)."""
        vectors = to_device_f(coefficients, self.complex_dtype, self.device)
        if vectors.dim() == 1:
            vectors = vectors[:, None]
        weights = to_device_f(band_weights, torch.float64, self.device).contiguous()
        if vectors.dim() != 2 or vectors.shape[1] != weights.numel():
            raise ValueError("density coefficients and band weights disagree")
        if tuple(density.shape) != self.shape:
            raise ValueError("density accumulator has the wrong local shape")
        host = not isinstance(density, torch.Tensor)
        rho = torch.zeros(self.shape, dtype=torch.float64, device=self.device) if host else density
        if rho.dtype != torch.float64 or not rho.is_contiguous():
            raise ValueError("density must be a contiguous float64 grid")
        nb = vectors.shape[1]
        lib = _lib.load()
        stream = stream_handle()
        ld = leading_dimension(vectors)
        elem = vectors.element_size()
        batch = nb if self.serial_fft_batch_size is None else max(1, int(self.serial_fft_batch_size))
        batch = min(max(batch, 1), 65535)
        for start in range(0, nb, batch):
            count = min(batch, nb - start)
            scratch, nbytes = self._scratch(count)
            status = lib.qeb_accumulate_density(
                self._plan, scratch.data_ptr(), nbytes,
                vectors.data_ptr() + start * ld * elem, ld, count,
                weights.data_ptr() + start * 8, rho.data_ptr(), stream,
            )
            _lib.check("qeb_accumulate_density", status)
        if host:
            density += rho.cpu().numpy()

    def prepare_potential(self, potential_g) -> np.ndarray:
        """Real part of the unnormalised inverse transform of V(G) (basis.py:777-796).

        Set-up path (once per Hamiltonian), not the H|psi> hot path.
        """
        values = np.asarray(potential_g, dtype=np.complex128)
        return np.real(np.fft.ifftn(values) * values.size).copy()


def potential_matrix(vg: np.ndarray, indices: np.ndarray) -> np.ndarray:
    """Dense V(G - G') (qepy_pw/basis.py:1685-1688); a test helper."""
    delta = indices[:, None, :] - indices[None, :, :]
    return vg[tuple(delta[:, :, a] % vg.shape[a] for a in range(3))]


def apply_local_potential(vg: np.ndarray, indices: np.ndarray, coefficients: np.ndarray):
    """V psi through the GPU workspace (qepy_pw/basis.py:1691-1698)."""
    workspace = LocalPotentialWorkspace(indices, vg.shape)
    return workspace.apply(workspace.prepare_potential(vg), coefficients)


_MULTI_SCRATCH = FFTScratchPool()


def set_persistent_passes(enabled: bool) -> None:
    """Run the three four-step passes of a local apply (one k point or a
    batch) as one persistent cooperative launch with grid barriers between
    them (True), or as three launches (False, the default).  Process-wide;
    the arithmetic is the same either way (qeb_set_persistent_passes)."""
    _lib.check("qeb_set_persistent_passes",
               _lib.load().qeb_set_persistent_passes(1 if enabled else 0))


def persistent_passes() -> bool:
    return bool(_lib.load().qeb_persistent_passes())


def apply_local_multi(workspaces, potential: torch.Tensor, vectors, kinetics, targets,
                      scratch_pool: FFTScratchPool | None = None) -> None:
    """targets[k] = (T_k + V) vectors[k] for several k points on one grid, one
    launch per FFT pass (qeb_apply_local_multi; at most 16 k points per call,
    more are taken 16 at a time).  ``potential`` is the native (nz, nx, ny)
    grid in the workspaces' precision; ``kinetics[k]`` may be None.
    ``scratch_pool``: the stick scratch (default: one pool shared by all
    calls; a captured graph passes its own)."""
    pool = _MULTI_SCRATCH if scratch_pool is None else scratch_pool
    nk_all = len(workspaces)
    if not (len(vectors) == len(kinetics) == len(targets) == nk_all):
        raise ValueError("one vector block, kinetic term and target per workspace")
    lib = _lib.load()
    stream = stream_handle()
    for start in range(0, nk_all, 16):
        part = range(start, min(nk_all, start + 16))
        nk = len(part)
        plans = (ctypes.c_void_p * nk)(*[workspaces[k]._plan.value for k in part])
        nbands = (ctypes.c_int64 * nk)(*[vectors[k].shape[1] for k in part])
        need = int(lib.qeb_local_multi_scratch_bytes(nk, plans, nbands))
        if need < 0:
            raise ValueError("invalid plans or band counts")
        scratch = pool.buffer("sticks", max(need, 256), workspaces[start].device)
        psi = (ctypes.c_void_p * nk)(*[vectors[k].data_ptr() for k in part])
        ld_psi = (ctypes.c_int64 * nk)(*[leading_dimension(vectors[k]) for k in part])
        kin = (ctypes.c_void_p * nk)(*[0 if kinetics[k] is None else kinetics[k].data_ptr()
                                       for k in part])
        out = (ctypes.c_void_p * nk)(*[targets[k].data_ptr() for k in part])
        ld_out = (ctypes.c_int64 * nk)(*[leading_dimension(targets[k]) for k in part])
        _lib.check("qeb_apply_local_multi", lib.qeb_apply_local_multi(
            nk, plans, scratch.data_ptr(), need, psi, ld_psi, nbands, potential.data_ptr(), kin,
            out, ld_out, stream))
