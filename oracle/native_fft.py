"""CPU oracle: a NumPy/SciPy restatement of qepy-pw's ``_native_fft`` module.

TEST INFRASTRUCTURE ONLY.  This module is the checker for the B200 hot path:
only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it.  The product package never routes work here.

The reference's native module (``qepy_pw/_native_fft.pyx``, Cython + C with
FFTW, CBLAS/LAPACKE and MPI) cannot be built in this environment (no FFTW, no
MPI).  Every entry point that the single-rank reference path calls is restated
here with the same argument order, in-place conventions and error behaviour,
so that the reference's pure-Python driver can be imported with this module
registered as ``qepy_pw._native_fft`` (see ``oracle/reference_env.py``).

Conventions restated from the reference:
  * backward FFT = sign +1, forward = sign -1, both unnormalised; the gather
    after the forward transform divides by N_r
    (``_native_fft.pyx:2020-2037, 2405``);
  * index maps may be uint16/uint32/int64 (``_native_fft.pyx:52-56``);
  * the spatial kernels address grids z-major: ``z*nx*ny + x*ny + y``
    (``_native_fft.pyx:58-135``), densities as ``xy*nz + z`` (``:190``).
"""

from __future__ import annotations

import numpy as np
import scipy.fft
import scipy.linalg

_WORKERS = 1


def set_workers(count: int) -> None:
    """Thread count used by SciPy's pocketfft inside the oracle."""
    global _WORKERS
    _WORKERS = max(1, int(count))


def _backward(values: np.ndarray, axes) -> np.ndarray:
    # Unnormalised sign +1 transform (FFTW_BACKWARD).
    return scipy.fft.ifftn(values, axes=axes, norm="forward", workers=_WORKERS)


def _forward(values: np.ndarray, axes) -> np.ndarray:
    # Unnormalised sign -1 transform (FFTW_FORWARD).
    return scipy.fft.fftn(values, axes=axes, workers=_WORKERS)


def configure_openmp_threads(nthreads: int) -> None:
    """``_native_fft.pyx:845-849``: only validates the count here."""
    if nthreads < 1:
        raise ValueError("OpenMP thread count must be positive")


def fftw_mpi_available() -> bool:
    """``_native_fft.pyx:2089-2091``: the oracle has no distributed FFT."""
    return False


class NativeFFTWPlan:
    """In-place batched complex DFT pair (``_native_fft.pyx:1973-2086``).

    ``lengths`` is the transform shape, ``howmany`` transforms of stride
    ``stride`` and distance ``distance`` elements in the owner array.
    """

    def __init__(self, array, lengths, howmany, stride, distance, flags=64, nthreads=1):
        if array.dtype != np.complex128 or not array.flags.c_contiguous:
            raise ValueError("native FFTW plans require C-contiguous complex128")
        dims = tuple(int(v) for v in np.atleast_1d(lengths))
        if len(dims) < 1:
            raise ValueError("native FFTW plan needs at least one dimension")
        if nthreads < 1:
            raise ValueError("FFTW thread count must be positive")
        self._owner = array
        self.lengths = dims
        self._howmany = int(howmany)
        self.stride = int(stride)
        self.distance = int(distance)

    def _views(self):
        flat = self._owner.reshape(-1)
        size = int(np.prod(self.lengths))
        rank = len(self.lengths)
        for index in range(self._howmany):
            base = index * self.distance
            if self.stride == 1:
                yield flat[base: base + size].reshape(self.lengths)
            else:
                # Elements of one transform are ``stride`` apart; the
                # innermost dimension is the fastest varying.
                strides = []
                running = self.stride
                for extent in reversed(self.lengths):
                    strides.append(running)
                    running *= extent
                strides = tuple(reversed(strides))
                yield np.lib.stride_tricks.as_strided(
                    flat[base:],
                    shape=self.lengths,
                    strides=tuple(s * flat.itemsize for s in strides),
                )
            del rank

    def execute(self, direction):
        if direction not in ("forward", "backward"):
            raise ValueError("FFT direction must be 'forward' or 'backward'")
        transform = _forward if direction == "forward" else _backward
        for view in self._views():
            view[...] = transform(view, axes=tuple(range(view.ndim)))


def _grid_shape(plan: NativeFFTWPlan, fft_size: int) -> tuple[int, ...]:
    shape = tuple(plan.lengths)
    if int(np.prod(shape)) != int(fft_size):
        raise ValueError("plan lengths do not match the FFT size")
    return shape


def inverse_real(reciprocal, lengths, flags=64, nthreads=1):
    """``_native_fft.pyx:2188-2202``: real part of one unnormalised inverse FFT.

    The input array is overwritten, as the in-place native plan does.
    """
    if reciprocal.dtype != np.complex128 or not reciprocal.flags.c_contiguous:
        raise ValueError("native inverse input must be contiguous complex128")
    shape = tuple(int(v) for v in lengths)
    view = reciprocal.reshape(shape)
    view[...] = _backward(view, axes=(0, 1, 2))
    return np.asarray(reciprocal.real).copy()


def inverse_serial(grid, vectors, slots, plan, fft_size, grid_stride):
    """``_native_fft.pyx:2205-2244``: zero, scatter by linear slot, FFT^+."""
    shape = _grid_shape(plan, fft_size)
    nbands = vectors.shape[1]
    grid[...] = 0.0
    rows = grid.reshape(-1, grid_stride)
    index = np.asarray(slots, dtype=np.int64)
    for band in range(nbands):
        rows[band, index] = vectors[:, band]
        cube = rows[band, :fft_size].reshape(shape)
        cube[...] = _backward(cube, axes=(0, 1, 2))
    return grid


def forward_serial(grid, slots, plan, fft_size, grid_stride):
    """``_native_fft.pyx:2247-2281``: FFT^-, gather by slot, divide by N."""
    shape = _grid_shape(plan, fft_size)
    rows = grid.reshape(-1, grid_stride)
    nbands = rows.shape[0]
    index = np.asarray(slots, dtype=np.int64)
    result = np.empty((index.size, nbands), dtype=np.complex128)
    for band in range(nbands):
        cube = rows[band, :fft_size].reshape(shape)
        cube[...] = _forward(cube, axes=(0, 1, 2))
        result[:, band] = rows[band, index] / fft_size
    return result


def add_diagonal_product(result, diagonal, vectors):
    """``_native_fft.pyx:2284-2335``: ``result += diag[:,None] * vectors``."""
    if (
        result.ndim != 2 or vectors.ndim != 2
        or result.dtype != np.complex128 or vectors.dtype != np.complex128
        or result.shape != vectors.shape
    ):
        raise ValueError("result and vectors must be matching complex128 matrices")
    if diagonal.ndim != 1 or diagonal.dtype != np.float64 or diagonal.size != vectors.shape[0]:
        raise ValueError("diagonal must be contiguous float64")
    result += diagonal[:, None] * vectors


def apply_serial(grid, vectors, potential, slots, plan, fft_size, grid_stride,
                 result, result_offset, diagonal=None):
    """``_native_fft.pyx:2338-2455``: per band scatter -> FFT^+ -> x V(r) ->
    FFT^- -> gather/N (+ T_G psi_G) into ``result[:, offset + b]``.

    ``potential`` is the C-order (nx, ny, nz) float64 grid.
    """
    if potential.dtype != np.float64 or not potential.flags.c_contiguous:
        raise ValueError("native local potential must be contiguous float64")
    if result.dtype != np.complex128 or result.ndim != 2:
        raise ValueError("native local result must be a complex128 matrix")
    if diagonal is not None:
        if diagonal.dtype != np.float64 or diagonal.ndim != 1 or diagonal.size != vectors.shape[0]:
            raise ValueError("kinetic diagonal must be contiguous float64")
    shape = _grid_shape(plan, fft_size)
    index = np.asarray(slots, dtype=np.int64)
    pot = potential.reshape(shape)
    for band in range(vectors.shape[1]):
        cube = np.zeros(fft_size, dtype=np.complex128)
        cube[index] = vectors[:, band]
        cube = _backward(cube.reshape(shape), axes=(0, 1, 2))
        cube *= pot
        cube = _forward(cube, axes=(0, 1, 2)).reshape(-1)
        column = cube[index] / fft_size
        if diagonal is not None:
            column = column + diagonal * vectors[:, band]
        result[:, result_offset + band] = column
    grid.reshape(-1)[...] = 0.0


def apply_serial_spatial(grid, vectors, potential, z_major_slots, stick_positions,
                         z_plan, xy_plan, fft_size, grid_stride, result,
                         result_offset, diagonal=None):
    """``_native_fft.pyx:58-135, 2458-2534``: the stick/plane factorisation.

    ``potential`` is the native (nz, nx, ny) layout; grids are z-major.  The
    z transforms run only on the occupied (x, y) sticks, exactly as the
    reference does, so rounding follows the same factorisation.
    """
    if potential.dtype != np.float64 or not potential.flags.c_contiguous:
        raise ValueError("spatial serial potential must be contiguous float64")
    if potential.ndim != 3 or potential.size != fft_size:
        raise ValueError("spatial serial potential has the wrong shape")
    if diagonal is not None:
        if diagonal.dtype != np.float64 or diagonal.ndim != 1 or diagonal.size != vectors.shape[0]:
            raise ValueError("kinetic diagonal must be contiguous float64")
    nz, nx, ny = potential.shape
    slots = np.asarray(z_major_slots, dtype=np.int64)
    sticks = np.asarray(stick_positions, dtype=np.int64)
    for band in range(vectors.shape[1]):
        cube = np.zeros((nz, nx * ny), dtype=np.complex128)
        cube.reshape(-1)[slots] = vectors[:, band]
        cube[:, sticks] = _backward(cube[:, sticks], axes=(0,))
        planes = cube.reshape(nz, nx, ny)
        planes[...] = _backward(planes, axes=(1, 2))
        planes *= potential
        planes[...] = _forward(planes, axes=(1, 2))
        cube[:, sticks] = _forward(cube[:, sticks], axes=(0,))
        column = cube.reshape(-1)[slots] / fft_size
        if diagonal is not None:
            column = column + diagonal * vectors[:, band]
        result[:, result_offset + band] = column


def accumulate_density_serial(density, grid, vectors, band_weights, slots, plan,
                              fft_size, grid_stride):
    """``_native_fft.pyx:2592-2648``: ``density += sum_b w_b |FFT^+ psi_b|^2``
    with the density in C-order (nx, ny, nz)."""
    shape = _grid_shape(plan, fft_size)
    index = np.asarray(slots, dtype=np.int64)
    flat = density.reshape(-1)
    total = np.zeros(fft_size, dtype=np.float64)
    for band in range(vectors.shape[1]):
        cube = np.zeros(fft_size, dtype=np.complex128)
        cube[index] = vectors[:, band]
        cube = _backward(cube.reshape(shape), axes=(0, 1, 2)).reshape(-1)
        total += band_weights[band] * (cube.real ** 2 + cube.imag ** 2)
    flat += total


def accumulate_density_serial_spatial(density, grid, vectors, band_weights,
                                      z_major_slots, stick_positions, z_plan,
                                      xy_plan, fft_size, grid_stride):
    """``_native_fft.pyx:137-193, 2537-2589``: z-major inverse transform and
    accumulation into ``density[xy*nz + z]``."""
    if density.dtype != np.float64 or not density.flags.c_contiguous:
        raise ValueError("density must be contiguous float64")
    nz = density.shape[2]
    plane = fft_size // nz
    nx, ny = density.shape[0], density.shape[1]
    slots = np.asarray(z_major_slots, dtype=np.int64)
    sticks = np.asarray(stick_positions, dtype=np.int64)
    total = np.zeros((nz, plane), dtype=np.float64)
    for band in range(vectors.shape[1]):
        cube = np.zeros((nz, plane), dtype=np.complex128)
        cube.reshape(-1)[slots] = vectors[:, band]
        cube[:, sticks] = _backward(cube[:, sticks], axes=(0,))
        planes = cube.reshape(nz, nx, ny)
        planes[...] = _backward(planes, axes=(1, 2))
        total += band_weights[band] * (cube.real ** 2 + cube.imag ** 2)
    density.reshape(plane, nz)[...] += total.T


def projector_overlaps(beta, vectors):
    """``_native_fft.pyx:694-731``: ``beta^H vectors`` (ZGEMM ConjTrans).

    Declines (returns None) unless both operands are column-major.
    """
    if (
        beta.ndim != 2 or vectors.ndim != 2
        or beta.dtype != np.complex128 or vectors.dtype != np.complex128
        or beta.shape[0] != vectors.shape[0]
    ):
        raise ValueError("projector and vector matrices disagree")
    if not beta.flags.f_contiguous or not vectors.flags.f_contiguous:
        return None
    return np.asfortranarray(beta.conj().T @ vectors)


def accumulate_projector_diagonal(diagonal, coupled, beta, multiplicity):
    """``_native_fft.pyx:734-779``: ``diag += m * Re[sum_i coupled_gi conj(beta_gi)]``."""
    if (
        diagonal.ndim != 1 or coupled.ndim != 2 or beta.ndim != 2
        or diagonal.dtype != np.float64 or coupled.dtype != np.complex128
        or beta.dtype != np.complex128 or diagonal.size != beta.shape[0]
        or coupled.shape != beta.shape or not diagonal.flags.c_contiguous
    ):
        raise ValueError("projector diagonal operands disagree")
    diagonal += multiplicity * np.real(np.sum(coupled * beta.conj(), axis=1))
    return diagonal


def add_projector_product(result, beta, coupled):
    """``_native_fft.pyx:782-836``: ``result += beta @ coupled`` (ZGEMM beta=1).

    Returns False (decline) for layouts the native ZGEMM bridge refuses.
    """
    if (
        result.ndim != 2 or beta.ndim != 2 or coupled.ndim != 2
        or result.dtype != np.complex128 or beta.dtype != np.complex128
        or coupled.dtype != np.complex128
        or result.shape[0] != beta.shape[0]
        or beta.shape[1] != coupled.shape[0]
        or result.shape[1] != coupled.shape[1]
    ):
        raise ValueError("projector product matrices disagree")
    if not beta.flags.f_contiguous:
        return False
    if result.strides[1] == 16 and coupled.flags.c_contiguous:
        pass
    elif result.flags.f_contiguous and coupled.flags.f_contiguous:
        pass
    else:
        return False
    result += beta @ coupled
    return True


def generalized_eigh(hamiltonian, overlap, roots):
    """``_native_fft.pyx:667-691``: LAPACK ``zhegvd`` (itype 1, 'V', lower).

    SciPy's ``eigh(..., driver='gvd')`` calls the same LAPACK routine.
    """
    a = np.array(hamiltonian, dtype=np.complex128, order="F", copy=True)
    b = np.array(overlap, dtype=np.complex128, order="F", copy=True)
    try:
        values, vectors = scipy.linalg.eigh(
            a, b, lower=True, driver="gvd", check_finite=False
        )
    except scipy.linalg.LinAlgError as exc:
        raise np.linalg.LinAlgError(f"native LAPACK zhegvd failed: {exc}") from exc
    return values[:roots].copy(), np.asfortranarray(vectors[:, :roots])


def qe_precondition(residuals, eigenvalues, diagonal):
    """``_native_fft.pyx:852-899``: QE ``g_psi``:
    x = 2(H_GG - e), d = (1 + x + sqrt(1 + (x-1)^2))/2, out = 2 r / d."""
    if residuals.ndim != 2 or residuals.dtype != np.complex128:
        raise ValueError("residuals must be a complex128 matrix")
    if eigenvalues.ndim != 1 or eigenvalues.dtype != np.float64 or eigenvalues.size != residuals.shape[1]:
        raise ValueError("eigenvalues must be contiguous float64")
    if diagonal.ndim != 1 or diagonal.dtype != np.float64 or diagonal.size != residuals.shape[0]:
        raise ValueError("diagonal must be contiguous float64")
    x_ry = 2.0 * (diagonal[:, None] - eigenvalues[None, :])
    denominator = 0.5 * (1.0 + x_ry + np.sqrt(1.0 + (x_ry - 1.0) ** 2))
    return np.asfortranarray(2.0 * residuals / denominator)


def column_squared_norms(vectors):
    """``_native_fft.pyx:1153-1190``."""
    if vectors.ndim != 2 or vectors.dtype != np.complex128:
        raise ValueError("vectors must be a complex128 matrix")
    return np.sum(vectors.real ** 2 + vectors.imag ** 2, axis=0)


def subtract_band_energies(result, vectors, energies):
    """``_native_fft.pyx:1193-1234``: in place ``result[:,b] -= e_b vectors[:,b]``."""
    if (
        result.ndim != 2 or vectors.ndim != 2
        or result.dtype != np.complex128 or vectors.dtype != np.complex128
        or result.shape != vectors.shape
    ):
        raise ValueError("residual matrices disagree")
    if energies.dtype != np.float64 or energies.size != vectors.shape[1]:
        raise ValueError("band energies must be contiguous float64")
    result -= vectors * energies[None, :]
    return result


def column_inner_products(left, right):
    """``_native_fft.pyx:1237-1291``: columnwise ``left^H right``."""
    if (
        left.ndim != 2 or right.ndim != 2
        or left.dtype != np.complex128 or right.dtype != np.complex128
        or left.shape != right.shape
    ):
        raise ValueError("inner-product matrices disagree")
    return np.sum(left.conj() * right, axis=0)


def column_diagonal_expectations(vectors, diagonal):
    """``_native_fft.pyx:1294-1343``."""
    if vectors.ndim != 2 or vectors.dtype != np.complex128:
        raise ValueError("vectors must be complex128")
    if diagonal.dtype != np.float64 or diagonal.size != vectors.shape[0]:
        raise ValueError("diagonal must be contiguous float64")
    return np.sum(diagonal[:, None] * (vectors.real ** 2 + vectors.imag ** 2), axis=0)


def rmm_kinetic_precondition(residuals, kinetic, expectations, selected):
    """``_native_fft.pyx:1346-1408``: Kresse-Furthmueller diagonal."""
    cols = np.asarray(selected, dtype=np.int64)
    x = kinetic[:, None] / (1.5 * expectations[None, :])
    x2 = x * x
    numerator = 27.0 + x * (18.0 + x * (12.0 + 8.0 * x))
    denominator = numerator + 16.0 * x2 * x2
    scale = (-4.0 / 3.0) * numerator / (expectations[None, :] * denominator)
    return np.asfortranarray(scale * residuals[:, cols])


def _qe_randy_stream(count: int, table: np.ndarray, current: int, seed: int):
    """QE ``randy`` table-shuffled LCG (``_native_fft.pyx:1425-1438``)."""
    out = np.empty(count, dtype=np.float64)
    state = table
    for position in range(count):
        index = (97 * current) // 714025
        current = int(state[index])
        out[position] = current / 714025.0
        seed = (1366 * seed + 150889) % 714025
        state[index] = seed
    return out, current, seed


def qe_random_pairs(plane_waves, bands, table, current, seed):
    """``_native_fft.pyx:1411-1444``: band-major (amplitude, phase) pairs."""
    if table.dtype != np.int64 or table.size != 97:
        raise ValueError("QE random table must contain 97 contiguous int64 values")
    stream, current, seed = _qe_randy_stream(2 * plane_waves * bands, table, int(current), int(seed))
    pairs = stream.reshape(bands, plane_waves, 2)
    first = np.asfortranarray(pairs[:, :, 0].T)
    second = np.asfortranarray(pairs[:, :, 1].T)
    return first, second, current, seed


def qe_random_pairs_rows(plane_waves, bands, rows, table, current, seed):
    """``_native_fft.pyx:1447-1492``: the same stream, keeping selected rows."""
    first, second, current, seed = qe_random_pairs(plane_waves, bands, table, current, seed)
    selected = np.asarray(rows, dtype=np.int64)
    return (np.asfortranarray(first[selected]), np.asfortranarray(second[selected]),
            current, seed)


def normalize_selected_columns(vectors, squared_norms, selected):
    """``_native_fft.pyx:1495-1530``."""
    if vectors.ndim != 2 or vectors.dtype != np.complex128:
        raise ValueError("vectors must be a complex128 matrix")
    cols = np.asarray(selected, dtype=np.int64)
    return np.asfortranarray(vectors[:, cols] / np.sqrt(squared_norms[cols])[None, :])


def row_norms3(vectors):
    """``_native_fft.pyx:1533-1553``."""
    if vectors.ndim != 2 or vectors.shape[1] != 3 or vectors.dtype != np.float64:
        raise ValueError("vectors must be an N-by-3 float64 matrix")
    return np.sqrt(vectors[:, 0] ** 2 + vectors[:, 1] ** 2 + vectors[:, 2] ** 2)


def qe_cubic_interpolate(table, q, dq):
    """``_native_fft.pyx:1556-1600``: QE four-point Lagrange table lookup."""
    if dq <= 0.0:
        raise ValueError("dq must be positive")
    scaled = q / dq
    lower = scaled.astype(np.int64)
    f = scaled - lower
    u, v, w = 1.0 - f, 2.0 - f, 3.0 - f
    t = np.asarray(table)
    return np.ascontiguousarray(
        t[lower] * (u * v * w / 6.0)[:, None]
        + t[lower + 1] * (f * v * w / 2.0)[:, None]
        - t[lower + 2] * (f * u * w / 2.0)[:, None]
        + t[lower + 3] * (f * u * v / 6.0)[:, None]
    )


_S_L0 = 1.0 / np.sqrt(4.0 * np.pi)
_S_L1 = np.sqrt(3.0 / (4.0 * np.pi))
_S_20 = np.sqrt(5.0 / (16.0 * np.pi))
_S_21 = np.sqrt(15.0 / (4.0 * np.pi))
_S_22 = np.sqrt(15.0 / (16.0 * np.pi))


def _unit_rows(vectors, lengths):
    q = np.asarray(lengths)
    safe = q > 1.0e-14
    inv = np.where(safe, 1.0 / np.where(safe, q, 1.0), 0.0)
    x = np.where(safe, vectors[:, 0] * inv, 0.0)
    y = np.where(safe, vectors[:, 1] * inv, 0.0)
    z = np.where(safe, vectors[:, 2] * inv, 1.0)
    return x, y, z


def _harmonic(l, channel, x, y, z):
    if l == 0:
        return np.full_like(x, _S_L0)
    if l == 1:
        return (_S_L1 * z, -_S_L1 * x, -_S_L1 * y)[channel]
    return (
        _S_20 * (3.0 * z * z - 1.0), -_S_21 * x * z, -_S_21 * y * z,
        _S_22 * (x * x - y * y), _S_21 * x * y,
    )[channel]


def low_l_real_harmonics(angular_momentum, vectors, lengths):
    """``_native_fft.pyx:1603-1661``: QE ``ylmr2`` for l <= 2."""
    if angular_momentum < 0 or angular_momentum > 2:
        raise ValueError("native harmonics support l=0,1,2")
    x, y, z = _unit_rows(vectors, lengths)
    return np.stack(
        [_harmonic(angular_momentum, m, x, y, z) for m in range(2 * angular_momentum + 1)],
        axis=1,
    )


def phase_matrix(vectors, positions):
    """``_native_fft.pyx:1664-1699``: ``exp(-i G.r)`` as cos - i sin."""
    angle = vectors @ positions.T
    return np.asfortranarray(np.cos(angle) - 1j * np.sin(angle))


def assemble_low_l_projectors(radial, vectors, lengths, radial_indices, angular_momenta, channels):
    """``_native_fft.pyx:1702-1791``: (-i)^l Y_lm(q) beta_l(q) columns."""
    x, y, z = _unit_rows(vectors, lengths)
    out = np.empty((vectors.shape[0], radial_indices.size), dtype=np.complex128, order="F")
    for column in range(radial_indices.size):
        l = int(angular_momenta[column])
        value = radial[:, int(radial_indices[column])] * _harmonic(l, int(channels[column]), x, y, z)
        if l == 0:
            out[:, column] = value
        elif l == 1:
            out[:, column] = -1j * value
        else:
            out[:, column] = -value
    return out


def project_density_stars(coefficients, offsets, members, weight_table, weight_indices,
                          fill_table, fill_indices):
    """``_native_fft.pyx:1806-1879``: reciprocal star projector, in place."""
    rows = np.asarray(members, dtype=np.int64)
    w = weight_table[np.asarray(weight_indices, dtype=np.int64)]
    f = fill_table[np.asarray(fill_indices, dtype=np.int64)]
    off = np.asarray(offsets, dtype=np.int64)
    star_of = np.repeat(np.arange(off.size - 1), np.diff(off))
    averaged = np.zeros(off.size - 1, dtype=np.complex128)
    np.add.at(averaged, star_of, w * coefficients[rows])
    coefficients[rows] = f * averaged[star_of]


def hartree_coefficients(density_coefficients, g2, potential_coefficients):
    """``_native_fft.pyx:1882-1919``: ``4 pi rho(G)/G^2``, zero at G=0."""
    mask = g2 > 1.0e-14
    potential_coefficients[...] = 0.0
    potential_coefficients[mask] = 4.0 * np.pi * density_coefficients[mask] / g2[mask]


def hartree_residual_metric(residual_coefficients, g2):
    """``_native_fft.pyx:1922-1970``: Neumaier-compensated
    ``sum 4 pi |drho(G)|^2 / G^2`` over G != 0."""
    mask = g2 > 1.0e-14
    terms = (4.0 * np.pi) * (
        residual_coefficients[mask].real ** 2 + residual_coefficients[mask].imag ** 2
    ) / g2[mask]
    total = 0.0
    correction = 0.0
    for term in terms.tolist():
        updated = total + term
        if total >= term:
            correction += (total - updated) + term
        else:
            correction += (term - updated) + total
        total = updated
    return total + correction


def _unavailable(*_args, **_kwargs):
    raise NotImplementedError("the oracle restates the single-rank hot path only")


apply_streamed = _unavailable
accumulate_density_distributed = _unavailable
tetrahedron_integrated_sum = _unavailable
tetrahedron_dos_sums = _unavailable
tetrahedron_accumulate = _unavailable
