"""GPU parity of the local H|psi> operator and density against the oracle.

The oracle restates the reference's serial kernels (apply_serial,
apply_serial_spatial, accumulate_density_serial; qepy_pw/_native_fft.pyx
:2338-2648) in NumPy.  FP64 results must agree to 1e-12 relative to the
largest output entry; the FP32 chosen form to 2e-5.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import native_fft as oracle
from qe_python_b200.basis import (
    LocalPotentialWorkspace,
    grid_slots,
    make_bases,
    fft_shape,
    potential_matrix,
)

pytestmark = pytest.mark.gpu

FP64_RTOL = 1.0e-12
FP32_RTOL = 2.0e-5


def _case(lattice, k, ecut, ecutrho, nbands, seed):
    reciprocal = 2.0 * np.pi * np.linalg.inv(lattice).T
    basis = make_bases(reciprocal, k, ecut)[0]
    shape = fft_shape([basis], reciprocal, ecutrho)
    rng = np.random.default_rng(seed)
    npw = len(basis)
    psi = np.asfortranarray(rng.standard_normal((npw, nbands)) + 1j * rng.standard_normal((npw, nbands)))
    v = np.ascontiguousarray(rng.uniform(-1.0, 1.0, shape))
    return basis, shape, psi, v


def _oracle_apply(basis, shape, psi, v, kinetic=None):
    linear, _z, _p, _s = grid_slots(basis.indices, shape)
    size = int(np.prod(shape))
    grid = np.zeros((psi.shape[1], size), dtype=np.complex128)
    plan = oracle.NativeFFTWPlan(grid, shape, psi.shape[1], 1, size)
    result = np.zeros_like(psi)
    oracle.apply_serial(grid, psi, v, linear, plan, size, size, result, 0, kinetic)
    return result


FCC = 10.26 / 2.0 * np.array([[-1.0, 0.0, 1.0], [0.0, 1.0, 1.0], [-1.0, 1.0, 0.0]])
CASES = [
    ("fcc-24", FCC, np.array([0.125, 0.125, 0.375]), 20.0, 80.0),
    ("cubic-64", np.eye(3) * 15.8, np.zeros(3), 30.0, 150.0),
    ("tilted", np.array([[9.0, 0.4, 0.0], [0.3, 11.0, 0.2], [0.0, 0.7, 13.0]]),
     np.array([0.3, -0.2, 0.1]), 18.0, 72.0),
    ("diamond-36", np.eye(3) * 10.26, np.array([1 / 3, 0.0, 1 / 3]), 25.0, 100.0),
]


@pytest.mark.parametrize("name,lattice,k,ecut,ecutrho", CASES, ids=[c[0] for c in CASES])
def test_apply_local_fp64_matches_oracle(cuda_device, name, lattice, k, ecut, ecutrho):
    import torch

    basis, shape, psi, v = _case(lattice, k, ecut, ecutrho, nbands=6, seed=7)
    kinetic = basis.kinetic
    expected = _oracle_apply(basis, shape, psi, v, kinetic)
    ws = LocalPotentialWorkspace(basis, shape)
    got = ws.apply(torch.from_numpy(v).cuda(), torch.from_numpy(psi).cuda(),
                   diagonal=torch.from_numpy(kinetic).cuda())
    got = got.cpu().numpy()
    scale = np.max(np.abs(expected))
    assert np.max(np.abs(got - expected)) <= FP64_RTOL * scale


def test_apply_local_native_layout_and_spatial_oracle(cuda_device):
    """The native (nz, nx, ny) potential layout of apply_serial_spatial."""
    import torch

    basis, shape, psi, v = _case(FCC, np.array([0.25, 0.0, 0.5]), 20.0, 80.0, nbands=5, seed=3)
    _l, zslots, positions, _s = grid_slots(basis.indices, shape)
    native = np.ascontiguousarray(np.moveaxis(v, 2, 0))
    size = int(np.prod(shape))
    grid = np.zeros((5, size), dtype=np.complex128)
    expected = np.zeros_like(psi)
    oracle.apply_serial_spatial(grid, psi, native, zslots, positions, None, None, size, size,
                                expected, 0, basis.kinetic)
    ws = LocalPotentialWorkspace(basis, shape)
    got = ws.apply(torch.from_numpy(native).cuda(), torch.from_numpy(psi).cuda(),
                   native_potential_layout=True, diagonal=torch.from_numpy(basis.kinetic).cuda())
    assert np.max(np.abs(got.cpu().numpy() - expected)) <= FP64_RTOL * np.max(np.abs(expected))


def test_convolution_identity(cuda_device):
    """The reference's own known answer (tests/unit/core/test_basis.py:76-88):
    FFT application equals the explicit convolution to 2e-14."""
    shape = (6, 6, 6)
    grid = np.indices(shape).sum(axis=0)
    potential_r = 0.3 + 0.2 * np.cos(2.0 * np.pi * grid / shape[0])
    potential_g = np.fft.fftn(potential_r) / np.prod(shape)
    indices = np.asarray([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0]], dtype=np.int32)
    coefficients = np.asarray([1.0 + 0.2j, -0.3j, 0.4, -0.1 + 0.5j])
    expected = potential_matrix(potential_g, indices) @ coefficients
    ws = LocalPotentialWorkspace(indices, shape)
    actual = ws.apply(ws.prepare_potential(potential_g), coefficients)
    np.testing.assert_allclose(actual, expected, atol=2.0e-14)


def test_apply_local_strided_columns_and_batches(cuda_device):
    """ld > npw, a column offset in the output and bounded band batches."""
    import torch

    basis, shape, psi, v = _case(FCC, np.zeros(3), 20.0, 80.0, nbands=9, seed=11)
    npw = len(basis)
    expected = _oracle_apply(basis, shape, psi, v, None)
    ld = npw + 13
    storage = torch.zeros((12, ld), dtype=torch.complex128, device="cuda")
    storage[:9, :npw] = torch.from_numpy(psi.T.copy()).cuda()
    psi_view = storage.T[:npw, :9]
    out_storage = torch.zeros((14, ld), dtype=torch.complex128, device="cuda")
    out_view = out_storage.T[:npw, 3:12]
    ws = LocalPotentialWorkspace(basis, shape, serial_fft_batch_size=4)
    ws.apply(torch.from_numpy(v).cuda(), psi_view, out=out_view)
    got = out_storage.T[:npw, 3:12].cpu().numpy()
    assert np.max(np.abs(got - expected)) <= FP64_RTOL * np.max(np.abs(expected))
    assert torch.count_nonzero(out_storage[:3]) == 0
    assert torch.count_nonzero(out_storage[12:]) == 0


def test_apply_local_fp32_chosen_form(cuda_device):
    import torch

    basis, shape, psi, v = _case(np.eye(3) * 15.8, np.zeros(3), 30.0, 150.0, nbands=4, seed=5)
    expected = _oracle_apply(basis, shape, psi, v, basis.kinetic)
    ws = LocalPotentialWorkspace(basis, shape, precision="f32")
    got = ws.apply(torch.from_numpy(v).cuda(), torch.from_numpy(psi).cuda(),
                   diagonal=torch.from_numpy(basis.kinetic).cuda())
    assert got.dtype == torch.complex64
    err = np.max(np.abs(got.cpu().numpy().astype(np.complex128) - expected))
    assert err <= FP32_RTOL * np.max(np.abs(expected))


def test_host_arrays_round_trip(cuda_device):
    """NumPy in, NumPy out (the end-to-end path of the drop-in API)."""
    basis, shape, psi, v = _case(FCC, np.zeros(3), 20.0, 80.0, nbands=3, seed=2)
    expected = _oracle_apply(basis, shape, psi, v, basis.kinetic)
    ws = LocalPotentialWorkspace(basis, shape)
    got = ws.apply(v, psi, diagonal=basis.kinetic)
    assert isinstance(got, np.ndarray)
    assert np.max(np.abs(got - expected)) <= FP64_RTOL * np.max(np.abs(expected))
    single = ws.apply(v, psi[:, 1], diagonal=basis.kinetic)
    assert single.shape == (len(basis),)
    assert np.max(np.abs(single - expected[:, 1])) <= FP64_RTOL * np.max(np.abs(expected))


@pytest.mark.parametrize("precision,rtol", [("f64", 1.0e-12), ("f32", 2.0e-5)])
def test_accumulate_density_matches_oracle(cuda_device, precision, rtol):
    import torch

    basis, shape, psi, _v = _case(FCC, np.array([0.125, 0.25, 0.0]), 20.0, 80.0, nbands=7, seed=9)
    weights = np.linspace(0.2, 1.0, 7)
    linear, _z, _p, _s = grid_slots(basis.indices, shape)
    size = int(np.prod(shape))
    expected = np.full(shape, 0.5)
    grid = np.zeros((7, size), dtype=np.complex128)
    plan = oracle.NativeFFTWPlan(grid, shape, 7, 1, size)
    oracle.accumulate_density_serial(expected, grid, psi, weights, linear, plan, size, size)
    ws = LocalPotentialWorkspace(basis, shape, precision=precision)
    rho = torch.full(shape, 0.5, dtype=torch.float64, device="cuda")
    ws.accumulate_density(rho, torch.from_numpy(psi).cuda(), torch.from_numpy(weights).cuda())
    err = np.max(np.abs(rho.cpu().numpy() - expected))
    assert err <= rtol * np.max(np.abs(expected))


def test_bad_shapes_raise(cuda_device):
    import torch

    basis, shape, psi, v = _case(FCC, np.zeros(3), 20.0, 80.0, nbands=2, seed=1)
    ws = LocalPotentialWorkspace(basis, shape)
    with pytest.raises(ValueError):
        ws.apply(torch.from_numpy(v).cuda(), torch.zeros((len(basis) + 1, 2), dtype=torch.complex128, device="cuda"))
    with pytest.raises(ValueError):
        ws.apply(torch.zeros((5, 5, 5), dtype=torch.float64, device="cuda"), torch.from_numpy(psi).cuda())
    empty = ws.apply(torch.from_numpy(v).cuda(), torch.zeros((len(basis), 0), dtype=torch.complex128, device="cuda"))
    assert tuple(empty.shape) == (len(basis), 0)
