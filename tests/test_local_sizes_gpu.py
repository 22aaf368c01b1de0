"""Four-step and generic FFT kernels on the benchmark grids (GPU).

The 90^3 and 135^3 grids of the 64- and 216-atom cells run through the
four-step register kernels; the same operator with QEB_FORCE_GENERIC=1 set at
plan creation runs the generic Stockham kernels.  Both must agree with the
oracle (apply_serial, qepy_pw/_native_fft.pyx:2338-2455) to 1e-12 (FP64).
"""

from __future__ import annotations

import os

import numpy as np
import pytest

from oracle import native_fft as oracle
from qe_python_b200.basis import LocalPotentialWorkspace, fft_shape, grid_slots, make_bases

pytestmark = pytest.mark.gpu


def _oracle(miller, shape, psi, v, kinetic):
    linear, *_ = grid_slots(miller, shape)
    size = int(np.prod(shape))
    grid = np.zeros((psi.shape[1], size), dtype=np.complex128)
    plan = oracle.NativeFFTWPlan(grid, shape, psi.shape[1], 1, size)
    out = np.zeros_like(psi)
    oracle.apply_serial(grid, psi, v, linear, plan, size, size, out, 0, kinetic)
    return out


def _workspace(basis, shape, precision, generic):
    previous = os.environ.get("QEB_FORCE_GENERIC")
    os.environ["QEB_FORCE_GENERIC"] = "1" if generic else "0"
    try:
        return LocalPotentialWorkspace(basis, shape, precision=precision)
    finally:
        if previous is None:
            del os.environ["QEB_FORCE_GENERIC"]
        else:
            os.environ["QEB_FORCE_GENERIC"] = previous


@pytest.mark.parametrize("length,ecut,ecutrho,expected", [
    (20.52, 30.0, 180.0, (90, 90, 90)),
    (30.78, 30.0, 180.0, (135, 135, 135)),
    (10.26, 25.0, 100.0, (36, 36, 36)),
])
def test_benchmark_grids_fast_and_generic(cuda_device, length, ecut, ecutrho, expected):
    import torch

    reciprocal = 2.0 * np.pi * np.linalg.inv(np.eye(3) * length).T
    basis = make_bases(reciprocal, np.array([0.0, 0.5, 0.0]) if length < 30 else np.zeros(3), ecut)[0]
    shape = fft_shape([basis], reciprocal, ecutrho)
    assert shape == expected
    rng = np.random.default_rng(int(length * 100))
    nb = 2
    psi = np.asfortranarray(rng.standard_normal((len(basis), nb)) + 1j * rng.standard_normal((len(basis), nb)))
    v = np.ascontiguousarray(rng.uniform(-1.0, 1.0, shape))
    expected_out = _oracle(basis.indices, shape, psi, v, basis.kinetic)
    scale = np.max(np.abs(expected_out))
    for generic in (False, True):
        ws = _workspace(basis, shape, "f64", generic)
        got = ws.apply(torch.from_numpy(v).cuda(), torch.from_numpy(psi).cuda(),
                       diagonal=torch.from_numpy(basis.kinetic).cuda()).cpu().numpy()
        assert np.max(np.abs(got - expected_out)) <= 1e-12 * scale, f"generic={generic}"
    ws = _workspace(basis, shape, "f32", False)
    got = ws.apply(torch.from_numpy(v).cuda(), torch.from_numpy(psi).cuda(),
                   diagonal=torch.from_numpy(basis.kinetic).cuda()).cpu().numpy()
    assert np.max(np.abs(got - expected_out)) <= 3e-5 * scale


@pytest.mark.parametrize("precision,rtol", [("f64", 1e-12), ("f32", 2e-5)])
def test_density_fast_matches_generic(cuda_device, precision, rtol):
    import torch

    reciprocal = 2.0 * np.pi * np.linalg.inv(np.eye(3) * 15.8).T
    basis = make_bases(reciprocal, np.zeros(3), 30.0)[0]
    shape = fft_shape([basis], reciprocal, 150.0)
    rng = np.random.default_rng(1)
    psi = torch.from_numpy(np.asfortranarray(rng.standard_normal((len(basis), 5))
                                             + 1j * rng.standard_normal((len(basis), 5)))).cuda()
    weights = torch.linspace(0.1, 1.0, 5, dtype=torch.float64, device="cuda")
    results = []
    for generic in (False, True):
        ws = _workspace(basis, shape, precision, generic)
        rho = torch.zeros(shape, dtype=torch.float64, device="cuda")
        ws.accumulate_density(rho, psi, weights)
        results.append(rho.cpu().numpy())
    assert np.max(np.abs(results[0] - results[1])) <= rtol * np.max(np.abs(results[1]))


FOUR_STEP_LENGTHS = (16, 24, 32, 36, 48, 64, 72, 90, 96, 108, 128, 135, 144, 180)


@pytest.mark.parametrize("n", FOUR_STEP_LENGTHS)
def test_every_four_step_length(cuda_device, n):
    """Each listed four-step length (cubic n^3 grid, G sphere of radius n/6)
    in both precisions against the oracle, the factor pairs with an odd N2
    (8 x 9, 9 x 15, 12 x 15) included: their line groups exchange through a
    buffer of stride N2."""
    import torch

    length = 10.0
    reciprocal = 2.0 * np.pi * np.linalg.inv(np.eye(3) * length).T
    ecut = (2.0 * np.pi * (n / 6.0) / length) ** 2
    basis = make_bases(reciprocal, np.zeros(3), ecut)[0]
    shape = (n, n, n)
    rng = np.random.default_rng(n)
    nb = 3
    psi = np.asfortranarray(rng.standard_normal((len(basis), nb)) + 1j * rng.standard_normal((len(basis), nb)))
    v = np.ascontiguousarray(rng.uniform(-1.0, 1.0, shape))
    expected_out = _oracle(basis.indices, shape, psi, v, basis.kinetic)
    scale = np.max(np.abs(expected_out))
    for precision, tol in (("f64", 1e-12), ("f32", 3e-5)):
        ws = _workspace(basis, shape, precision, False)
        got = ws.apply(torch.from_numpy(v).cuda(), torch.from_numpy(psi).cuda(),
                       diagonal=torch.from_numpy(basis.kinetic).cuda()).cpu().numpy()
        assert np.max(np.abs(got - expected_out)) <= tol * scale, precision
