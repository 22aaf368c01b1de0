"""Plans of different sizes share kernels: creating a smaller plan after a
larger one must not lower the larger plan's shared-memory limit (a launch
would then fail).  Both plans are used after both exist and checked against
the oracle (qepy_pw/_native_fft.pyx:2338-2455)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import native_fft as oracle
from qe_python_b200.basis import LocalPotentialWorkspace, fft_shape, grid_slots, make_bases

pytestmark = pytest.mark.gpu


def _oracle(miller, shape, psi, v):
    linear, *_ = grid_slots(miller, shape)
    size = int(np.prod(shape))
    grid = np.zeros((psi.shape[1], size), dtype=np.complex128)
    plan = oracle.NativeFFTWPlan(grid, shape, psi.shape[1], 1, size)
    out = np.zeros_like(psi)
    oracle.apply_serial(grid, psi, v, linear, plan, size, size, out, 0, None)
    return out


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_large_plan_after_small_plan(cuda_device, precision):
    import torch

    lattice = 10.26 / 2.0 * np.array([[-1.0, 0.0, 1.0], [0.0, 1.0, 1.0], [-1.0, 1.0, 0.0]])
    reciprocal = 2.0 * np.pi * np.linalg.inv(lattice).T
    large = make_bases(reciprocal, np.array([0.125, 0.375, 0.0]), 20.0)[0]
    small = make_bases(reciprocal, np.zeros(3), 4.0)[0]
    shape = fft_shape([large], reciprocal, 80.0)
    rng = np.random.default_rng(5)
    v = np.ascontiguousarray(rng.uniform(-1, 1, shape))
    ws_large = LocalPotentialWorkspace(large, shape, precision=precision)
    ws_small = LocalPotentialWorkspace(small, shape, precision=precision)
    tol = 1e-12 if precision == "f64" else 2e-5
    for basis, ws in ((large, ws_large), (small, ws_small)):
        psi = np.asfortranarray(rng.standard_normal((len(basis), 3)) + 1j * rng.standard_normal((len(basis), 3)))
        want = _oracle(basis.indices, shape, psi, v)
        got = ws.apply(torch.from_numpy(v).cuda(), torch.from_numpy(psi).cuda()).cpu().numpy()
        assert np.max(np.abs(got - want)) <= tol * np.max(np.abs(want))
        rho = torch.zeros(shape, dtype=torch.float64, device="cuda")
        ws.accumulate_density(rho, torch.from_numpy(psi).cuda(), torch.ones(3, dtype=torch.float64, device="cuda"))
        assert float(rho.sum()) > 0.0
