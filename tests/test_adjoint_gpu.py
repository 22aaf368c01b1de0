"""Hand-written adjoint of the band energy against central finite differences.

Cell: the 8-atom displaced diamond cell (scf-dia8-disp) reduced to the Gamma
point and 16 bands so each solve takes seconds.  V_Hxc is a smooth seeded
field.  Checks:
  * d E_band / d V_Hxc along a smooth direction vs central differences
    (steps 1e-4 and 5e-5, Richardson-extrapolated)
  * d E_band / d tau for two coordinates vs central differences, h = 1e-3 and
    5e-4 bohr, Richardson-extrapolated
    (tolerance 1e-5 Ha/bohr = 2e-5 Ry/bohr, well inside the 1e-4 Ry/bohr bar)
  * the mixed-precision gradient (FP32/split-TF32 solve, FP64 polish)
    against the FP64 gradient (1e-4 Ry/bohr).
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(precision):
    from qe_python_b200.adjoint import BandProblem
    from qe_python_b200.scf import benchmark_system

    system = benchmark_system("scf-dia8-disp")
    system.kpoints = np.zeros((1, 3))
    system.weights = np.ones(1)
    system.nbnd = 16
    return BandProblem(system, precision=precision, tolerance=1e-10)


def _smooth(shape, seed, amplitude):
    rng = np.random.default_rng(seed)
    grid = np.indices(shape).reshape(3, -1).T / np.array(shape)
    field = np.zeros(len(grid))
    for _ in range(6):
        k = rng.integers(-2, 3, 3)
        field += rng.uniform(-1, 1) * np.cos(2 * np.pi * grid @ k + rng.uniform(0, 2 * np.pi))
    return amplitude * field.reshape(shape)


def test_band_energy_gradients_match_finite_differences(cuda_device):
    import torch

    from qe_python_b200.adjoint import BandEnergy

    problem = _problem("f64")
    v = torch.from_numpy(_smooth(problem.shape, 1, 0.2)).cuda().requires_grad_(True)
    tau = torch.from_numpy(problem.system.positions.copy()).cuda().requires_grad_(True)
    energy = BandEnergy.apply(v, tau, problem)
    energy.backward()
    dv = _smooth(problem.shape, 2, 1.0)

    def e_at(vv, pos):
        return problem.solve(vv, pos)[0]

    def richardson(f, step):
        # central differences at step and step/2 combined to cancel the
        # O(step^2) truncation term: (4 D(h/2) - D(h)) / 3
        d1 = (f(step) - f(-step)) / (2 * step)
        d2 = (f(step / 2) - f(-step / 2)) / step
        return (4.0 * d2 - d1) / 3.0, d1

    base_v = v.detach().cpu().numpy()
    base_tau = problem.system.positions.copy()
    fd_v, plain_v = richardson(lambda e: e_at(base_v + e * dv, base_tau), 1e-4)
    an_v = float(np.sum(v.grad.cpu().numpy() * dv))
    assert abs(fd_v - an_v) <= 1e-6 * max(1.0, abs(fd_v)), (fd_v, plain_v, an_v)

    def moved(atom, axis, e):
        pos = base_tau.copy()
        pos[atom, axis] += e
        return pos

    for atom, axis in ((0, 0), (3, 2)):
        fd, plain = richardson(lambda e: e_at(base_v, moved(atom, axis, e)), 1e-3)
        an = float(tau.grad[atom, axis])
        assert abs(fd - an) < 1e-5, (atom, axis, fd, plain, an)


def test_mixed_gradient_matches_fp64(cuda_device):
    import torch

    from qe_python_b200.adjoint import BandEnergy

    grads = []
    for precision in ("f64", "mixed"):
        problem = _problem(precision)
        v = torch.from_numpy(_smooth(problem.shape, 1, 0.2)).cuda().requires_grad_(True)
        tau = torch.from_numpy(problem.system.positions.copy()).cuda().requires_grad_(True)
        BandEnergy.apply(v, tau, problem).backward()
        grads.append(tau.grad.cpu().numpy())
    assert np.max(np.abs(grads[0] - grads[1])) * 2.0 < 1e-4  # Ry/bohr
