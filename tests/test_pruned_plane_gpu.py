"""The pruned plane pass of the 64-point four-step planes.

When every stick of a plan lies within the rows and columns [0, 16) and
[48, 64) of a 64 x 64 plane (K = 2 blocks of N2 = 8 at each end), pass B
keeps only those 32 rows and skips the D1 blocks 2..5 that are zero on input
to the inverse line transforms and unread after the forward ones.  Every
step adds or multiplies the same values as the active-row plane pass, so the
two give the same output bit for bit (QEB_PRUNE_PLANE=0 builds a plan on
the active-row plane).  Both are checked against the oracle's apply_serial
(qepy_pw/_native_fft.pyx:2338-2455); a basis whose sticks reach past the
kept rows stays on the active-row plane.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import native_fft as oracle
from qe_python_b200.basis import LocalPotentialWorkspace, grid_slots, make_bases, fft_shape

pytestmark = pytest.mark.gpu

CUBIC = np.eye(3) * 15.8


def _case(ecut, ecutrho, nbands, seed):
    reciprocal = 2.0 * np.pi * np.linalg.inv(CUBIC).T
    basis = make_bases(reciprocal, np.zeros(3), ecut)[0]
    shape = fft_shape([basis], reciprocal, ecutrho)
    rng = np.random.default_rng(seed)
    npw = len(basis)
    psi = np.asfortranarray(rng.standard_normal((npw, nbands))
                            + 1j * rng.standard_normal((npw, nbands)))
    v = np.ascontiguousarray(rng.uniform(-1.0, 1.0, shape))
    return basis, shape, psi, v


def _oracle_apply(basis, shape, psi, v):
    linear, _z, _p, _s = grid_slots(basis.indices, shape)
    size = int(np.prod(shape))
    grid = np.zeros((psi.shape[1], size), dtype=np.complex128)
    plan = oracle.NativeFFTWPlan(grid, shape, psi.shape[1], 1, size)
    result = np.zeros_like(psi)
    oracle.apply_serial(grid, psi, v, linear, plan, size, size, result, 0, basis.kinetic)
    return result


def _apply(ws, psi, v, kinetic):
    import torch

    return ws.apply(torch.from_numpy(v).cuda(), torch.from_numpy(psi).cuda(),
                    diagonal=torch.from_numpy(kinetic).cuda()).cpu().numpy()


@pytest.mark.parametrize("precision,rtol", [("f64", 1.0e-12), ("f32", 2.0e-5)])
def test_pruned_plane_equals_the_active_row_plane(cuda_device, monkeypatch, precision, rtol):
    basis, shape, psi, v = _case(30.0, 150.0, nbands=5, seed=21)
    assert shape == (64, 64, 64)
    coords = np.asarray(basis.indices)[:, :2]
    assert np.max(np.abs(coords)) < 16  # every stick inside the kept rows
    pruned = LocalPotentialWorkspace(basis, shape, precision=precision)
    assert pruned.pruned_plane == 2
    monkeypatch.setenv("QEB_PRUNE_PLANE", "0")
    plain = LocalPotentialWorkspace(basis, shape, precision=precision)
    assert plain.pruned_plane == 0
    got = _apply(pruned, psi, v, basis.kinetic)
    want = _apply(plain, psi, v, basis.kinetic)
    assert np.array_equal(got, want)
    expected = _oracle_apply(basis, shape, psi, v)
    err = np.max(np.abs(got.astype(np.complex128) - expected))
    assert err <= rtol * np.max(np.abs(expected))


def test_sticks_past_the_kept_rows_use_the_active_row_plane(cuda_device):
    # ecutrho = 2.4 ecutwfc: the wave-function sphere reaches |x| >= 16 on 64 points
    basis, shape, psi, v = _case(60.0, 144.0, nbands=3, seed=22)
    assert shape == (64, 64, 64)
    assert np.max(np.abs(np.asarray(basis.indices)[:, :2])) >= 16
    ws = LocalPotentialWorkspace(basis, shape)
    assert ws.pruned_plane == 0
    got = _apply(ws, psi, v, basis.kinetic)
    expected = _oracle_apply(basis, shape, psi, v)
    assert np.max(np.abs(got - expected)) <= 1.0e-12 * np.max(np.abs(expected))


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_pruned_plane_in_a_k_point_batch(cuda_device, monkeypatch, precision):
    """Several k points in one launch per pass (qeb_apply_local_multi), each
    with its own slot tables: the same bits as the active-row plane batch."""
    import torch

    from qe_python_b200.basis import apply_local_multi
    from qe_python_b200.device import empty_f, to_device_f

    reciprocal = 2.0 * np.pi * np.linalg.inv(CUBIC).T
    ks = np.array([[0.0, 0.0, 0.0], [0.25, 0.0, 0.0], [0.25, 0.25, 0.0], [0.5, 0.5, 0.5]])
    bases = make_bases(reciprocal, ks, 30.0)
    shape = fft_shape(bases, reciprocal, 150.0)
    assert shape == (64, 64, 64)
    rng = np.random.default_rng(23)
    v = torch.from_numpy(rng.uniform(-1.0, 1.0, shape)).cuda()
    cdt = torch.complex64 if precision == "f32" else torch.complex128
    rdt = torch.float32 if precision == "f32" else torch.float64

    def run(env):
        if env is not None:
            monkeypatch.setenv("QEB_PRUNE_PLANE", env)
        else:
            monkeypatch.delenv("QEB_PRUNE_PLANE", raising=False)
        workspaces = [LocalPotentialWorkspace(b, shape, precision=precision) for b in bases]
        local = np.random.default_rng(24)
        vectors, targets, kinetics = [], [], []
        for i, b in enumerate(bases):
            nb = 3 + i  # uneven band counts, odd and even (two bands per block)
            psi = local.standard_normal((len(b), nb)) + 1j * local.standard_normal((len(b), nb))
            vectors.append(to_device_f(psi, cdt, torch.device("cuda")))
            targets.append(empty_f(len(b), nb, cdt, torch.device("cuda")))
            kinetics.append(torch.from_numpy(np.asarray(b.kinetic)).cuda().to(rdt))
        potential = workspaces[0].native_potential(v, False)
        apply_local_multi(workspaces, potential, vectors, kinetics, targets)
        torch.cuda.synchronize()
        return [w.pruned_plane for w in workspaces], [t.cpu() for t in targets]

    flags, pruned = run(None)
    assert flags == [2] * len(bases)
    flags0, plain = run("0")
    assert flags0 == [0] * len(bases)
    for got, want in zip(pruned, plain):
        assert torch.equal(got, want)
