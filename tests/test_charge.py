"""Device charge-grid steps against their host restatements (CPU tensors).

qe_python_b200.charge runs the SCF's density-grid work on the GPU in FP64;
the same code on CPU tensors must reproduce the host versions in
qe_python_b200.scf / pseudo_tables (which are pinned to the reference by
tests/test_scf_setup.py) to FP64 round-off.
"""

from __future__ import annotations

import numpy as np
import torch

from qe_python_b200.charge import DeviceBroydenMixer, DeviceChargeGrid, DeviceLinearMixer
from qe_python_b200.charge import pz81 as device_pz81
from qe_python_b200.pseudo_tables import pz81
from qe_python_b200.scf import BroydenMixer, ChargeGrid, LinearMixer, hartree, neumaier_metric


def _grid():
    lattice = 10.26 / 2.0 * np.array([[-1.0, 0.0, 1.0], [0.0, 1.0, 1.0], [-1.0, 1.0, 0.0]])
    reciprocal = 2.0 * np.pi * np.linalg.inv(lattice).T
    return ChargeGrid((15, 15, 15), reciprocal, 80.0)


def _density(shape, seed):
    rng = np.random.default_rng(seed)
    return 0.05 + 0.02 * rng.random(shape)


def test_transforms_hartree_metric_and_lda():
    host = _grid()
    dev = DeviceChargeGrid(host, torch.device("cpu"))
    rho = _density(host.shape, 1)
    rho_t = torch.from_numpy(rho)
    g_host = host.to_g(rho)
    g_dev = dev.to_g(rho_t).numpy()
    np.testing.assert_allclose(g_dev, g_host, rtol=0, atol=1e-16)
    np.testing.assert_allclose(dev.to_r(torch.from_numpy(g_host)).numpy(), host.to_r(g_host),
                               rtol=0, atol=1e-15)
    np.testing.assert_allclose(dev.hartree(torch.from_numpy(g_host)).numpy(),
                               hartree(g_host, host.g2), rtol=1e-15, atol=0)
    res = g_host - host.to_g(_density(host.shape, 2))
    assert abs(dev.residual_metric(torch.from_numpy(res)) - neumaier_metric(res, host.g2)) \
        <= 1e-14 * neumaier_metric(res, host.g2)
    dens = 10.0 ** np.random.default_rng(3).uniform(-12, 1, 3000)
    dens[:5] = [0.0, 1e-11, 1e-10, 2e-10, -0.3]
    e_h, v_h = pz81(dens)
    e_d, v_d = device_pz81(torch.from_numpy(dens))
    np.testing.assert_allclose(e_d.numpy(), e_h, rtol=1e-14, atol=1e-300)
    np.testing.assert_allclose(v_d.numpy(), v_h, rtol=1e-14, atol=1e-300)


def test_mixers_match_host_over_several_steps():
    host = _grid()
    dev = DeviceChargeGrid(host, torch.device("cpu"))
    hb = BroydenMixer(host, 0.7, 4, 80.0)
    db = DeviceBroydenMixer(dev, 0.7, 4)
    rho_h = _density(host.shape, 4)
    rho_d = torch.from_numpy(rho_h.copy())
    for step in range(7):  # past the history length: exercises the cyclic slot
        out = _density(host.shape, 10 + step)
        res_h = host.to_g(out - rho_h)
        rho_h = hb.mix(rho_h, res_h)
        rho_d = db.mix(rho_d, dev.to_g(torch.from_numpy(out) - rho_d))
        np.testing.assert_allclose(rho_d.numpy(), rho_h, rtol=0, atol=1e-13)
    lin_h, lin_d = LinearMixer(0.7), DeviceLinearMixer(0.7)
    a, b = _density(host.shape, 30), _density(host.shape, 31)
    np.testing.assert_array_equal(lin_d.mix(torch.from_numpy(a), torch.from_numpy(b)).numpy(),
                                  lin_h.mix(a, b))


def test_broyden_modes_match_reference_sequence():
    """tests/golden/broyden.npz: the reference's PlainBroydenMixer
    (qepy_pw/mixing.py:262-413) in 'plain' and 'TF' modes over seven steps."""
    from pathlib import Path

    from qe_python_b200.scf import thomas_fermi_g2  # noqa: F401  (TF screening)

    data = np.load(Path(__file__).resolve().parent / "golden" / "broyden.npz")
    lattice = data["lattice"]
    reciprocal = 2.0 * np.pi * np.linalg.inv(lattice).T
    volume = abs(np.linalg.det(lattice))
    host = ChargeGrid(tuple(data["shape"]), reciprocal, 20.0)
    dev = DeviceChargeGrid(host, torch.device("cpu"))
    for mode in ("plain", "TF"):
        hb = BroydenMixer(host, 0.7, 4, 20.0, mode=mode, nelec=8.0, volume=volume)
        db = DeviceBroydenMixer(dev, 0.7, 4, mode, 8.0, volume)
        rho_h = data["start"].copy()
        rho_d = torch.from_numpy(rho_h.copy())
        for out, expected in zip(data["outs"], data[f"mixed_{mode}"]):
            rho_h = hb.mix(rho_h, host.to_g(out - rho_h))
            rho_d = db.mix(rho_d, dev.to_g(torch.from_numpy(out) - rho_d))
            np.testing.assert_allclose(rho_h, expected, rtol=0, atol=1e-13)
            np.testing.assert_allclose(rho_d.numpy(), expected, rtol=0, atol=1e-13)
