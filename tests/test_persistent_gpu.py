"""The persistent form of the local passes (one cooperative launch with grid
barriers between pass A, B and C, qeb_set_persistent_passes) against the
three launches: bit for bit, for one k point in both precisions, for a
batch of four k points with different band counts, and replayed from a
captured CUDA graph; no barrier gives up (error word zero)."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _apply(ham, psi):
    import torch

    out = torch.empty_like(psi.T).T
    ham.local_workspace._launch_apply(ham._potential, psi, ham._kinetic_kernel, out)
    torch.cuda.synchronize()
    return out


def test_persistent_passes_equal_three_launches(cuda_device):
    import torch

    from qe_python_b200 import kernels as K
    from qe_python_b200.basis import (LocalPotentialWorkspace, apply_local_multi, make_bases,
                                      persistent_passes, set_persistent_passes)
    from qe_python_b200.device import to_device_f
    from qe_python_b200.diagonalization import HpsiGraph, PlaneWaveHamiltonian
    from qe_python_b200.scf import benchmark_system, scf_setup, starting_hamiltonians
    from qe_python_b200.workloads import hpsi_microbench

    work = hpsi_microbench(nbands=96)
    basis = make_bases(work.reciprocal, np.zeros(3), 30.0)[0]
    try:
        for precision in ("f32", "f64"):
            ws = LocalPotentialWorkspace(basis, work.shape, precision=precision)
            ham = PlaneWaveHamiltonian(basis, None, ((work.beta, work.coupling),),
                                       local_workspace=ws,
                                       real_potential=torch.from_numpy(work.potential).cuda(),
                                       potential_average=0.0)
            psi = to_device_f(work.psi, ham.dtype, cuda_device)
            set_persistent_passes(False)
            three = _apply(ham, psi)
            set_persistent_passes(True)
            assert persistent_passes()
            one = _apply(ham, psi)
            assert torch.equal(one, three), precision
            graph = HpsiGraph(ham, 96)
            replayed = graph(psi)
            set_persistent_passes(False)
            assert torch.equal(replayed, graph(psi)), precision  # the captured launch stays
            assert torch.equal(ham.apply(psi), replayed), precision
        # a batch of four k points with different band counts
        system = benchmark_system("scf-dia64")
        hams, _v, _setup = starting_hamiltonians(system, "f32")
        rng = np.random.default_rng(1)
        blocks = [to_device_f(rng.standard_normal((len(h.basis), nb))
                              + 1j * rng.standard_normal((len(h.basis), nb)),
                              torch.complex64, cuda_device) for h, nb in zip(hams, (7, 33, 16, 1))]
        results = {}
        for mode in (False, True):
            set_persistent_passes(mode)
            targets = [torch.empty_like(b.T).T for b in blocks]
            apply_local_multi([h.local_workspace for h in hams], hams[0]._potential, blocks,
                              [h._kinetic_kernel for h in hams], targets)
            torch.cuda.synchronize()
            results[mode] = targets
        for a, b in zip(results[False], results[True]):
            assert torch.equal(a, b)
        assert K.tf32_error() == 0
    finally:
        set_persistent_passes(False)
