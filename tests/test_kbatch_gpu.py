"""All k points in one launch per FFT pass (qeb_apply_local_multi) and the
lockstep Davidson built on it: a batched H application is bit-identical to
the k-by-k one (single plans run through the same batched kernels)."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cell(precision, ks=None):
    import torch

    from qe_python_b200.basis import LocalPotentialWorkspace, fft_shape, make_bases
    from qe_python_b200.diagonalization import PlaneWaveHamiltonian
    from qe_python_b200.pseudo_tables import SpeciesTables
    from qe_python_b200.scf import benchmark_system, projector_terms
    from qe_python_b200.symmetry import fft_factors

    system = benchmark_system("scf-fcc2")
    kpoints = system.kpoints if ks is None else system.kpoints[ks]
    bases = make_bases(system.reciprocal, kpoints, system.ecutwfc)
    shape = fft_shape(bases, system.reciprocal, system.ecutrho, fft_factors(system.operations))
    tables = {l: SpeciesTables(p, system.volume) for l, p in system.pseudos.items()}
    rng = np.random.default_rng(3)
    potential = torch.from_numpy(rng.uniform(-0.5, 0.5, shape)).cuda()
    hams = []
    for basis in bases:
        ws = LocalPotentialWorkspace(basis, shape, precision=precision)
        hams.append(PlaneWaveHamiltonian(basis, None, projector_terms(system, tables, basis),
                                         local_workspace=ws, real_potential=potential,
                                         potential_average=0.0))
    return hams, rng


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_batched_local_and_full_apply_equal_per_k(cuda_device, precision):
    import torch

    from qe_python_b200.basis import apply_local_multi
    from qe_python_b200.device import empty_f, to_device_f
    from qe_python_b200.diagonalization import apply_hamiltonians

    hams, rng = _cell(precision)
    vectors, targets, expected = [], [], []
    for i, ham in enumerate(hams):
        nb = 3 + (i % 4)  # uneven band counts per k point
        npw = len(ham.basis)
        psi = rng.standard_normal((npw, nb)) + 1j * rng.standard_normal((npw, nb))
        v = to_device_f(psi, ham.dtype, ham.device)
        vectors.append(v)
        targets.append(empty_f(npw, nb, ham.dtype, ham.device))
        expected.append(ham.apply(v))
    # the local part alone against the per-k local launches
    local = [empty_f(t.shape[0], t.shape[1], t.dtype, t.device) for t in targets]
    apply_local_multi([h.local_workspace for h in hams], hams[0]._potential, vectors,
                      [h._kinetic_kernel for h in hams], local)
    for ham, v, out in zip(hams, vectors, local):
        ref = empty_f(out.shape[0], out.shape[1], out.dtype, out.device)
        ham.local_workspace._launch_apply(ham._potential, v, ham._kinetic_kernel, ref)
        assert torch.equal(out, ref)
    apply_hamiltonians(hams, [(i, v, t) for i, (v, t) in enumerate(zip(vectors, targets))])
    torch.cuda.synchronize()
    for out, ref in zip(targets, expected):
        assert torch.equal(out, ref)


def test_lockstep_scf_reproduces_k_by_k_scf(cuda_device):
    """The H applications are bit-identical; the density kernel sums bands
    with FP64 atomics, whose order varies from run to run, so two SCFs agree
    to the last bits rather than bit for bit: energies to 1e-12 relative,
    eigenvalues to 2e-9 Ha (the refined iterations stop once eigenvalues
    move less than their threshold, at least 1e-3 x conv_thr = 1e-11 Ha, so
    two paths' last eigenvalues differ by a few 1e-10)."""
    from qe_python_b200.scf import benchmark_system, run_scf

    a = run_scf(benchmark_system("scf-fcc2"), precision="mixed", batch_kpoints=True)
    b = run_scf(benchmark_system("scf-fcc2"), precision="mixed", batch_kpoints=False)
    assert a.converged and b.converged
    assert len(a.energies_ha) == len(b.energies_ha)
    np.testing.assert_allclose(a.energies_ha, b.energies_ha, rtol=1e-12, atol=0)
    for x, y in zip(a.eigenvalues_ha, b.eigenvalues_ha):
        np.testing.assert_allclose(x, y, rtol=0, atol=2e-9)
