"""The host density symmetrizer against the reference's own (CPU only).

qe_python_b200.symmetry.DensitySymmetrizer.apply restates the reference's
real-space symmetrizer (qepy_pw/symmetry.py:28-238): the same operations,
the same summation order, so the results agree bit for bit.  The GPU
kernel is checked against this restatement in tests/test_setup_kernels_gpu.py.
Needs the reference package (staged or mounted); skipped elsewhere.
"""

from __future__ import annotations

import numpy as np
import pytest

from tests.golden import reference_env


@pytest.mark.skipif(not reference_env.reference_available(),
                    reason="the reference package is not available")
@pytest.mark.parametrize("name", ["scf-fcc2", "scf-dia8-disp"])
def test_host_symmetrizer_matches_reference(name):
    reference_env.load_reference()
    from qepy_pw.symmetry import DensitySymmetrizer as Reference

    from qe_python_b200.basis import fft_shape, make_bases
    from qe_python_b200.scf import benchmark_system
    from qe_python_b200.symmetry import DensitySymmetrizer, fft_factors

    system = benchmark_system(name)
    bases = make_bases(system.reciprocal, system.kpoints, system.ecutwfc)
    shape = fft_shape(bases, system.reciprocal, system.ecutrho, fft_factors(system.operations))
    rho = np.random.default_rng(11).random(shape)
    ours = DensitySymmetrizer(system.operations, shape).apply(rho)
    theirs = Reference(shape, tuple(system.operations)).apply(rho)
    assert np.array_equal(ours, theirs)
    assert len(system.operations) > 1 or np.array_equal(ours, rho)
