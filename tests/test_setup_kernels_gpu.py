"""Per-k projector construction and density symmetrisation on the GPU.

* qeb_projector_basis against the reference's projector columns
  (tests/golden/setup_tables.npz, qepy_pw/upf.py:483-556) to 1e-13, and
  against the oracle's qe_cubic_interpolate + assemble_low_l_projectors
  (_native_fft.pyx:1556-1600, 1702-1791) for l = 0, 1, 2 on a seeded table.
* qeb_symmetrize_density against the host restatement of the reference's
  real-space symmetrizer (qepy_pw/symmetry.py:178-238), bit for bit, on the
  grids and space groups of the 2-atom fcc and 64-atom cells.
* qeb_random_trials (the first iteration's random wavefunctions from the
  stream's integer draws) against the reference's host formula
  amp e^(2 pi i phase) / (1 + 2 T) (qepy_pw/pw/scf.py:855-869) on the
  oracle's double pairs: the draws bit for bit, the complex exponential to
  a few ulps (CUDA's sincos against NumPy's exp).
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def test_projector_basis_matches_reference_columns(cuda_device, tmp_path):
    from qe_python_b200.pseudo import read_synthetic_upf, write_synthetic_upf
    from qe_python_b200.pseudo_tables import SpeciesTables, device_projectors

    tables = np.load(GOLDEN / "setup_tables.npz")
    pseudo = read_synthetic_upf(write_synthetic_upf(tmp_path / "X.upf"))
    species = SpeciesTables(pseudo, float(tables["volume"]))
    beta, coupling = device_projectors(species, tables["kg"])
    got = beta.cpu().numpy()
    np.testing.assert_allclose(got, tables["beta"], rtol=1e-13, atol=1e-15)
    np.testing.assert_array_equal(coupling, tables["coupling"])
    host, _ = species.projectors(tables["kg"])
    assert np.max(np.abs(got - host)) <= 1e-14 * np.max(np.abs(host))


def test_projector_basis_l2_matches_oracle(cuda_device):
    import torch

    from oracle import native_fft as oracle
    from qe_python_b200 import _lib
    from qe_python_b200.device import empty_f, leading_dimension, stream_handle

    rng = np.random.default_rng(17)
    npw = 3000
    kg = rng.normal(size=(npw, 3)) * 2.5
    kg[7] = 0.0  # the G = 0 row takes z = 1
    dq = 0.01
    q = np.sqrt(np.sum(kg * kg, axis=1))
    rows = int(q.max() / dq) + 8
    grid = np.arange(rows) * dq
    table = np.ascontiguousarray(np.stack([np.exp(-grid ** 2 / (2 + c)) * (1 + c * grid)
                                           for c in range(3)], axis=1))
    channels = [(0, 0, 0), (1, 1, 0), (1, 1, 1), (1, 1, 2)] + [(2, 2, m) for m in range(5)]
    radial_idx = np.array([c[0] for c in channels], dtype=np.int32)
    ls = np.array([c[1] for c in channels], dtype=np.int32)
    ms = np.array([c[2] for c in channels], dtype=np.int32)
    radial = oracle.qe_cubic_interpolate(table, q, dq)
    expected = oracle.assemble_low_l_projectors(radial, kg, q, radial_idx.astype(np.int64), ls, ms)
    device = cuda_device
    kg_cols = torch.from_numpy(np.ascontiguousarray(kg.T)).to(device)
    table_dev = torch.from_numpy(table).to(device)
    beta = empty_f(npw, len(channels), torch.complex128, device)
    lib = _lib.load()
    _lib.check("qeb_projector_basis", lib.qeb_projector_basis(
        npw, kg_cols.data_ptr(), table_dev.data_ptr(), rows, 3, dq, len(channels),
        radial_idx.ctypes.data, ls.ctypes.data, ms.ctypes.data, beta.data_ptr(),
        leading_dimension(beta), stream_handle()))
    got = beta.cpu().numpy()
    assert np.max(np.abs(got - expected)) <= 1e-14 * np.max(np.abs(expected))
    # an invalid channel is refused before any launch
    bad = np.array([3], dtype=np.int32)
    status = lib.qeb_projector_basis(npw, kg_cols.data_ptr(), table_dev.data_ptr(), rows, 3, dq,
                                     1, radial_idx.ctypes.data, bad.ctypes.data, ms.ctypes.data,
                                     beta.data_ptr(), leading_dimension(beta), stream_handle())
    assert status == -1


@pytest.mark.parametrize("name", ["scf-fcc2", "scf-dia64"])
def test_symmetrize_density_matches_host(cuda_device, name):
    import torch

    from qe_python_b200.basis import fft_shape, make_bases
    from qe_python_b200.scf import benchmark_system
    from qe_python_b200.symmetry import DensitySymmetrizer, fft_factors

    system = benchmark_system(name)
    bases = make_bases(system.reciprocal, system.kpoints, system.ecutwfc)
    shape = fft_shape(bases, system.reciprocal, system.ecutrho, fft_factors(system.operations))
    sym = DensitySymmetrizer(system.operations, shape)
    assert sym.count > 1
    rho = np.random.default_rng(3).random(shape)
    host = sym.apply(rho)
    got = sym.apply_device(torch.from_numpy(rho).to(cuda_device)).cpu().numpy()
    assert np.array_equal(got, host)


@pytest.mark.parametrize("dtype_name", ["complex128", "complex64"])
def test_random_trials_match_reference_formula(cuda_device, dtype_name):
    import torch

    from oracle import native_fft as oracle
    from qe_python_b200.diagonalization import PlaneWaveHamiltonian
    from qe_python_b200.scf import QERandom, benchmark_system, random_starting_subspace, scf_setup

    system = benchmark_system("scf-fcc2")
    setup = scf_setup(system, cuda_device)
    basis = setup.bases[0]
    npw, bands = len(basis), 8
    rng = QERandom()
    table, cur, seed = rng.table.copy(), rng.current, rng.seed
    amp, phase, _, _ = oracle.qe_random_pairs(npw, bands, table, cur, seed)
    want = amp * np.exp(2j * np.pi * phase) / (1.0 + 2.0 * basis.kinetic[:, None])
    first, second = rng.draws(npw, bands)
    np.testing.assert_array_equal(first / 714025.0, amp)
    np.testing.assert_array_equal(second / 714025.0, phase)

    captured = {}

    class Recording(PlaneWaveHamiltonian):
        def apply(self, x):
            captured["trials"] = x.clone()
            return super().apply(x)

    from qe_python_b200.basis import LocalPotentialWorkspace
    from qe_python_b200.scf import projector_terms

    precision = "f64" if dtype_name == "complex128" else "f32"
    ws = LocalPotentialWorkspace(basis, setup.shape, precision=precision, device=cuda_device)
    ham = Recording(basis, None, projector_terms(system, setup.tables, basis), local_workspace=ws,
                    real_potential=setup.v_ion, potential_average=setup.v_ion_average)
    random_starting_subspace(ham, basis, (first, second), bands)
    got = captured["trials"]
    assert got.dtype == getattr(torch, dtype_name)
    got = got.to(torch.complex128).cpu().numpy()
    bound = 1.0e-15 if dtype_name == "complex128" else 1.2e-7
    assert np.max(np.abs(got - want)) <= bound * np.max(np.abs(want))
