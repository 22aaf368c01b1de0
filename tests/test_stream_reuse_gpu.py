"""Streams reused across Hamiltonians and Davidson solves (diagonalization.STREAMS).

The caching allocator keeps one pool of blocks per stream: a stream created
for each Hamiltonian or each overlapped reduced solve started its
allocations from an empty pool, so every SCF run made new device
allocations (each of which waited for the GPU work queued before it).  With
the side stream shared per device and the solver streams pooled, a second
run of the same SCF (lockstep k points with overlapped solves, the mixed
form) reuses the first run's blocks: it makes no device allocation.
"""

from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


def test_second_scf_run_allocates_no_device_memory(cuda_device):
    import torch

    from qe_python_b200.diagonalization import STREAMS
    from qe_python_b200.scf import benchmark_system, run_scf

    first = run_scf(benchmark_system("scf-fcc2"), precision="mixed")
    torch.cuda.synchronize()
    before = torch.cuda.memory_stats()["num_device_alloc"]
    second = run_scf(benchmark_system("scf-fcc2"), precision="mixed")
    torch.cuda.synchronize()
    assert torch.cuda.memory_stats()["num_device_alloc"] == before
    assert second.converged and first.converged
    assert abs(second.total_energy_ry - first.total_energy_ry) < 1.0e-10
    side = STREAMS.shared(torch.device("cuda"))
    assert side is STREAMS.shared(torch.device("cuda"))
