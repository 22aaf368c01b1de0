"""CUDA-graph capture of the whole H|psi> (chosen form, FP32/split-TF32 and
FP64): a replay must reproduce the direct application bit for bit."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_graph_replay_equals_direct_apply(cuda_device, precision):
    import torch

    from qe_python_b200.basis import LocalPotentialWorkspace, make_bases
    from qe_python_b200.device import to_device_f
    from qe_python_b200.diagonalization import HpsiGraph, PlaneWaveHamiltonian
    from qe_python_b200.workloads import hpsi_microbench

    work = hpsi_microbench(nbands=32)
    basis = make_bases(work.reciprocal, np.zeros(3), 30.0)[0]
    ws = LocalPotentialWorkspace(basis, work.shape, precision=precision)
    ham = PlaneWaveHamiltonian(basis, None, ((work.beta, work.coupling),), local_workspace=ws,
                               real_potential=torch.from_numpy(work.potential).cuda(),
                               potential_average=0.0)
    psi = to_device_f(work.psi, ham.dtype, ham.device)
    direct = ham.apply(psi)
    graph = HpsiGraph(ham, psi.shape[1])
    replayed = graph(psi)
    torch.cuda.synchronize()
    assert torch.equal(direct, replayed)
    # a second replay with other data
    psi2 = (psi * 0.5).T.contiguous().T
    assert torch.equal(ham.apply(psi2), graph(psi2))


def test_host_streamed_hpsi_equals_direct_apply(cuda_device):
    """Chunked host -> device -> host H|psi> with overlapped copies equals the
    direct application, including a partial last chunk (to FP32 round-off:
    a chunk may take another K split of the projector GEMMs)."""
    import torch

    from qe_python_b200.basis import LocalPotentialWorkspace, make_bases
    from qe_python_b200.device import to_device_f
    from qe_python_b200.diagonalization import HostStreamedHpsi, PlaneWaveHamiltonian
    from qe_python_b200.workloads import hpsi_microbench

    work = hpsi_microbench(nbands=40)
    basis = make_bases(work.reciprocal, np.zeros(3), 30.0)[0]
    ws = LocalPotentialWorkspace(basis, work.shape, precision="f32")
    ham = PlaneWaveHamiltonian(basis, None, ((work.beta, work.coupling),), local_workspace=ws,
                               real_potential=torch.from_numpy(work.potential).cuda(),
                               potential_average=0.0)
    npw = len(basis)
    # graphs replay concurrently on two compute streams, each with its own
    # scratch: every chunk must still match the direct application
    # (uneven chunks: sizes of their own, one buffer each, an odd size among them)
    for kwargs in (dict(chunk=16, buffers=2), dict(chunk=8, buffers=4),
                   dict(chunks=(5, 15, 15, 5)), dict(chunks=(8, 24, 8), compute_streams=1)):
        streamed = HostStreamedHpsi(ham, 40, **kwargs)
        host_in, host_out = streamed.host_buffers()
        host_in[:, :npw] = torch.from_numpy(work.psi.T.astype(np.complex64))
        starts = np.cumsum([0] + streamed.sizes[:-1]).tolist()
        for _ in range(2):
            host_out.zero_()
            streamed(host_in, host_out)
            torch.cuda.synchronize()
            for start, size in zip(starts, streamed.sizes):
                stop = start + size
                block = to_device_f(work.psi[:, start:stop], torch.complex64)
                expected = ham.apply(block).cpu().T
                got = host_out[start:stop, :npw]
                scale = float(expected.abs().max())
                assert float((got - expected).abs().max()) <= 1e-5 * scale
        # the same pipeline captured as one CUDA graph (every chunk's kernels
        # on the compute streams) reproduces the eager pipeline's result
        eager = host_out.clone()
        streamed.capture(host_in, host_out)
        scale = float(eager[:, :npw].abs().max())
        for _ in range(2):
            host_out.zero_()
            streamed.replay()
            torch.cuda.synchronize()
            assert float((host_out[:, :npw] - eager[:, :npw]).abs().max()) <= 1e-6 * scale
    with pytest.raises(ValueError):
        HostStreamedHpsi(ham, 40, chunks=(10, 20, 20))  # sizes must sum to the band count
