"""Lockstep Davidson rounds replayed from CUDA graphs (RoundGraphs).

The chosen-form H applications of one lockstep round of the 64-atom cell's
four k points (one launch per FFT pass for all of them, then each k point's
split-TF32 projector GEMMs) are captured on first use and replayed later.
Checks: the replay equals the eager round on the same padded blocks bit for
bit; the rounds' outputs for the requested columns equal the eager rounds
on the unpadded blocks to FP32 round-off (a 5-column block is padded to 16,
wider ones to multiples of 32); after a new potential is set the replay
follows it; a round of a single k point replays the same batched launches.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_round_graphs_match_eager_rounds(cuda_device):
    import torch

    from qe_python_b200.device import to_device_f
    from qe_python_b200.diagonalization import RoundGraphs, apply_hamiltonians
    from qe_python_b200.scf import benchmark_system, starting_hamiltonians

    hams, _v, _setup = starting_hamiltonians(benchmark_system("scf-dia64"), "f32")
    graphs = RoundGraphs(hams, max_width=96)
    rng = np.random.default_rng(4)
    widths = [37, 5, 90, 64]

    def block(k, n):
        a = rng.standard_normal((len(hams[k].basis), n)) + 1j * rng.standard_normal(
            (len(hams[k].basis), n))
        return to_device_f(a, torch.complex64, cuda_device)

    def outputs_like(vectors):
        return [torch.empty_like(v.T).T for v in vectors]

    for trial in range(3):
        vectors = [block(k, n) for k, n in enumerate(widths)]
        got = outputs_like(vectors)
        graphs([(k, v, g) for k, (v, g) in enumerate(zip(vectors, got))])
        # eager round on the same padded static blocks the graph read
        key = tuple(sorted((k, graphs.width(n)) for k, n in enumerate(widths)))
        padded = [graphs.inputs[k][:, :w].clone() for k, w in key]
        eager_padded = outputs_like(padded)
        apply_hamiltonians(hams, [(k, p, e) for (k, _w), p, e in zip(key, padded, eager_padded)],
                           potential=graphs.potential)
        for (k, n), e in zip(enumerate(widths), eager_padded):
            assert torch.equal(got[k], e[:, :n]), (trial, k)
        # eager round on the unpadded blocks
        eager = outputs_like(vectors)
        apply_hamiltonians(hams, [(k, v, e) for k, (v, e) in enumerate(zip(vectors, eager))])
        for g, e in zip(got, eager):
            scale = float(e.abs().max())
            assert float((g - e).abs().max()) <= 2e-6 * scale
    assert graphs.captures == 1 and graphs.replays == 2

    # a new local potential: the replay follows it
    new_v = hams[0]._potential * 0.5
    graphs.set_potential(new_v)
    vectors = [block(k, n) for k, n in enumerate(widths)]
    got = outputs_like(vectors)
    graphs([(k, v, g) for k, (v, g) in enumerate(zip(vectors, got))])
    eager = outputs_like(vectors)
    apply_hamiltonians(hams, [(k, v, e) for k, (v, e) in enumerate(zip(vectors, eager))],
                       potential=new_v)
    for g, e in zip(got, eager):
        assert float((g - e).abs().max()) <= 2e-6 * float(e.abs().max())
    assert graphs.replays == 3

    # a round in which one k point alone is still solving: the same batched
    # launches, captured with their own key, twice (capture, then replay)
    for _ in range(2):
        vector = block(2, 20)
        got = torch.empty_like(vector.T).T
        graphs([(2, vector, got)])
        eager = torch.empty_like(vector.T).T
        apply_hamiltonians(hams, [(2, vector, eager)], potential=new_v, always_batched=True)
        assert float((got - eager).abs().max()) <= 2e-6 * float(eager.abs().max())
    assert graphs.captures == 2 and graphs.replays == 4
