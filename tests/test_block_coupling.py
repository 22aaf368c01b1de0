"""Host side of the block-diagonal projector coupling (kernels.BlockCoupling).

diagonal_blocks must return the smallest contiguous diagonal blocks that
cover every nonzero entry of the coupling D (0.5 D_Ry per atom,
qepy_pw/upf.py:541-551, assembled over the atoms as in
qepy_pw/diagonalization.py:348): consecutive, starting at 0, covering every
index, every nonzero inside one block, and no block splittable into two.
"""

from __future__ import annotations

import numpy as np

from qe_python_b200.kernels import diagonal_blocks


def _check(matrix):
    n = matrix.shape[0]
    blocks = diagonal_blocks(matrix)
    assert sum(size for _, size in blocks) == n
    start = 0
    owner = np.empty(n, dtype=int)
    for b, (s, size) in enumerate(blocks):
        assert s == start and size >= 1
        owner[s:s + size] = b
        start += size
    rows, cols = np.nonzero(matrix)
    assert np.array_equal(owner[rows], owner[cols])  # every nonzero inside a block
    for s, size in blocks:  # minimal: every cut inside a block splits a nonzero pair
        for cut in range(s + 1, s + size):
            crossing = ((rows < cut) & (cols >= cut)) | ((cols < cut) & (rows >= cut))
            assert crossing.any(), (s, size, cut)
    return blocks


def test_atom_blocks_of_a_projector_coupling():
    rng = np.random.default_rng(0)
    coupling = np.zeros((864, 864), dtype=np.complex128)
    for atom in range(216):
        block = rng.standard_normal((4, 4))
        coupling[4 * atom:4 * atom + 4, 4 * atom:4 * atom + 4] = block + block.T
    assert _check(coupling) == [(4 * a, 4) for a in range(216)]


def test_random_sparsity_patterns():
    rng = np.random.default_rng(1)
    for _ in range(300):
        n = int(rng.integers(1, 50))
        matrix = np.zeros((n, n))
        for _ in range(int(rng.integers(0, 10))):
            i, j = rng.integers(0, n, 2)
            matrix[i, j] = 1.0
        _check(matrix)
    assert diagonal_blocks(np.zeros((0, 0))) == []
    assert diagonal_blocks(np.zeros((3, 3))) == [(0, 1), (1, 1), (2, 1)]
