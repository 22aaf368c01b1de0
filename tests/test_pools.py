"""k-point pools on two gloo ranks (CPU): partition, density sum, eigenvalue
gather and the SCF bookkeeping built on them (band energy and occupations
equal on every rank and equal to the single-rank result)."""

from __future__ import annotations

import os

import numpy as np
import pytest
import torch

from qe_python_b200.occupations import smeared_occupations
from qe_python_b200.pools import KPointPools, pool_slices


def test_pool_slices_cover_every_k_once():
    for nk in range(1, 12):
        for npool in range(1, nk + 1):
            slices = pool_slices(nk, npool)
            flat = [k for s in slices for k in s]
            assert flat == list(range(nk))
            sizes = [len(s) for s in slices]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        pool_slices(3, 0)


def test_single_rank_pools_are_identity():
    pools = KPointPools()
    assert pools.size == 1 and pools.rank == 0
    assert list(pools.local_kpoints(5)) == [0, 1, 2, 3, 4]
    t = torch.arange(4, dtype=torch.float64)
    assert torch.equal(pools.sum_(t.clone()), t)


WORKER = r"""
import os, sys
import numpy as np
import torch
import torch.distributed as dist
from qe_python_b200.occupations import smeared_occupations
from qe_python_b200.pools import KPointPools
rank, size, port, path = int(sys.argv[1]), int(sys.argv[2]), sys.argv[3], sys.argv[4]
os.environ["MASTER_ADDR"] = "127.0.0.1"
os.environ["MASTER_PORT"] = port
dist.init_process_group("gloo", rank=rank, world_size=size)
try:
    pools = KPointPools()
    nk, nbnd, shape = 5, 6, (4, 4, 4)
    rng = np.random.default_rng(0)
    eig_all = [np.sort(rng.uniform(-0.5, 0.5, nbnd)) for _ in range(nk)]
    weights = rng.uniform(0.5, 1.0, nk)
    weights /= weights.sum()
    partial = [rng.random(shape) for _ in range(nk)]
    mine = list(pools.local_kpoints(nk))
    rho = torch.zeros(shape, dtype=torch.float64)
    for k in mine:
        rho += torch.from_numpy(partial[k])
    pools.sum_(rho)
    eig = pools.gather_eigenvalues(nk, {k: eig_all[k] for k in mine}, nbnd)
    ef, occ, demet = smeared_occupations(eig, weights, 7.0, 0.01, 0)
    band = sum(w * float(np.sum(e * f)) for w, e, f in zip(weights, eig, occ))
    np.savez(path, mine=np.array(mine), rho=rho.numpy(), eig=np.array(eig),
             scalars=np.array([ef, demet, band]))
finally:
    dist.destroy_process_group()
"""


def test_two_gloo_ranks_reproduce_single_rank_bookkeeping(tmp_path):
    import socket
    import subprocess
    import sys
    from pathlib import Path

    repo = Path(__file__).resolve().parents[1]
    with socket.socket() as sock:  # a free local port for the rendezvous
        sock.bind(("127.0.0.1", 0))
        port = str(sock.getsockname()[1])
    env = dict(os.environ, PYTHONPATH=str(repo))
    procs = [subprocess.Popen([sys.executable, "-c", WORKER, str(r), "2", port,
                               str(tmp_path / f"rank{r}.npz")], env=env, cwd=str(repo))
             for r in range(2)]
    for p in procs:
        assert p.wait(timeout=180) == 0
    r0, r1 = (np.load(tmp_path / f"rank{r}.npz") for r in range(2))
    mine0, mine1 = list(r0["mine"]), list(r1["mine"])
    assert sorted(mine0 + mine1) == [0, 1, 2, 3, 4] and not set(mine0) & set(mine1)
    # single-rank reference of the same quantities
    rng = np.random.default_rng(0)
    eig_all = [np.sort(rng.uniform(-0.5, 0.5, 6)) for _ in range(5)]
    weights = rng.uniform(0.5, 1.0, 5)
    weights /= weights.sum()
    rho_ref = sum(rng.random((4, 4, 4)) for _ in range(5))
    ef, occ, demet = smeared_occupations(eig_all, weights, 7.0, 0.01, 0)
    band = sum(w * float(np.sum(e * f)) for w, e, f in zip(weights, eig_all, occ))
    for r in (r0, r1):
        np.testing.assert_allclose(r["rho"], rho_ref, rtol=0, atol=1e-14)
        np.testing.assert_array_equal(r["eig"], np.array(eig_all))
        assert list(r["scalars"]) == [ef, demet, band]
