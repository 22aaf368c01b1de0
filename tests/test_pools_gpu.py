"""run_scf(pools=...) with two ranks sharing one GPU (gloo process group).

Each rank solves its own k points of the 2-atom fcc cell (10 irreducible
points, five per rank) on the GPU; the partial densities are summed and the
eigenvalues gathered through the process group, as the k-point pools of
qepy_pw (QE's -npool) combine them.  Both ranks must reproduce the
single-rank SCF: total energy within 1e-10 Ry, eigenvalues within 1e-9 Ry,
the same iteration count, and the analytic stress (its kinetic and nonlocal
k sums combined over the pools) within 1e-12 Ha/bohr^3.  The collectives are gloo's (host memory), so the
two processes' kernels never wait on one another.
"""

from __future__ import annotations

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WORKER = r"""
import json, os, sys
from datetime import timedelta
import numpy as np
import torch
import torch.distributed as dist
from qe_python_b200.pools import KPointPools
from qe_python_b200.scf import benchmark_system, run_scf
rank, size, port, path = int(sys.argv[1]), int(sys.argv[2]), sys.argv[3], sys.argv[4]
os.environ["MASTER_ADDR"] = "127.0.0.1"
os.environ["MASTER_PORT"] = port
dist.init_process_group("gloo", rank=rank, world_size=size, timeout=timedelta(seconds=120))
try:
    torch.cuda.set_device(0)
    system = benchmark_system("scf-fcc2")
    system.stress = True
    result = run_scf(system, precision="f64", pools=KPointPools())
    Path = __import__("pathlib").Path
    Path(path).write_text(json.dumps({
        "energy_ry": result.total_energy_ry, "iterations": result.iterations,
        "converged": bool(result.converged),
        "stress": np.asarray(result.stress_ha_per_bohr3).tolist(),
        "eigenvalues_ry": [(2.0 * np.asarray(e)).tolist() for e in result.eigenvalues_ha]}))
finally:
    dist.destroy_process_group()
"""


def test_two_pools_on_one_gpu_reproduce_single_rank_scf(cuda_device, tmp_path):
    from qe_python_b200.scf import benchmark_system, run_scf

    system = benchmark_system("scf-fcc2")
    system.stress = True
    single = run_scf(system, precision="f64")
    assert single.converged
    repo = Path(__file__).resolve().parents[1]
    with socket.socket() as sock:  # a free local port for the rendezvous
        sock.bind(("127.0.0.1", 0))
        port = str(sock.getsockname()[1])
    env = dict(os.environ, PYTHONPATH=str(repo))
    procs = [subprocess.Popen([sys.executable, "-c", WORKER, str(r), "2", port,
                               str(tmp_path / f"rank{r}.json")], env=env, cwd=str(repo))
             for r in range(2)]
    try:
        for p in procs:
            assert p.wait(timeout=300) == 0
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    for r in range(2):
        got = json.loads((tmp_path / f"rank{r}.json").read_text())
        assert got["converged"]
        assert got["iterations"] == single.iterations
        assert abs(got["energy_ry"] - single.total_energy_ry) <= 1e-10
        for mine, ref in zip(got["eigenvalues_ry"], single.eigenvalues_ha):
            assert np.max(np.abs(np.asarray(mine) - 2.0 * np.asarray(ref))) <= 1e-9
        assert np.max(np.abs(np.asarray(got["stress"]) - single.stress_ha_per_bohr3)) <= 1e-12
