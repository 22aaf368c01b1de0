"""k-point pools: the SCF's k points distributed over the ranks of a process
group, one GPU per rank (qepy_pw/mpi.py pools; Quantum ESPRESSO's -npool).

Each rank runs the Davidson solves of its own k points.  The exchanges of
one SCF iteration are
  * the partial densities, summed in place (all-reduce of N_r FP64 values),
  * the eigenvalues of every k point, gathered so that every rank computes
    the same occupations, Fermi level and band energy,
  * per-atom force contributions at convergence, summed.
With torch.distributed's NCCL backend the density sum runs over NVLink; the
same code runs on gloo for the CPU tests.  Without a process group (or with
one rank) every method is the identity.
"""

from __future__ import annotations

import numpy as np
import torch


def pool_slices(nk: int, npool: int) -> list[range]:
    """Contiguous k ranges per pool, the first ``nk % npool`` pools one
    larger (the split of Quantum ESPRESSO's divide_et_impera)."""
    if npool < 1:
        raise ValueError("npool must be positive")
    base, extra = divmod(nk, npool)
    out, start = [], 0
    for p in range(npool):
        size = base + (1 if p < extra else 0)
        out.append(range(start, start + size))
        start += size
    return out


class KPointPools:
    """Rank ``rank`` of ``size`` owns ``pool_slices(nk, size)[rank]``."""

    def __init__(self, group=None) -> None:
        import torch.distributed as dist

        self.group = group
        self.distributed = dist.is_available() and dist.is_initialized()
        self.size = dist.get_world_size(group) if self.distributed else 1
        self.rank = dist.get_rank(group) if self.distributed else 0

    def local_kpoints(self, nk: int) -> range:
        if nk < self.size:
            raise ValueError(f"{nk} k points cannot feed {self.size} pools")
        return pool_slices(nk, self.size)[self.rank]

    def sum_(self, tensor: torch.Tensor) -> torch.Tensor:
        """In-place sum over the pools (the density, force partials)."""
        if self.size > 1:
            import torch.distributed as dist

            dist.all_reduce(tensor, op=dist.ReduceOp.SUM, group=self.group)
        return tensor

    def sum_array(self, values: np.ndarray, device=None) -> np.ndarray:
        t = torch.from_numpy(np.ascontiguousarray(values, dtype=np.float64))
        if device is not None:
            t = t.to(device)
        return self.sum_(t).cpu().numpy()

    def gather_eigenvalues(self, nk: int, local: dict[int, np.ndarray], nbnd: int,
                           device=None) -> list[np.ndarray]:
        """Eigenvalues of all nk k points on every rank: each rank fills its
        own rows of an (nk, nbnd) array of zeros, and the rows are summed."""
        table = np.zeros((nk, nbnd))
        for k, values in local.items():
            table[k] = values
        table = self.sum_array(table, device)
        return [table[k].copy() for k in range(nk)]
