"""k-points over ranks for the SCF of crystals (the reference's comm_bzsm layout).

The reference splits the k-points of an SCF into contiguous blocks, one per k group of
processes (id_bzsm / ir_bzsm of init_parallel, src/parallel_module.f90: the first nk mod np
groups take one extra point), runs the band update of its own block, and exchanges only what
the SCF loop needs across the blocks: the eigenvalues for the Fermi level (esp_gather), the
density, summed over k (calc_density's allreduce), and the band-energy sums of the total
energy.  The band update itself needs no collective.  KpointGroup does the same over a
torch.distributed process group (NCCL on GPUs, gloo on CPUs), one rank per block; without an
initialised group it is a single rank that owns every k-point.
"""
from __future__ import annotations

import numpy as np


def k_blocks(nk: int, nprocs: int) -> list:
    """(first, count) per rank: contiguous blocks, the first nk mod nprocs ranks one larger."""
    base, extra = divmod(nk, nprocs)
    out, k0 = [], 0
    for r in range(nprocs):
        c = base + (1 if r < extra else 0)
        out.append((k0, c))
        k0 += c
    return out


class KpointGroup:
    """local=True (or no initialised process group): one rank owning every k-point."""

    def __init__(self, nk: int, group=None, local: bool = False):
        import torch.distributed as dist
        self._dist = dist if (not local and dist.is_available() and dist.is_initialized()) else None
        self.group = group
        self.rank = self._dist.get_rank(group) if self._dist else 0
        self.size = self._dist.get_world_size(group) if self._dist else 1
        if nk < self.size:
            raise ValueError(f"{nk} k-points cannot give every one of {self.size} ranks a block")
        self.nk = nk
        self.blocks = k_blocks(nk, self.size)
        k0, c = self.blocks[self.rank]
        self.klist = list(range(k0, k0 + c))

    def _device(self):
        backend = self._dist.get_backend(self.group) if self._dist else "gloo"
        return "cuda" if backend == "nccl" else "cpu"

    def gather_esp(self, esp_local: np.ndarray) -> np.ndarray:
        """(ns, nk_local, nb) of this rank -> (ns, nk, nb) in global k order on every rank."""
        if self._dist is None:
            return np.asarray(esp_local, np.float64)
        import torch
        ns, _, nb = esp_local.shape
        cmax = max(c for _, c in self.blocks)
        pad = np.zeros((ns, cmax, nb))
        pad[:, :esp_local.shape[1]] = esp_local
        t = torch.from_numpy(pad).to(self._device())
        parts = [torch.empty_like(t) for _ in range(self.size)]
        self._dist.all_gather(parts, t, group=self.group)
        return np.concatenate([p.cpu().numpy()[:, :c] for p, (_, c) in zip(parts, self.blocks)], axis=1)

    def sum(self, x):
        """Sum of an array (or float) over the ranks, returned on every rank."""
        if self._dist is None:
            return x
        import torch
        a = np.asarray(x, np.float64)
        t = torch.from_numpy(np.ascontiguousarray(a).copy()).to(self._device())
        self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM, group=self.group)
        r = t.cpu().numpy()
        return float(r) if np.ndim(x) == 0 else r
