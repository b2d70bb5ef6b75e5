"""Multi-GPU plumbing of the paths that shard: ensembles partitioned across ranks, and
data-parallel training of the closure network.  One process per GPU, ``torch.distributed``
(NCCL on GPUs, gloo in CPU tests); no collective in any kernel.

* :func:`partition_by_points` / :class:`ShardedEnsemble` — independent runs spread over ranks
  with balanced grid points (largest first onto the least-loaded rank); each rank advances its
  share with one batched :class:`~pyspectral_b200.ensemble.Ensemble`; per-member results are
  gathered on the host in the global member order only when asked for.
* :func:`train_data_parallel` — every rank draws its own tiles (seed offset by rank), the batch
  gradients are averaged with one all-reduce of 15440 floats per optimiser step, and every rank
  applies the same Adam update, so the parameters stay identical across ranks.
"""

from __future__ import annotations

from collections.abc import Callable, Sequence
from typing import Any

import numpy as np

from pyspectral_b200.config import Config


def partition_by_points(sizes: Sequence[int], world: int) -> list[list[int]]:
    """Member indices per rank: members sorted by n^2 (largest first, then index) go one by
    one to the rank with the fewest points so far (lowest rank on ties).  Deterministic."""
    if world < 1:
        raise ValueError("world must be positive")
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]) ** 2, i)):
        r = min(range(world), key=lambda r: (load[r], r))
        parts[r].append(i)
        load[r] += int(sizes[i]) ** 2
    return [sorted(p) for p in parts]


class Comm:
    """Rank, world and the few collectives the sharded paths use (process group already
    initialised by the caller, or a single process)."""

    def __init__(self, device: Any = None) -> None:
        import torch.distributed as dist

        self.dist = dist if dist.is_available() and dist.is_initialized() else None
        self.rank = self.dist.get_rank() if self.dist else 0
        self.world = self.dist.get_world_size() if self.dist else 1
        self.device = device  # where collective buffers live (a CUDA device for NCCL)

    def all_gather_rows(self, local: np.ndarray, counts: Sequence[int]) -> list[np.ndarray]:
        """Every rank's (counts[r], k) float64 rows; each rank passes its own.  Without a
        process group the rows are returned as they are; with one (of any size, one rank
        included) they go through the group's ``all_gather``."""
        if self.dist is None:
            return [np.asarray(local, dtype=np.float64)]
        import torch

        k = int(local.shape[1]) if local.ndim == 2 else 1
        mx = max(counts)
        buf = np.zeros((mx, k), np.float64)
        buf[: len(local)] = np.asarray(local, np.float64).reshape(len(local), k)
        t = torch.from_numpy(buf).to(self.device or "cpu")
        out = [torch.empty_like(t) for _ in range(self.world)]
        self.dist.all_gather(out, t)
        return [o.cpu().numpy()[: counts[r]] for r, o in enumerate(out)]

    def allreduce_mean_(self, t: Any) -> Any:
        """In-place mean of a tensor over the ranks (the group's ``all_reduce`` whenever a
        process group exists, one rank included)."""
        if self.dist is not None:
            self.dist.all_reduce(t)
            if self.world > 1:
                t /= self.world
        return t


class ShardedEnsemble:
    """An ensemble whose members are spread over the ranks by :func:`partition_by_points`.

    ``factory(configs)`` builds the local batched ensemble (default
    :class:`~pyspectral_b200.ensemble.Ensemble`).  Stepping is local and needs no collective;
    :meth:`diagnostics` and :meth:`max_velocity_sum` gather every member's values in the
    global order on every rank (all ranks must call them together)."""

    def __init__(self, members: Sequence[Config], comm: Comm | None = None,
                 factory: Callable[[list[Config]], Any] | None = None) -> None:
        self.members = list(members)
        self.comm = comm or Comm()
        self.parts = partition_by_points([c.n for c in self.members], self.comm.world)
        self.local = self.parts[self.comm.rank]
        if factory is None:
            from pyspectral_b200.ensemble import Ensemble

            factory = Ensemble
        self.ens = factory([self.members[i] for i in self.local]) if self.local else None

    @property
    def local_points(self) -> int:
        return sum(self.members[i].n ** 2 for i in self.local)

    def set_states(self, states: Sequence[np.ndarray]) -> None:
        """All members' states (every rank passes the full list; each keeps its own)."""
        if self.ens is not None:
            self.ens.set_states([states[i] for i in self.local])

    def _local(self, values: Any) -> np.ndarray:
        v = np.broadcast_to(np.asarray(values, np.float64), (len(self.members),))
        return v[self.local]

    def step(self, dt: Any) -> None:
        if self.ens is not None:
            self.ens.step(self._local(dt))

    def run_steps(self, nsteps: int, **kw: Any) -> None:
        if self.ens is not None:
            self.ens.run_steps(nsteps, **kw)

    def _gather(self, local: np.ndarray, k: int) -> np.ndarray:
        counts = [len(p) for p in self.parts]
        rows = self.comm.all_gather_rows(local.reshape(len(self.local), k), counts)
        out = np.zeros((len(self.members), k))
        for r, part in enumerate(self.parts):
            out[part] = rows[r]
        return out

    def diagnostics(self, band_klo: float = 0.0, band_khi: float = -1.0) -> np.ndarray:
        loc = self.ens.diagnostics(band_klo, band_khi) if self.ens is not None else np.zeros((0, 4))
        return self._gather(np.asarray(loc, np.float64), 4)

    def max_velocity_sum(self) -> np.ndarray:
        loc = self.ens.max_velocity_sum() if self.ens is not None else np.zeros(0)
        return self._gather(np.asarray(loc, np.float64), 1)[:, 0]


class _CudaArray:
    """A CUDA array interface over a raw device pointer (torch.as_tensor aliases it)."""

    def __init__(self, ptr: int, n: int) -> None:
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False),
                                         "version": 2, "strides": None}


def train_data_parallel(net: Any, steps: int, batch_tiles: int, seed: int,
                        comm: Comm | None = None) -> np.ndarray:
    """``steps`` optimiser steps of ``net`` (a ClosureNet) with the batch gradients averaged over
    the ranks; every rank samples its own tiles (seed + 7919 * rank).  Returns this rank's local
    mean losses.  With one rank this is exactly ClosureNet.train."""
    import torch

    comm = comm or Comm(net.device)
    lib = net.lib
    ptr = lib.sp_closure_grad_buffer(net.handle)
    grad = torch.as_tensor(_CudaArray(int(ptr), 15440), device=net.device)
    first = net.step_count
    st = net._stream()
    rank_seed = int(seed) + 7919 * comm.rank
    for _ in range(steps):
        net._check(lib.sp_closure_train_begin(net.handle, int(batch_tiles), rank_seed, st),
                   "sp_closure_train_begin")
        comm.allreduce_mean_(grad)
        net._check(lib.sp_closure_train_finish(net.handle, st), "sp_closure_train_finish")
    net.check()
    return net.losses(first, steps)

