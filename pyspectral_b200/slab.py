"""Slab-decomposed 3D runs: one run spread over several GPUs (``sp_slab_*`` in csrc/slab3d.cu).

No reference counterpart (the reference runs on one device).  Each rank holds a ky slab of the
spectral state (n, n/P, n/2+1 per component) and an x slab of the physical fields; an RK stage
is three local parts with an all-to-all of equal, contiguous blocks after parts 0 and 1.

* :class:`SlabSolver` — one rank's share, the exchange through ``torch.distributed``
  (``all_to_all_single``, NCCL over NVLink / NVSwitch; a device copy for one rank).
* :class:`LocalSlabGroup` — all P ranks of a decomposition in one process on one device, the
  exchange done by device copies between the ranks' buffers (everything on one stream, no
  kernel waits for another): runs the distributed algorithm, and checks it, on a single GPU.
"""

from __future__ import annotations

import ctypes
import math
import weakref
from typing import Any

import numpy as np

from pyspectral_b200 import _lib
from pyspectral_b200.base import BackendUnavailable
from pyspectral_b200.config import Config
from pyspectral_b200.solver import _cuda_reason

_NSIZE = 8  # sp_slab_query_sizes entries


def exchange_blocks(recv: Any, send: Any, block_bytes: int, nranks: int, comm: Any) -> None:
    """All-to-all of ``nranks`` equal contiguous blocks: block p of this rank's ``send`` lands
    in block (this rank) of rank p's ``recv`` (``comm``: torch.distributed, NCCL on GPUs).
    Without ``comm`` a single rank's exchange is a device copy; with ``comm`` the collective runs
    for any number of ranks, one included."""
    nb = nranks * block_bytes
    if comm is None:
        if nranks != 1:
            raise ValueError("an exchange between several ranks needs a process group")
        if recv.data_ptr() != send.data_ptr():
            recv[:nb].copy_(send[:nb])
        return
    comm.all_to_all_single(recv[:nb], send[:nb])


class SlabSolver:
    """Rank ``rank`` of a 3D run decomposed over ``nranks`` ranks (n divisible by nranks).

    ``set_state`` takes the whole spectral state (3, n, n, n/2+1) and keeps this rank's slab;
    ``get_state`` returns the slab (3, n, n/nranks, n/2+1)."""

    def __init__(self, cfg: Config, rank: int = 0, nranks: int = 1, comm: Any = None) -> None:
        why = _cuda_reason()
        if why:
            raise BackendUnavailable(f"slab: {why}")
        if cfg.dim != 3:
            raise BackendUnavailable("slab decomposition: 3D runs only")
        import torch

        self.torch, self.cfg = torch, cfg
        self.lib = lib = _lib.load()
        self.comm = comm
        self.rank, self.nranks = int(rank), int(nranks)
        self.n = n = cfg.n
        form = cfg.resolved_form("basdevant")
        st = ctypes.c_int(0)
        h = lib.sp_slab_create(n, self.nranks, self.rank, _lib.FORM_CODES[form],
                               int(cfg.is_fp64), ctypes.byref(st))
        if not h:
            raise _lib.EngineError(f"sp_slab_create failed: {(lib.sp_create_error() or b'').decode()}")
        self._h = h
        self._fin = weakref.finalize(self, lib.sp_slab_destroy, ctypes.c_void_p(h))
        sz = (ctypes.c_int64 * _NSIZE)()
        self._check(lib.sp_slab_query_sizes(h, sz, _NSIZE), "sp_slab_query_sizes")
        self.m = int(sz[6])
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.cdt = torch.complex128 if cfg.is_fp64 else torch.complex64
        shape = (3, n, self.m, n // 2 + 1)
        self.u0 = torch.zeros(shape, dtype=self.cdt, device=self.device)
        self.acc = torch.zeros_like(self.u0)
        u8 = dict(dtype=torch.uint8, device=self.device)
        self.W = torch.zeros(int(sz[2]), **u8)
        self.send = torch.zeros(int(sz[3]), **u8)
        # one rank without a process group: the all-to-all is the identity, so receive where
        # the blocks were packed; through a process group the collective needs its own buffer
        self.recv = (self.send if self.nranks == 1 and comm is None
                     else torch.zeros(int(sz[3]), **u8))
        self.aux = torch.zeros(int(sz[4]), **u8)
        self.ws = torch.empty(max(1, int(sz[5])), **u8)
        self._check(lib.sp_slab_bind(h, _lib.dptr(self.u0), _lib.dptr(self.acc), _lib.dptr(self.W),
                                     _lib.dptr(self.send), _lib.dptr(self.recv),
                                     _lib.dptr(self.aux), _lib.dptr(self.ws)), "sp_slab_bind")
        self._check(lib.sp_slab_set_physics(h, float(cfg.nu), float(cfg.alpha),
                                            float(cfg.drag_k2), float(cfg.force_klo),
                                            float(cfg.force_khi)), "sp_slab_set_physics")
        self.force_amp = float(cfg.force_amp)
        self._check(lib.sp_slab_set_forcing_amplitude(h, self.force_amp), "set_forcing_amplitude")
        self.t = 0.0
        self.nstep = 0

    # ------------------------------------------------------------------ plumbing
    def _check(self, status: int, what: str) -> None:
        if status != 0:
            msg = (self.lib.sp_slab_last_error(self._h) or b"").decode()
            raise _lib.EngineError(f"{what} failed: {_lib.STATUS_NAMES.get(status, status)}: {msg}")

    def _stream(self) -> ctypes.c_void_p:
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def block_bytes(self, part: int) -> int:
        """Bytes of one exchange block (one per destination rank) after ``part`` (0 or 1)."""
        return int(self.lib.sp_slab_exchange_block_bytes(self._h, int(part)))

    def part(self, part: int, stage: int) -> None:
        self._check(self.lib.sp_slab_stage_part(self._h, int(part), int(stage), self._stream()),
                    "sp_slab_stage_part")

    def exchange(self, part: int) -> None:
        """This rank's all-to-all after ``part`` (every rank calls it in the same order)."""
        exchange_blocks(self.recv, self.send, self.block_bytes(part), self.nranks, self.comm)

    @property
    def kernel_launches(self) -> int:
        return int(self.lib.sp_slab_kernel_launches(self._h))

    # ------------------------------------------------------------------ state
    def ky_slice(self) -> slice:
        return slice(self.rank * self.m, (self.rank + 1) * self.m)

    def set_state(self, state: Any) -> None:
        """Whole spectral state (3, n, n, n/2+1), host or device; this rank keeps its slab."""
        a = state[:, :, self.ky_slice(), :]
        if isinstance(a, np.ndarray):
            a = self.torch.from_numpy(np.ascontiguousarray(a))
        self.u0.copy_(a.to(self.cdt))
        self._check(self.lib.sp_slab_prepare(self._h, self._stream()), "sp_slab_prepare")

    def get_state(self) -> np.ndarray:
        return self.u0.detach().cpu().numpy().astype(np.complex128)

    def set_forcing_amplitude(self, amp: float) -> None:
        self.force_amp = float(amp)
        self._check(self.lib.sp_slab_set_forcing_amplitude(self._h, self.force_amp),
                    "sp_slab_set_forcing_amplitude")

    def set_dt(self, dt: float) -> None:
        self._check(self.lib.sp_slab_set_dt(self._h, float(dt), self._stream()), "sp_slab_set_dt")

    # ------------------------------------------------------------------ stepping
    def step(self, dt: float) -> None:
        self.set_dt(dt)
        for stage in range(4):
            self.part(0, stage)
            self.exchange(0)
            self.part(1, stage)
            self.exchange(1)
            self.part(2, stage)
        self.t += dt
        self.nstep += 1

    # ------------------------------------------------------------------ diagnostics
    def local_energy(self) -> float:
        out = ctypes.c_double(0.0)
        self._check(self.lib.sp_slab_energy(self._h, _lib.dptr(self.u0), ctypes.byref(out),
                                            self._stream()), "sp_slab_energy")
        return float(out.value)

    def local_max_velocity(self) -> list[float]:
        """max |u_i| of the velocity the last stage 0 transformed (this rank's x slab)."""
        out = (ctypes.c_double * 3)()
        self._check(self.lib.sp_slab_max_velocity(self._h, out, self._stream()),
                    "sp_slab_max_velocity")
        return [float(v) for v in out]


class LocalSlabGroup:
    """Every rank of an ``nranks`` decomposition in this process on the current device."""

    def __init__(self, cfg: Config, nranks: int) -> None:
        self.cfg, self.n, self.nranks = cfg, cfg.n, nranks
        self.ranks = [SlabSolver(cfg, r, nranks) for r in range(nranks)]
        self.t = 0.0

    def set_state(self, state: Any) -> None:
        for s in self.ranks:
            s.set_state(state)

    def _exchange(self, part: int) -> None:
        nb = self.ranks[0].block_bytes(part)
        for src in self.ranks:
            for dst in self.ranks:
                # block `dst` of the sender lands in block `src` of the receiver
                dst.recv[src.rank * nb:(src.rank + 1) * nb].copy_(
                    src.send[dst.rank * nb:(dst.rank + 1) * nb])

    def step(self, dt: float) -> None:
        for s in self.ranks:
            s.set_dt(dt)
        for stage in range(4):
            for s in self.ranks:
                s.part(0, stage)
            self._exchange(0)
            for s in self.ranks:
                s.part(1, stage)
            self._exchange(1)
            for s in self.ranks:
                s.part(2, stage)
        for s in self.ranks:
            s.t += dt
            s.nstep += 1
        self.t += dt

    def set_forcing_amplitude(self, amp: float) -> None:
        for s in self.ranks:
            s.set_forcing_amplitude(amp)

    def get_state(self) -> np.ndarray:
        return np.concatenate([s.get_state() for s in self.ranks], axis=2)

    def energy(self) -> float:
        return math.fsum(s.local_energy() for s in self.ranks)

    def max_velocity_sum(self) -> float:
        per = np.max([s.local_max_velocity() for s in self.ranks], axis=0)
        return float(per.sum())
