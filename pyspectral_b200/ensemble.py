"""Batched ensembles: many independent 2D runs, of uneven grid sizes, advanced together.

No counterpart in the reference (one pyspectral solver is one run).  Members are grouped into
size classes (same n and precision); each class is one batched engine (``sp_batch_*`` in
include/spectral_b200.h) whose every phase is one launch over all its members, and all classes
step from one CUDA graph (``sp_group_step``), one branch per class.  Each member has its own
viscosity, time step (CFL) and band-forcing rate (constant power), evaluated with batched
device reductions — one launch and one device-to-host copy per quantity for all members.

Every member computes exactly what a single :class:`~pyspectral_b200.solver.B200FusedSolver`
with the same configuration and the same dt / amplitude sequence computes (bit for bit).
"""

from __future__ import annotations

import ctypes
import json
import math
import os
import weakref
from collections.abc import Sequence
from pathlib import Path
from typing import Any

import numpy as np

from pyspectral_b200 import _lib
from pyspectral_b200.base import BackendUnavailable
from pyspectral_b200.config import Config
from pyspectral_b200.grid import spectral_shape


def nu_for_kmax_eta(n: int, power: float, k_force: float, kmax_eta: float = 1.0) -> float:
    """Viscosity giving ``kmax * eta = kmax_eta`` on an n^2 grid (kmax = n/3) for 2D turbulence
    forced at wavenumber ``k_force`` with power ``power``.

    2D dissipation scale of the enstrophy cascade (Kraichnan): eta = (nu^3 / beta)^(1/6) with
    beta the enstrophy injection (= dissipation) rate, estimated a priori as
    beta = k_force^2 * power.  Solving for nu: nu = beta^(1/3) (kmax_eta / kmax)^2.
    """
    beta = k_force * k_force * power
    return beta ** (1.0 / 3.0) * (kmax_eta / (n / 3.0)) ** 2


TILES = (1, 2, 4)


def tune_cache_path() -> Path:
    """JSON cache of tile choices (PYSPECTRAL_B200_TUNE_CACHE, else ~/.cache/pyspectral_b200)."""
    p = os.environ.get("PYSPECTRAL_B200_TUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "pyspectral_b200" / "tiles.json"


def load_tune_cache(path: Path) -> dict[str, Any]:
    try:
        data = json.loads(Path(path).read_text())
        return data if isinstance(data, dict) else {}
    except (OSError, ValueError):
        return {}


def save_tune_cache(path: Path, data: dict[str, Any]) -> None:
    path = Path(path)
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        tmp = path.with_suffix(".tmp")
        tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
        tmp.replace(path)
    except OSError:
        pass  # a read-only home only loses the cache


def tune_key(gpu: str, n: int, fp64: bool, members: int) -> str:
    return f"{gpu}|n={n}|{'fp64' if fp64 else 'fp32'}|members={members}"


class TileTuner:
    """Chooses each size class's tile (sub-blocks per CTA of the fused row and column passes,
    1, 2 or 4 times the default) by timing the class's batched step on the device (CUDA
    events, ``reps`` steps after two warm-up steps); choices are cached in a JSON file keyed by
    GPU model, grid, precision and member count.  Tiles change results at round-off only."""

    def __init__(self, path: Path | None = None, reps: int = 5) -> None:
        self.path = Path(path) if path is not None else tune_cache_path()
        self.reps = reps
        self.cache = load_tune_cache(self.path)
        self.report: dict[str, Any] = {}

    def choose(self, sc: _SizeClass, stream: Any) -> int:
        torch, lib = sc.torch, sc.lib
        gpu = torch.cuda.get_device_name(sc.u0.device)
        key = tune_key(gpu, sc.n, sc.fp64, sc.count)
        cands = [t for t in TILES if lib.sp_batch_tile_supported(sc.n, t)]
        hit = self.cache.get(key)
        if isinstance(hit, dict) and hit.get("tile") in cands:
            self.report[key] = dict(hit, cached=True)
            return int(hit["tile"])
        if len(cands) == 1:
            return cands[0]
        sc.set_step(np.full(sc.count, 1e-4), np.zeros(sc.count), stream)
        sc._check(lib.sp_batch_prepare(sc.h, stream), "sp_batch_prepare")
        times: dict[int, float] = {}
        cur = torch.cuda.current_stream(sc.u0.device)
        for t in cands:
            sc._check(lib.sp_batch_set_tile(sc.h, t), "sp_batch_set_tile")
            for _ in range(2):
                sc._check(lib.sp_batch_step(sc.h, stream), "sp_batch_step")
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(cur)
            for _ in range(self.reps):
                sc._check(lib.sp_batch_step(sc.h, stream), "sp_batch_step")
            e1.record(cur)
            e1.synchronize()
            times[t] = e0.elapsed_time(e1) / self.reps
        best = min(times, key=times.get)
        entry = {"tile": best, "ms_per_step": {str(k): v for k, v in times.items()}}
        self.cache[key] = entry
        self.report[key] = dict(entry, cached=False)
        save_tune_cache(self.path, self.cache)
        return best


    def choose_worklist(self, ens: Ensemble) -> int:
        """The group step's form: the work-list passes with CTAs of 64 or 128 threads, or one
        launch per class and phase (0) — whichever steps the group fastest (CUDA events,
        ``reps`` group steps after two warm-up steps); cached per GPU model and class set."""
        torch, lib = ens.torch, ens.lib
        gpu = torch.cuda.get_device_name(ens.device)
        sig = ",".join(f"{c.n}{'d' if c.fp64 else 'f'}x{c.count}" for c in ens.classes)
        key = f"{gpu}|group|{sig}"
        cands = [0] + [mt for mt in (64, 128) if ens._worklist_ok(mt)]
        hit = self.cache.get(key)
        if isinstance(hit, dict) and hit.get("worklist") in cands:
            self.report[key] = dict(hit, cached=True)
            return int(hit["worklist"])
        if len(cands) == 1:
            return 0
        st = ens._stream()
        for c in ens.classes:
            c.set_step(np.full(c.count, 1e-4), np.zeros(c.count), st)
            c._check(lib.sp_batch_prepare(c.h, st), "sp_batch_prepare")
        cur = torch.cuda.current_stream(ens.device)
        times: dict[int, float] = {}
        for mt in cands:
            ens.set_worklist(mt)
            for _ in range(2):
                ens._gcheck(lib.sp_group_step(ens._group, st), "sp_group_step")
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(cur)
            for _ in range(self.reps):
                ens._gcheck(lib.sp_group_step(ens._group, st), "sp_group_step")
            e1.record(cur)
            e1.synchronize()
            times[mt] = e0.elapsed_time(e1) / self.reps
        best = min(times, key=times.get)
        entry = {"worklist": best, "ms_per_step": {str(k): v for k, v in times.items()}}
        self.cache[key] = entry
        self.report[key] = dict(entry, cached=False)
        save_tune_cache(self.path, self.cache)
        return best


class _SizeClass:
    """One batched engine: the members of one (n, dtype) class."""

    def __init__(self, lib: Any, torch: Any, device: Any, cfgs: list[Config]) -> None:
        c0 = cfgs[0]
        for c in cfgs[1:]:
            if (c.alpha, c.alpha_kmax, c.force_klo, c.force_khi) != \
                    (c0.alpha, c0.alpha_kmax, c0.force_klo, c0.force_khi):
                raise ValueError("members of one size class share drag and forcing band")
        self.lib, self.torch, self.n, self.cfgs = lib, torch, c0.n, cfgs
        self.fp64 = c0.is_fp64
        self.count = len(cfgs)
        st = ctypes.c_int(0)
        h = lib.sp_batch_create(c0.n, int(self.fp64), self.count, ctypes.byref(st))
        if not h:
            msg = (lib.sp_create_error() or b"").decode()
            if st.value in (-1, -5):
                raise BackendUnavailable(f"ensemble n={c0.n}: {msg}")
            raise _lib.EngineError(f"sp_batch_create failed: {msg}")
        self.h = h
        self._fin = weakref.finalize(self, lib.sp_batch_destroy, ctypes.c_void_p(h))
        sizes = (ctypes.c_int64 * 6)()
        self._check(lib.sp_batch_query_sizes(h, sizes, 6), "sp_batch_query_sizes")
        cdt = torch.complex128 if self.fp64 else torch.complex64
        self.cdt = cdt
        self.u0 = torch.zeros((self.count,) + spectral_shape(c0.n, 2), dtype=cdt, device=device)
        assert self.u0.nbytes == sizes[2]
        self.work = torch.zeros(int(sizes[4]), dtype=torch.uint8, device=device)
        self.aux = torch.zeros(int(sizes[5]), dtype=torch.uint8, device=device)
        self._check(lib.sp_batch_bind(h, _lib.dptr(self.u0), _lib.dptr(self.work),
                                      _lib.dptr(self.aux)), "sp_batch_bind")
        nu = np.array([c.nu for c in cfgs], dtype=np.float64)
        self._check(lib.sp_batch_set_physics(h, nu.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                             float(c0.alpha), float(c0.drag_k2),
                                             float(c0.force_klo), float(c0.force_khi)),
                    "sp_batch_set_physics")

    def _check(self, status: int, what: str) -> None:
        if status != 0:
            msg = (self.lib.sp_batch_last_error(self.h) if getattr(self, "h", None)
                   else self.lib.sp_create_error()) or b""
            raise _lib.EngineError(f"{what} failed ({_lib.STATUS_NAMES.get(status)}): "
                                   f"{msg.decode()}")

    def set_tile(self, tile: int) -> None:
        self._check(self.lib.sp_batch_set_tile(self.h, int(tile)), "sp_batch_set_tile")

    @property
    def tile(self) -> int:
        return int(self.lib.sp_batch_tile(self.h))

    def set_step(self, dt: np.ndarray, amp: np.ndarray, stream: Any) -> None:
        dt = np.ascontiguousarray(dt, dtype=np.float64)
        amp = np.ascontiguousarray(amp, dtype=np.float64)
        dp = ctypes.POINTER(ctypes.c_double)
        self._check(self.lib.sp_batch_set_step(self.h, dt.ctypes.data_as(dp),
                                               amp.ctypes.data_as(dp), stream),
                    "sp_batch_set_step")


class Ensemble:
    """Independent 2D Basdevant runs (2/3 dealiasing, IF-RK4) advanced together on one GPU.

    ``members``: one :class:`Config` per run (dim 2; n a power of two, 16..8192 fp32 /
    16..4096 fp64).  Runs of the same n and dtype form a size class and must share drag and
    forcing band; viscosity, time step and forcing amplitude are per run.  ``autotune``: pick
    each class's tile and the group's work-list CTA size with :class:`TileTuner` (default on,
    see PYSPECTRAL_B200_AUTOTUNE).  ``worklist``: the group step as one persistent launch per
    phase over a packed work list of every class (``sp_group_set_worklist``: 64 or 128 threads
    per CTA; 0 = one launch per class and phase; None = the tuner's choice, else 64), where the
    classes allow it (one precision, n = 32..1024).
    """

    def __init__(self, members: Sequence[Config], autotune: bool | None = None,
                 worklist: int | None = None) -> None:
        import torch

        from pyspectral_b200.solver import _cuda_reason

        why = _cuda_reason()
        if why:
            raise BackendUnavailable(f"ensemble: {why}")
        for c in members:
            if c.dim != 2 or c.resolved_form() != "basdevant" or c.dealias != "2/3":
                raise BackendUnavailable("ensemble: 2D Basdevant form with 2/3 dealiasing only")
        self.torch = torch
        self.lib = lib = _lib.load()
        self.members = list(members)
        self.device = torch.device("cuda", torch.cuda.current_device())
        keys: dict[tuple[int, str], list[int]] = {}
        for i, c in enumerate(self.members):
            keys.setdefault((c.n, c.dtype), []).append(i)
        self.classes: list[_SizeClass] = []
        self.where: list[tuple[int, int]] = [(0, 0)] * len(self.members)
        for ci, ((_n, _dt), idx) in enumerate(sorted(keys.items())):
            self.classes.append(_SizeClass(lib, torch, self.device, [self.members[i] for i in idx]))
            for slot, i in enumerate(idx):
                self.where[i] = (ci, slot)
        self.index = [[i for i in range(len(self.members)) if self.where[i][0] == ci]
                      for ci in range(len(self.classes))]
        # tile choices: the autotuner (default; PYSPECTRAL_B200_AUTOTUNE=0 keeps tile 1), before
        # the group graph is captured
        if autotune is None:
            autotune = os.environ.get("PYSPECTRAL_B200_AUTOTUNE", "1") != "0"
        self.tuner: TileTuner | None = None
        if autotune:
            self.tuner = TileTuner()
            st = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
            for c in self.classes:
                c.set_tile(self.tuner.choose(c, st))
        arr = (ctypes.c_void_p * len(self.classes))(*[c.h for c in self.classes])
        st = ctypes.c_int(0)
        g = lib.sp_group_create(arr, len(self.classes), ctypes.byref(st))
        if not g:
            raise _lib.EngineError("sp_group_create failed")
        self._group = g
        self._gfin = weakref.finalize(self, lib.sp_group_destroy, ctypes.c_void_p(g))
        # the work list: a caller-owned device buffer, CTA size tuned or given
        nbytes = ctypes.c_int64(0)
        self._gcheck(lib.sp_group_worklist_bytes(g, ctypes.byref(nbytes)), "sp_group_worklist_bytes")
        self._wl = None
        if nbytes.value > 0:
            self._wl = torch.zeros(int(nbytes.value), dtype=torch.uint8, device=self.device)
            self._gcheck(lib.sp_group_bind(g, _lib.dptr(self._wl)), "sp_group_bind")
            if worklist is None:
                worklist = self.tuner.choose_worklist(self) if self.tuner is not None else 64
            if worklist and not self._worklist_ok(int(worklist)):
                worklist = 0
            self.set_worklist(int(worklist or 0))
        elif worklist:
            raise BackendUnavailable("ensemble: these size classes have no work-list path "
                                     "(one precision, n = 32..1024)")
        # pinned host staging of set_states / get_states, one buffer per class, and the event
        # after the last copy from it to the device
        self._pinned: dict[int, Any] = {}
        self._staged: dict[int, Any] = {}
        self.t = np.zeros(len(self.members))
        self.nstep = 0
        self.force_amp = np.array([c.force_amp for c in self.members], dtype=np.float64)
        self.dt = np.full(len(self.members), np.nan)

    # ------------------------------------------------------------------ plumbing
    def __len__(self) -> int:
        return len(self.members)

    def _gcheck(self, status: int, what: str) -> None:
        if status != 0:
            msg = (self.lib.sp_group_last_error(self._group) or b"").decode()
            raise _lib.EngineError(f"{what} failed ({_lib.STATUS_NAMES.get(status)}): {msg}")

    def _worklist_ok(self, mt: int) -> bool:
        fp = {c.fp64 for c in self.classes}
        return len(fp) == 1 and all(32 <= c.n <= 1024 and c.n // 16 <= mt and 16 * mt // c.n <= c.n
                                    for c in self.classes)

    def set_worklist(self, mt: int) -> None:
        """Step the group through the work-list passes with CTAs of mt threads (64 or 128), or
        through one launch per class and phase (mt = 0)."""
        self._gcheck(self.lib.sp_group_set_worklist(self._group, int(mt)), "sp_group_set_worklist")

    @property
    def worklist(self) -> int:
        """CTA threads of the work-list passes in use; 0 when each class launches its own."""
        return int(self.lib.sp_group_worklist(self._group))

    def _stream(self) -> ctypes.c_void_p:
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def _per_class(self, values: np.ndarray, ci: int) -> np.ndarray:
        return np.asarray(values, dtype=np.float64)[self.index[ci]]

    def _upload(self, dt: np.ndarray) -> None:
        for ci, c in enumerate(self.classes):
            c.set_step(self._per_class(dt, ci), self._per_class(self.force_amp, ci),
                       self._stream())

    # ------------------------------------------------------------------ state
    def set_states(self, states: Sequence[np.ndarray]) -> None:
        """Load every member's spectral state (host arrays, NumPy r2c layout).  Each size class
        goes through one pinned host buffer of its state's size, kept for the ensemble's
        lifetime and shared with get_states."""
        if len(states) != len(self.members):
            raise ValueError("one state per member")
        for i, a in enumerate(states):
            c = self.classes[self.where[i][0]]
            if np.shape(a) != spectral_shape(c.n, 2):
                raise ValueError(f"member {i}: state shape {np.shape(a)} != "
                                 f"{spectral_shape(c.n, 2)}")
        # per class: cast into the pinned staging buffer (torch's threaded copy), one copy to
        # the device
        torch = self.torch
        for ci, c in enumerate(self.classes):
            stage = self._staging(ci)
            for slot, i in enumerate(self.index[ci]):
                stage[slot].copy_(torch.from_numpy(np.ascontiguousarray(states[i])))
            c.u0.copy_(stage, non_blocking=True)
            self._staged[ci].record(torch.cuda.current_stream(self.device))
        self._upload(np.where(np.isnan(self.dt), 0.0, self.dt))
        for c in self.classes:
            c._check(self.lib.sp_batch_prepare(c.h, self._stream()), "sp_batch_prepare")
        self.t[:] = 0.0

    def state_native(self, i: int) -> Any:
        """Member i's live state (device tensor, NumPy layout)."""
        ci, slot = self.where[i]
        c = self.classes[ci]
        c._check(self.lib.sp_batch_sync_state(c.h, self._stream()), "sp_batch_sync_state")
        return c.u0[slot]

    def get_state(self, i: int) -> np.ndarray:
        return self.state_native(i).detach().cpu().numpy().astype(np.complex128)

    def _staging(self, ci: int) -> Any:
        """Class ci's pinned host buffer (its state's shape and dtype; allocated on first use,
        reused), once the last copy from it to the device has finished."""
        torch = self.torch
        if ci not in self._pinned:
            c = self.classes[ci]
            self._pinned[ci] = torch.empty(c.u0.shape, dtype=c.u0.dtype, pin_memory=True)
            self._staged[ci] = torch.cuda.Event()
            self._staged[ci].record(torch.cuda.current_stream(self.device))
        self._staged[ci].synchronize()
        return self._pinned[ci]

    def get_states(self) -> list[np.ndarray]:
        """Every member's state (host arrays, NumPy r2c layout, complex128): one state refresh
        and one device-to-host copy per size class, where get_state refreshes the member's
        whole class on every call."""
        from pyspectral_b200.solver import B200Solver

        torch = self.torch
        stream = torch.cuda.current_stream(self.device)
        out: list[Any] = [None] * len(self.members)
        for ci, c in enumerate(self.classes):
            c._check(self.lib.sp_batch_sync_state(c.h, self._stream()), "sp_batch_sync_state")
            # through a pinned buffer in chunks: the widening cast of a chunk (torch's threaded
            # copy) overlaps the PCIe copy of the next
            stage = self._staging(ci)
            src, sflat = c.u0.detach().reshape(-1), stage.view(-1)
            chunks = B200Solver._chunks(sflat.numel())
            landed = []
            for lo, hi in chunks:
                sflat[lo:hi].copy_(src[lo:hi], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(stream)
                landed.append(ev)
            res = torch.empty(c.u0.shape, dtype=torch.complex128)
            rflat = res.view(-1)
            for (lo, hi), ev in zip(chunks, landed):
                ev.synchronize()
                rflat[lo:hi].copy_(sflat[lo:hi])
            host = res.numpy()
            for slot, i in enumerate(self.index[ci]):
                out[i] = host[slot]
        return out

    # ------------------------------------------------------------------ stepping
    def set_forcing_amplitudes(self, amps: Any) -> None:
        self.force_amp = np.broadcast_to(np.asarray(amps, dtype=np.float64),
                                         (len(self.members),)).copy()

    def step(self, dt: Any) -> None:
        """One IF-RK4 step of every member; ``dt`` scalar or one value per member."""
        dt = np.broadcast_to(np.asarray(dt, dtype=np.float64), (len(self.members),)).copy()
        self._upload(dt)
        self.dt = dt
        status = self.lib.sp_group_step(self._group, self._stream())
        if status != 0:
            raise _lib.EngineError("sp_group_step failed: "
                                   + (self.lib.sp_group_last_error(self._group) or b"").decode())
        self.t += dt
        self.nstep += 1

    # ------------------------------------------------------------------ diagnostics
    def diagnostics(self, band_klo: float = 0.0, band_khi: float = -1.0) -> np.ndarray:
        """(members, 4): energy, enstrophy, palinstrophy, energy in band_klo <= |k| <= band_khi."""
        out = np.zeros((len(self.members), 4))
        for ci, c in enumerate(self.classes):
            buf = np.zeros((c.count, 4))
            c._check(self.lib.sp_batch_diagnostics(
                c.h, float(band_klo), float(band_khi),
                buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), self._stream()),
                "sp_batch_diagnostics")
            out[self.index[ci]] = buf
        return out

    def max_velocity_sum(self) -> np.ndarray:
        """(members,): max|u| + max|v| of each member (the CFL bound)."""
        out = np.zeros(len(self.members))
        for ci, c in enumerate(self.classes):
            buf = np.zeros(c.count)
            c._check(self.lib.sp_batch_max_velocity(
                c.h, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), self._stream()),
                "sp_batch_max_velocity")
            out[self.index[ci]] = buf
        return out

    def cfl_dt(self, cfl: float, dt_max: float) -> np.ndarray:
        """Per-member ``cfl * dx / sum_i max|u_i|`` capped at dt_max (simulate.cfl_dt rule)."""
        umax = self.max_velocity_sum()
        dx = np.array([2.0 * math.pi / c.n for c in self.members])
        ok = np.isfinite(umax) & (umax > 0)
        return np.where(ok, np.minimum(dt_max, cfl * dx / np.where(ok, umax, 1.0)), dt_max)

    def run_steps(self, nsteps: int, *, cfl: float = 0.5, dt_max: float = 0.05,
                  cfl_every: int = 10, target_power: float | None = None) -> np.ndarray:
        """``nsteps`` steps with per-member CFL dt (every ``cfl_every`` steps) and, with
        ``target_power``, constant-power forcing A = P / (2 E_band) per member (the rules of
        simulate.run).  Returns the (nsteps, members) dt history."""
        hist = np.zeros((nsteps, len(self.members)))
        dt = np.full(len(self.members), dt_max)
        klo = np.array([c.force_klo for c in self.members])
        khi = np.array([c.force_khi for c in self.members])
        for k in range(nsteps):
            if k % cfl_every == 0:
                dt = self.cfl_dt(cfl, dt_max)
                if target_power is not None:
                    eb = self._band_energy(klo, khi)
                    self.force_amp = np.where(eb > 0, target_power / (2.0 * np.where(eb > 0, eb, 1.0)), 0.0)
            self.step(dt)
            hist[k] = dt
        return hist

    def _band_energy(self, klo: np.ndarray, khi: np.ndarray) -> np.ndarray:
        out = np.zeros(len(self.members))
        for ci, c in enumerate(self.classes):
            lo, hi = self._per_class(klo, ci), self._per_class(khi, ci)
            # one forcing band per class (checked at construction)
            buf = np.zeros((c.count, 4))
            c._check(self.lib.sp_batch_diagnostics(
                c.h, float(lo[0]), float(hi[0]),
                buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), self._stream()),
                "sp_batch_diagnostics")
            out[self.index[ci]] = buf[:, 3]
        return out

    @property
    def tiles(self) -> list[int]:
        """Tile of each size class (sorted by n, dtype)."""
        return [c.tile for c in self.classes]

    @property
    def kernel_launches(self) -> int:
        return int(sum(self.lib.sp_batch_kernel_launches(c.h) for c in self.classes)
                   + self.lib.sp_group_kernel_launches(self._group))
