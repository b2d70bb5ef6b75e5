"""Learned subgrid closure for coarse 2D runs: network, snapshot bank, training, coarse solver.

No reference counterpart (the reference has no closure or ML code).  The pieces:

* :class:`ClosureNet` — a device-resident network 75 -> 64 -> 64 -> 64 -> 1 (GELU) with its
  Adam state and a bank of filtered-DNS snapshots (``sp_closure_*``).  Layers 1-3 run as BF16
  tcgen05 GEMMs with FP32 accumulation in tensor memory, forward and backward, in one
  persistent kernel per optimiser step.
* :func:`filter_spectrum` — pad_spectrum (src/pyspectral/validation.py:24-35) on the device,
  with the coarse grid's 2/3 mask: the sharp spectral filter that defines the coarse field.
* :func:`nonlinear_term` — ``NumpySolver.nonlinear`` (backends/numpy_ref.py:75-96) of a
  spectral state on the device.
* :class:`SnapshotPipeline` — fine DNS state -> bank entry (filtered vorticity, its gradient,
  and the subgrid term S = F[N(omega)] - N_c(F[omega])).
* :class:`ClosureSolver` — the coarse ``SpectralSolver`` variant whose every RK stage adds the
  network's S to the nonlinear term; inference is fused with the stage's physical-space
  products.
"""

from __future__ import annotations

import ctypes
import math
import weakref
from pathlib import Path
from typing import Any, ClassVar

import numpy as np

from pyspectral_b200 import _lib
from pyspectral_b200.base import BackendUnavailable
from pyspectral_b200.config import Config
from pyspectral_b200.solver import B200Solver, _cuda_reason

K, H, IN, TILE = 80, 64, 75, 128
WSZ = H * K
NPARAM = 3 * WSZ + K  # 15440
BIAS_IN, BIAS_H = 75, 64


def init_params(seed: int = 0, out_std: float = 0.1) -> np.ndarray:
    """LeCun-normal hidden weights, zero biases and padding, a small output layer."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, np.float32)
    for layer, fan in enumerate((IN, H, H)):
        W = np.zeros((H, K), np.float32)
        W[:, :fan] = rng.normal(0.0, 1.0 / math.sqrt(fan), (H, fan))
        p[layer * WSZ: (layer + 1) * WSZ] = W.ravel()
    p[3 * WSZ: 3 * WSZ + H] = rng.normal(0.0, out_std / math.sqrt(H), H)
    return p


def _fptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


class ClosureNet:
    """Network parameters, Adam state and snapshot bank on the current CUDA device.

    ``n``: coarse grid (power of two, 128..4096); ``capacity``: bank entries (4 n^2 floats each).
    """

    def __init__(self, n: int = 256, capacity: int = 64) -> None:
        why = _cuda_reason()
        if why:
            raise BackendUnavailable(f"closure: {why}")
        import torch

        self.torch = torch
        self.lib = lib = _lib.load()
        status = ctypes.c_int(0)
        h = lib.sp_closure_create(int(n), int(capacity), ctypes.byref(status))
        if not h:
            raise _lib.EngineError(f"sp_closure_create failed: {(lib.sp_create_error() or b'').decode()}")
        self._h = h
        self._fin = weakref.finalize(self, lib.sp_closure_destroy, ctypes.c_void_p(h))
        self.n = int(n)
        self.capacity = int(capacity)
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.inscale = np.ones(3, np.float32)
        self.outscale = 1.0
        self.clip = False
        self.nshell = int(lib.sp_closure_shell_count(h))
        self.shell_gain = np.ones(self.nshell, np.float32)
        self.every_stage = True

    # ------------------------------------------------------------------ plumbing
    @property
    def handle(self) -> int:
        return self._h

    def _check(self, status: int, what: str) -> None:
        if status != 0:
            msg = (self.lib.sp_closure_last_error(self._h) or b"").decode()
            raise _lib.EngineError(f"{what} failed: {_lib.STATUS_NAMES.get(status, status)}: {msg}")

    def _stream(self) -> ctypes.c_void_p:
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    @property
    def kernel_launches(self) -> int:
        return int(self.lib.sp_closure_kernel_launches(self._h))

    # ------------------------------------------------------------------ parameters
    def set_params(self, params: np.ndarray) -> None:
        """Load fp32 parameters; resets the optimiser state and the step counter."""
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.shape != (NPARAM,):
            raise ValueError(f"expected {NPARAM} parameters, got {p.shape}")
        self._check(self.lib.sp_closure_set_params(self._h, _fptr(p)), "sp_closure_set_params")

    def params(self) -> np.ndarray:
        out = np.zeros(NPARAM, np.float32)
        self._check(self.lib.sp_closure_get_params(self._h, _fptr(out)), "sp_closure_get_params")
        return out

    def grad(self) -> np.ndarray:
        out = np.zeros(NPARAM, np.float32)
        self._check(self.lib.sp_closure_get_grad(self._h, _fptr(out)), "sp_closure_get_grad")
        return out

    def set_scales(self, inscale: Any, outscale: float, clip: bool = False) -> None:
        """Inputs are fields * inscale; the network's output times outscale is S."""
        a = np.ascontiguousarray(inscale, dtype=np.float32).reshape(3)
        self._check(self.lib.sp_closure_set_scales(self._h, _fptr(a), float(outscale), int(clip)),
                    "sp_closure_set_scales")
        self.inscale, self.outscale, self.clip = a.copy(), float(outscale), bool(clip)

    def set_shell_gain(self, gain: Any) -> None:
        """Per-shell gains g(k) applied to the closure term in an attached solver's step."""
        g = np.ascontiguousarray(gain, dtype=np.float32)
        if g.shape != (self.nshell,):
            raise ValueError(f"expected {self.nshell} shell gains, got {g.shape}")
        self._check(self.lib.sp_closure_set_shell_gain(self._h, _fptr(g), self.nshell),
                    "sp_closure_set_shell_gain")
        self.shell_gain = g.copy()

    def set_update(self, every_stage: bool) -> None:
        """Network evaluated at every RK stage, or at the first stage of each step only."""
        self._check(self.lib.sp_closure_set_update(self._h, int(bool(every_stage))),
                    "sp_closure_set_update")
        self.every_stage = bool(every_stage)

    def fit_scales(self, max_entries: int = 64, clip: bool = False) -> None:
        """Unit-variance inputs and target from the standard deviations over (part of) the bank."""
        count = self.bank_count
        if count < 1:
            raise RuntimeError("snapshot bank is empty")
        idx = np.unique(np.linspace(0, count - 1, min(count, max_entries)).round().astype(int))
        sq = np.zeros(4)
        for i in idx:
            e = self.bank_entry(int(i)).astype(np.float64)
            sq += (e.reshape(4, -1) ** 2).mean(axis=1)
        std = np.sqrt(sq / len(idx))
        std = np.where(std > 0, std, 1.0)
        self.set_scales(1.0 / std[:3], float(std[3]), clip)

    def set_adam(self, lr: float = 1e-3, lr_min: float = 1e-5, beta1: float = 0.9,
                 beta2: float = 0.999, eps: float = 1e-8, total_steps: int = 20000,
                 warmup: int = 200) -> None:
        self._check(self.lib.sp_closure_set_adam(self._h, lr, lr_min, beta1, beta2, eps,
                                                 int(total_steps), int(warmup)),
                    "sp_closure_set_adam")

    # ------------------------------------------------------------------ bank
    @property
    def bank_count(self) -> int:
        return int(self.lib.sp_closure_bank_count(self._h))

    def load_bank(self, entries: np.ndarray) -> None:
        """Replace the bank by host entries (count, 4, n, n): omega, omega_x, omega_y, S."""
        a = np.ascontiguousarray(entries, dtype=np.float32)
        if a.ndim != 4 or a.shape[1:] != (4, self.n, self.n):
            raise ValueError(f"bank entries must be (count, 4, {self.n}, {self.n})")
        self._check(self.lib.sp_closure_bank_load(self._h, _fptr(a), a.shape[0]),
                    "sp_closure_bank_load")

    def bank_entry(self, i: int) -> np.ndarray:
        out = np.zeros((4, self.n, self.n), np.float32)
        self._check(self.lib.sp_closure_bank_read(self._h, int(i), _fptr(out)),
                    "sp_closure_bank_read")
        return out

    def reset_bank(self) -> None:
        self._check(self.lib.sp_closure_bank_reset(self._h), "sp_closure_bank_reset")

    def add_snapshot(self, wbar: Any, fine_nl: Any, coarse_nl: Any) -> None:
        """Append a bank entry from coarse device spectra (complex64, (n, n/2+1))."""
        shape = (self.n, self.n // 2 + 1)
        for a in (wbar, fine_nl, coarse_nl):
            if tuple(a.shape) != shape or a.dtype != self.torch.complex64 or not a.is_cuda:
                raise ValueError(f"snapshot spectra must be complex64 CUDA tensors of shape {shape}")
        self._check(self.lib.sp_closure_add_snapshot(self._h, _lib.dptr(wbar), _lib.dptr(fine_nl),
                                                     _lib.dptr(coarse_nl), self._stream()),
                    "sp_closure_add_snapshot")

    # ------------------------------------------------------------------ training
    def grad_at(self, step: int, batch_tiles: int = 512, seed: int = 0) -> tuple[np.ndarray, float]:
        """Gradient and mean loss of training step ``step`` without updating (for checks)."""
        self._check(self.lib.sp_closure_grad(self._h, int(step), int(batch_tiles), int(seed),
                                             self._stream()), "sp_closure_grad")
        return self.grad(), float(self.losses(step, 1)[0])

    def train(self, steps: int, batch_tiles: int = 512, seed: int = 0) -> np.ndarray:
        """``steps`` Adam steps of ``batch_tiles`` x 128 points; returns their mean losses."""
        first = self.step_count
        self._check(self.lib.sp_closure_train(self._h, int(steps), int(batch_tiles), int(seed),
                                              self._stream()), "sp_closure_train")
        return self.losses(first, steps)

    @property
    def step_count(self) -> int:
        return int(self.lib.sp_closure_step_count(self._h))

    def losses(self, first: int, count: int) -> np.ndarray:
        count = min(int(count), 1 << 16)
        out = np.zeros(count, np.float32)
        self._check(self.lib.sp_closure_losses(self._h, int(first), count, _fptr(out)),
                    "sp_closure_losses")
        return out

    # ------------------------------------------------------------------ inference
    def infer(self, fields: Any, out: Any | None = None, sync: bool = True) -> Any:
        """S at every point from device fields (3, n, n) float32: omega, omega_x, omega_y.
        ``sync=False`` only enqueues the launch (``check()`` reports a timed-out wait later)."""
        torch = self.torch
        f = fields.contiguous()
        if tuple(f.shape) != (3, self.n, self.n) or f.dtype != torch.float32 or not f.is_cuda:
            raise ValueError(f"fields must be a float32 CUDA tensor (3, {self.n}, {self.n})")
        if out is None:
            out = torch.empty((self.n, self.n), dtype=torch.float32, device=f.device)
        fn = self.lib.sp_closure_infer if sync else self.lib.sp_closure_infer_async
        self._check(fn(self._h, _lib.dptr(f), self.n * self.n, self.n, _lib.dptr(out), self.n,
                       self._stream()), "sp_closure_infer")
        return out

    def check(self) -> None:
        """Raise if a closure kernel launched inside a solver step reported a timed-out wait."""
        self._check(self.lib.sp_closure_check(self._h, self._stream()), "closure step")

    # ------------------------------------------------------------------ files
    def save(self, path: str | Path) -> None:
        np.savez(path, params=self.params(), inscale=self.inscale, outscale=self.outscale,
                 clip=self.clip, n=self.n, shell_gain=self.shell_gain)

    def load(self, path: str | Path) -> None:
        z = np.load(path)
        if int(z["n"]) != self.n:
            raise ValueError(f"closure file is for n={int(z['n'])}, this network has n={self.n}")
        self.set_params(z["params"])
        self.set_scales(z["inscale"], float(z["outscale"]), bool(z["clip"]))
        if "shell_gain" in z.files:
            self.set_shell_gain(z["shell_gain"])


# ---------------------------------------------------------------------- spectral helpers
def filter_spectrum(src: Any, n_to: int, dim: int = 2, dealias: bool = True) -> Any:
    """pad_spectrum to grid ``n_to`` (and its 2/3 mask) of a device spectrum, on the device."""
    import torch

    lib = _lib.load()
    n = int(src.shape[-2])
    if src.dtype not in (torch.complex64, torch.complex128) or not src.is_cuda:
        raise ValueError("filter_spectrum takes a complex CUDA tensor")
    fp64 = src.dtype == torch.complex128
    shape = (n_to,) * (dim - 1) + (n_to // 2 + 1,)
    out = torch.empty(shape, dtype=src.dtype, device=src.device)
    st = ctypes.c_void_p(torch.cuda.current_stream(src.device).cuda_stream)
    status = lib.sp_filter_spectrum(_lib.dptr(src.contiguous()), n, _lib.dptr(out), int(n_to),
                                    int(dim), int(fp64), int(dealias), st)
    _lib.check(lib, None, status, "sp_filter_spectrum")
    return out


def nonlinear_term(solver: B200Solver, state: Any, out: Any | None = None) -> Any:
    """Dealiased 2D nonlinear term of a device spectral state through ``solver``'s plans."""
    torch = solver.torch
    if out is None:
        out = torch.empty_like(solver.u0)
    solver._check(solver.lib.sp_nonlinear(solver.handle, _lib.dptr(state.contiguous()),
                                          _lib.dptr(out), solver._stream()), "sp_nonlinear")
    return out


class SnapshotPipeline:
    """Fine DNS states -> bank entries of ``net`` (filter to the coarse grid, fine and coarse
    nonlinear terms, physical fields).  ``n_fine``: the DNS grid."""

    def __init__(self, net: ClosureNet, n_fine: int) -> None:
        self.net = net
        self.fine = B200Solver(Config(n=n_fine, dim=2, dtype="float32"))
        self.coarse = B200Solver(Config(n=net.n, dim=2, dtype="float32"))
        self.fine_nl = net.torch.empty_like(self.fine.u0)
        self.cnl = net.torch.empty_like(self.coarse.u0)

    def coarse_state(self, state: Any) -> Any:
        """Sharp-filtered coarse spectrum of a fine state."""
        return filter_spectrum(state.to(self.net.torch.complex64), self.net.n)

    def add(self, state: Any) -> None:
        s = state.to(self.net.torch.complex64).contiguous()
        nonlinear_term(self.fine, s, self.fine_nl)
        wbar = filter_spectrum(s, self.net.n)
        fnl = filter_spectrum(self.fine_nl, self.net.n)
        nonlinear_term(self.coarse, wbar, self.cnl)
        self.net.add_snapshot(wbar, fnl, self.cnl)


# ---------------------------------------------------------------------- coarse solver
class ClosureSolver(B200Solver):
    """Coarse 2D fp32 solver whose RK stages add the network's subgrid term to the nonlinear
    term: stage = batch-5 inverse FFT (u, v, omega, omega_x, omega_y) -> products + network
    (one persistent tcgen05 kernel) -> batch-3 forward FFT (S, products) -> Lawson update.
    ``every_stage=False`` evaluates the network at the first stage of each step only and holds
    its term for the other three stages, which run the plain two-field transforms."""

    variant = "closure-les-graph"
    dims: ClassVar[tuple[int, ...]] = (2,)

    def __init__(self, cfg: Config, net: ClosureNet, every_stage: bool = True) -> None:
        if cfg.dim != 2 or cfg.is_fp64:
            raise BackendUnavailable("closure: 2D fp32 runs only")
        if cfg.n != net.n:
            raise ValueError(f"closure network is for n={net.n}, run has n={cfg.n}")
        self.net = net
        self.every_stage = bool(every_stage)
        self._mode: bool | None = None  # update mode the step graph was captured with
        super().__init__(cfg)

    def run_to(self, t_end: float, **kw: Any) -> int:
        self._sync_mode()
        n = super().run_to(t_end, **kw)
        self.net.check()
        return n

    def _sync_mode(self) -> None:
        if self._mode != self.every_stage or self.net.every_stage != self.every_stage:
            # the closure object is shared: set its mode and re-capture this solver's graph
            self.net.set_update(self.every_stage)
            self._check(self.lib.sp_set_graph(self._h, 0), "sp_set_graph")
            self._check(self.lib.sp_set_graph(self._h, int(self.use_graph)), "sp_set_graph")
            self._mode = self.every_stage

    def _step(self, dt: float) -> None:
        self._sync_mode()
        super()._step(dt)

    def _before_bind(self, h: int) -> None:
        _lib.check(self.lib, h, self.lib.sp_attach_closure(h, ctypes.c_void_p(self.net.handle)),
                   "sp_attach_closure")

    def synchronize(self) -> None:
        super().synchronize()
        self.net.check()
