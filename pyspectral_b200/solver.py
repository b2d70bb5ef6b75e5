"""B200 solver: the drop-in ``SpectralSolver`` over libspectral_b200.so.

Counterpart of the reference's CUDA C backend (``CupyCudaSolver``,
src/pyspectral/backends/cupy_cuda.py:32-213) with the same public behaviour: construction
raises ``BackendUnavailable`` for options it does not run (2D non-Basdevant form, phase-shift
dealiasing, no GPU, library not built); ``set_state`` checks the shape, dealiases (on the device)
and rebuilds the stage-0 FFT inputs; ``state_native`` is the live device state in NumPy r2c layout; a forcing-amplitude
or dt change is honoured on the next step.

Device memory is owned here as torch CUDA tensors (state, RK accumulator, FFT work fields,
parameter/scratch block, cuFFT work area) and handed to the engine as raw pointers; every call
runs on torch's current CUDA stream.
"""

from __future__ import annotations

import ctypes
import weakref
from typing import Any, ClassVar

import numpy as np

from pyspectral_b200 import _lib
from pyspectral_b200.base import BackendUnavailable, SpectralSolver
from pyspectral_b200.config import Config, fft_split
from pyspectral_b200.ops import TorchOps


def _cuda_reason() -> str:
    """Empty string when a CUDA device and the built library are present, else why not."""
    if not _lib.LIB_PATH.exists():
        return f"{_lib.LIB_PATH.name} is not built (run `python -m pyspectral_b200.build`)"
    try:
        import torch
    except Exception as e:  # noqa: BLE001
        return f"torch not importable: {e}"
    if not torch.cuda.is_available():
        return "no CUDA device"
    return ""


class B200Solver(SpectralSolver):
    """Fused sm_100a pointwise kernels + in-place batched cuFFT, one CUDA graph per step."""

    backend = "b200"
    variant = "fused-inplace-graph"
    default_form = "basdevant"
    forms = ("basdevant", "rotational")
    fft_mode: ClassVar[int] = _lib.FFT_CUFFT
    use_graph: ClassVar[bool] = True

    def __init__(self, cfg: Config) -> None:
        super().__init__(cfg)
        if self.dim == 2 and self.form != "basdevant":
            raise BackendUnavailable(f"{self.backend}: 2D supports the basdevant form only")
        why = _cuda_reason()
        if why:
            raise BackendUnavailable(f"{self.backend}/{self.variant}: {why}")
        import torch

        self.torch = torch
        self.lib = lib = _lib.load()
        fp64 = cfg.is_fp64
        status = ctypes.c_int(0)
        h = lib.sp_create(self.n, self.dim, _lib.FORM_CODES[self.form], int(fp64),
                          self.fft_mode, ctypes.byref(status))
        if not h:
            msg = (lib.sp_create_error() or b"").decode()
            if status.value in (-1, -5):
                raise BackendUnavailable(f"{self.backend}/{self.variant}: {msg}")
            raise _lib.EngineError(f"sp_create failed ({_lib.STATUS_NAMES.get(status.value)}): {msg}")
        self._h = h
        self._finalizer = weakref.finalize(self, lib.sp_destroy, ctypes.c_void_p(h))
        self._before_bind(h)
        sizes = (ctypes.c_int64 * _lib.SZ_COUNT)()
        self._check(lib.sp_query_sizes(h, sizes, _lib.SZ_COUNT), "sp_query_sizes")
        self.sizes = list(sizes)
        self.rdt = torch.float64 if fp64 else torch.float32
        self.cdt = torch.complex128 if fp64 else torch.complex64
        self.n_inv, self.n_fwd = fft_split(self.dim, self.form)
        self.nw = int(sizes[_lib.SZ_NWORK])
        dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.u0 = torch.zeros(self.state_shape(), dtype=self.cdt, device=dev)
        self.acc = torch.zeros_like(self.u0)
        self.W = torch.zeros(int(sizes[_lib.SZ_WORK_BYTES]), dtype=torch.uint8, device=dev)
        self.aux = torch.zeros(int(sizes[_lib.SZ_AUX_BYTES]), dtype=torch.uint8, device=dev)
        self.fftws = torch.empty(max(1, int(sizes[_lib.SZ_FFTWS_BYTES])), dtype=torch.uint8,
                                 device=dev)
        assert self.u0.nbytes == sizes[_lib.SZ_STATE_BYTES]
        self._check(lib.sp_bind(h, _lib.dptr(self.u0), _lib.dptr(self.acc), _lib.dptr(self.W),
                                _lib.dptr(self.aux), _lib.dptr(self.fftws)), "sp_bind")
        self._check(lib.sp_set_physics(h, float(cfg.nu), float(cfg.alpha), float(cfg.drag_k2),
                                       float(cfg.force_klo), float(cfg.force_khi)),
                    "sp_set_physics")
        self._check(lib.sp_set_forcing_amplitude(h, float(self.force_amp)),
                    "sp_set_forcing_amplitude")
        self._check(lib.sp_set_graph(h, int(self.use_graph)), "sp_set_graph")
        self._ops = TorchOps(str(dev))

    # ------------------------------------------------------------------ plumbing
    @classmethod
    def available(cls) -> tuple[bool, str]:
        why = _cuda_reason()
        return (not why), why

    def _check(self, status: int, what: str) -> None:
        _lib.check(self.lib, self._h, status, what)

    def _before_bind(self, h: int) -> None:
        """Hook between sp_create and sp_query_sizes / sp_bind (layout-changing attachments)."""

    def _stream(self) -> ctypes.c_void_p:
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    @property
    def handle(self) -> int:
        return self._h

    @property
    def ops(self) -> Any:
        return self._ops

    # ------------------------------------------------------------------ state
    def set_state(self, state_hat: Any) -> None:
        """Load a spectral state (host array, or a device tensor of the state's shape).

        Same contract as check_state + set_state of the reference (shape ValueError, 2/3 mask),
        with the mask applied on the device by the engine's load kernel: the host only casts
        into a pinned staging buffer (torch's threaded copy) and the copy to the device is
        asynchronous, chunk by chunk, so a chunk crosses PCIe while the next one is cast.
        """
        torch = self.torch
        if isinstance(state_hat, torch.Tensor) and state_hat.is_cuda:
            if tuple(state_hat.shape) != self.state_shape():
                raise ValueError(f"state shape {tuple(state_hat.shape)} != {self.state_shape()}")
            self.u0.copy_(state_hat.to(self.cdt))
        else:
            if isinstance(state_hat, torch.Tensor):
                state_hat = state_hat.detach().numpy()
            a = np.asarray(state_hat)
            if a.shape != self.state_shape():
                raise ValueError(f"state shape {a.shape} != {self.state_shape()}")
            stage = self._host_staging()
            # torch's CPU copy casts with all host threads (numpy's copyto casts on one)
            if a.dtype not in (np.complex64, np.complex128, np.float32, np.float64):
                a = a.astype(np.complex128)
            src = torch.from_numpy(np.ascontiguousarray(a)).view(-1)
            sflat, dflat = stage.view(-1), self.u0.view(-1)
            for lo, hi in self._chunks(sflat.numel()):
                sflat[lo:hi].copy_(src[lo:hi])
                dflat[lo:hi].copy_(sflat[lo:hi], non_blocking=True)
            self._staging_free.record(torch.cuda.current_stream(self.device))
        self._check(self.lib.sp_prepare(self._h, self._stream()), "sp_prepare")

    @staticmethod
    def _chunks(count: int, parts: int = 8) -> list[tuple[int, int]]:
        """[lo, hi) element ranges of a state split for host/PCIe overlap (states of a few
        MB move whole)."""
        if count < (1 << 21):
            return [(0, count)]
        step = -(-count // parts)
        return [(lo, min(count, lo + step)) for lo in range(0, count, step)]

    def _host_staging(self) -> Any:
        """Pinned host buffer of the state's shape and dtype (reused; waits for its last copy)."""
        torch = self.torch
        if getattr(self, "_staging", None) is None:
            self._staging = torch.empty(self.state_shape(), dtype=self.cdt, pin_memory=True)
            self._staging_free = torch.cuda.Event()
            self._staging_free.record(torch.cuda.current_stream(self.device))
        self._staging_free.synchronize()
        return self._staging

    def get_state(self) -> np.ndarray:
        """The state copied to the host as complex128 (through the pinned staging buffer, chunk
        by chunk: the widening cast of a chunk, on all host threads, overlaps the copy of the
        next one over PCIe)."""
        torch = self.torch
        stage = self._host_staging()
        src, sflat = self.state_native().view(-1), stage.view(-1)
        stream = torch.cuda.current_stream(self.device)
        chunks = self._chunks(sflat.numel())
        landed = []
        for lo, hi in chunks:
            sflat[lo:hi].copy_(src[lo:hi], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(stream)
            landed.append(ev)
        out = torch.empty(stage.shape, dtype=torch.complex128)
        oflat = out.view(-1)
        for (lo, hi), ev in zip(chunks, landed):
            ev.synchronize()
            oflat[lo:hi].copy_(sflat[lo:hi])
        _lib.check_device_errors(self.lib)
        return out.numpy()

    def state_native(self) -> Any:
        """The live state (NumPy r2c layout).  Engines that advance a transposed copy write it
        back here first, so the tensor is current when returned."""
        self._check(self.lib.sp_sync_state(self._h, self._stream()), "sp_sync_state")
        return self.u0

    @property
    def kernel_launches(self) -> int:
        """Own kernels launched so far (graph replays count their kernels; cuFFT excluded)."""
        return int(self.lib.sp_kernel_launches(self._h))

    # ------------------------------------------------------------------ stepping
    def set_forcing_amplitude(self, amp: float) -> None:
        super().set_forcing_amplitude(amp)
        self._check(self.lib.sp_set_forcing_amplitude(self._h, float(self.force_amp)),
                    "sp_set_forcing_amplitude")

    def _step(self, dt: float) -> None:
        self._check(self.lib.sp_step(self._h, float(dt), self._stream()), "sp_step")

    def run_to(self, t_end: float, *, cfl: float = 0.5, dt_max: float = 0.05,
               cfl_every: int = 10, target_power: float | None = None, dt: float | None = None,
               max_steps: int = 1 << 62) -> int:
        """simulate.run's loop to ``t_end`` with its control on the device (sp_run_to): CFL
        bound and constant-power amplitude every ``cfl_every`` steps from device reductions,
        dt = min(h, t_end - t) per step, chunks of ``cfl_every`` steps replayed from one graph.
        Returns the number of steps taken."""
        t = ctypes.c_double(self.t)
        steps = ctypes.c_int64(0)
        amp = ctypes.c_double(self.force_amp)
        self._check(self.lib.sp_run_to(
            self._h, float(t_end), float(cfl), float(dt_max), int(cfl_every),
            -1.0 if target_power is None else float(target_power), float(dt or 0.0),
            int(max_steps), ctypes.byref(t), ctypes.byref(steps), ctypes.byref(amp),
            self._stream()), "sp_run_to")
        self.t = t.value
        self.nstep += int(steps.value)
        self.force_amp = amp.value
        return int(steps.value)

    def run_phase(self, phase: int, stage: int = 0) -> None:
        """One phase of one stage by itself (0 inverse FFT, 1 phys, 2 forward FFT, 3 post)."""
        self._check(self.lib.sp_run_phase(self._h, int(phase), int(stage), self._stream()),
                    "sp_run_phase")

    def _make_diag(self) -> Any:
        from pyspectral_b200.diagnostics import DeviceDiagnostics

        return DeviceDiagnostics(self)


class B200EagerSolver(B200Solver):
    """Same kernels and plans, every launch issued one by one (no graph)."""

    variant = "fused-inplace"
    use_graph = False


class B200LeanSolver(B200Solver):
    """Single-field cuFFT plans looped over the batch: cuFFT work area of one field."""

    variant = "fused-inplace-lean"
    fft_mode = _lib.FFT_CUFFT_LEAN


class B200FusedSolver(B200Solver):
    """Hand-written FFTs fused with the pointwise phases, over the 2/3-dealiased modes only;
    no cuFFT; one CUDA graph per step.

    2D (Basdevant form; n a power of two, 16..8192 fp32 / 16..4096 fp64): per RK stage one row
    pass (inverse row FFT, products, forward row FFT) and one column pass (forward column FFT,
    Lawson update, inverse column FFT).  3D (Basdevant and rotational forms; n a power of two,
    16..512): per RK stage a y-inverse pass, a z pass (c2r, products, r2c), a y-forward pass
    and an x pass (forward FFT, Leray projection and Lawson update, inverse FFT)."""

    variant = "fused-fft-graph"
    dims = (2, 3)
    forms = ("basdevant", "rotational")
    fft_mode = _lib.FFT_FUSED


def set_column_streaming(enable: bool) -> bool:
    """Choose the fused 2D engine's column pass for single runs of n = 2048..8192, process-wide
    (``sp_set_column_streaming``): True = the streamed persistent pass (default), False = one
    column per CTA.  Graphs captured earlier keep their pass.  Returns the previous setting."""
    lib = _lib.load()
    prev = bool(lib.sp_column_streaming())
    lib.sp_set_column_streaming(int(bool(enable)))
    return prev
