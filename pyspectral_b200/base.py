"""Solver interface: the contract of the reference's ``SpectralSolver``
(src/pyspectral/backends/base.py:15-144), restated so this package stands alone.

A solver holds one spectral state (2D vorticity ``(n, n//2+1)`` or 3D velocity
``(3, n, n, n//2+1)``, unnormalised ``numpy.fft.rfftn`` coefficients) and advances it by Lawson
IF-RK4 steps.  The same attribute names, method names, argument meanings and exceptions are
kept, so code written against pyspectral (its driver, diagnostics users, tests) runs unchanged
against :class:`pyspectral_b200.solver.B200Solver`.
"""

from __future__ import annotations

from abc import ABC, abstractmethod
from typing import Any, ClassVar

import numpy as np

from pyspectral_b200.config import Config, ffts_per_stage
from pyspectral_b200.grid import dealias_mask, spectral_shape


class BackendUnavailable(RuntimeError):
    """The solver cannot run here (library not built, no GPU, unsupported option)."""


class SpectralSolver(ABC):
    """Pseudo-spectral Navier-Stokes solver on a periodic ``[0, 2 pi)^d`` box."""

    backend: ClassVar[str] = "base"
    variant: ClassVar[str] = "default"
    default_form: ClassVar[str] = "basdevant"
    dims: ClassVar[tuple[int, ...]] = (2, 3)
    dtypes: ClassVar[tuple[str, ...]] = ("float32", "float64")
    phase_shift: ClassVar[bool] = False
    forms: ClassVar[tuple[str, ...] | None] = None

    def __init__(self, cfg: Config) -> None:
        if cfg.dim not in self.dims:
            raise BackendUnavailable(f"{self.backend}: dim={cfg.dim} not supported")
        if cfg.dtype not in self.dtypes:
            raise BackendUnavailable(f"{self.backend}: dtype={cfg.dtype} not supported")
        if cfg.dealias != "2/3" and not self.phase_shift:
            raise BackendUnavailable(f"{self.backend}: only 2/3-rule dealiasing")
        self.cfg = cfg
        self.n = cfg.n
        self.dim = cfg.dim
        self.form = cfg.resolved_form(self.default_form)
        if self.forms is not None and self.form not in self.forms:
            raise BackendUnavailable(f"{self.backend}: form={self.form} not supported")
        self.force_amp = cfg.force_amp
        self.t = 0.0
        self.nstep = 0
        self._diag: Any = None

    @classmethod
    def available(cls) -> tuple[bool, str]:
        """(ok, reason) — whether this solver can run on this machine.  Never raises."""
        return True, ""

    @abstractmethod
    def set_state(self, state_hat: np.ndarray) -> None:
        """Load a spectral state given on the host (NumPy convention)."""

    @abstractmethod
    def state_native(self) -> Any:
        """The live spectral state as a device array in NumPy layout."""

    @abstractmethod
    def _step(self, dt: float) -> None:
        """Advance the state by one IF-RK4 step of size ``dt``."""

    @property
    @abstractmethod
    def ops(self) -> Any:
        """Array shim used by diagnostics."""

    def get_state(self) -> np.ndarray:
        """The state copied to the host as complex128."""
        return np.asarray(self.ops.to_numpy(self.state_native()), dtype=np.complex128)

    def step(self, dt: float) -> None:
        """One time step; advances ``t`` and ``nstep``."""
        self._step(dt)
        self.t += dt
        self.nstep += 1

    def advance(self, nsteps: int, dt: float) -> None:
        """``nsteps`` fixed steps of size ``dt``."""
        for _ in range(nsteps):
            self.step(dt)

    def synchronize(self) -> None:
        """Wait for queued device work."""
        self.ops.synchronize()

    def set_forcing_amplitude(self, amp: float) -> None:
        """Band-forcing growth rate ``A``, used from the next step on."""
        self.force_amp = float(amp)

    @property
    def diag(self) -> Any:
        """Diagnostics of this solver's grid (built on first use)."""
        if self._diag is None:
            self._diag = self._make_diag()
        return self._diag

    def _make_diag(self) -> Any:
        raise NotImplementedError

    @property
    def fft_per_step(self) -> int:
        """Real FFTs per time step (4 RK stages)."""
        return 4 * ffts_per_stage(self.dim, self.form)

    def linear_operator(self, k2: Any) -> Any:
        """``L(k)`` on a k^2 array (NumPy or torch): viscosity, drag band, forcing band."""
        c = self.cfg
        lin = -(c.nu * k2)
        if c.alpha != 0.0:
            lin = lin - (k2 * 0.0 + c.alpha) * (k2 <= c.drag_k2)
        if self.force_amp != 0.0:
            band = (k2 >= c.force_klo**2) * (k2 <= c.force_khi**2)
            lin = lin + (k2 * 0.0 + self.force_amp) * band
        return lin

    def mask_np(self) -> np.ndarray:
        """Dealiasing mask on the host."""
        return dealias_mask(self.n, self.dim, self.cfg.dealias)

    def state_shape(self) -> tuple[int, ...]:
        s = spectral_shape(self.n, self.dim)
        return s if self.dim == 2 else (3,) + s

    def check_state(self, state_hat: np.ndarray) -> np.ndarray:
        """Shape check (ValueError) and dealiasing of a host state."""
        a = np.asarray(state_hat, dtype=np.complex128)
        if a.shape != self.state_shape():
            raise ValueError(f"state shape {a.shape} != {self.state_shape()}")
        return a * self.mask_np()

    def describe(self) -> str:
        return (f"{self.backend}/{self.variant} dim={self.dim} n={self.n} {self.cfg.dtype} "
                f"form={self.form} ({self.fft_per_step} FFTs/step)")
