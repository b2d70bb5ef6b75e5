"""Device diagnostics of a :class:`~pyspectral_b200.solver.B200Solver`.

Same methods and meanings as the reference's ``Diagnostics`` (src/pyspectral/diagnostics.py:
20-109) — energy, enstrophy, palinstrophy, band energy, shell spectrum and the CFL velocity
bound — computed by the engine's reduction kernels (fp64 accumulation, fixed summation order)
instead of chains of array operations and library inverse FFTs.
"""

from __future__ import annotations

import ctypes
from typing import Any

import numpy as np

from pyspectral_b200 import _lib
from pyspectral_b200.grid import n_shells


class DeviceDiagnostics:
    """Energy/enstrophy/spectra of states on the solver's grid and device."""

    def __init__(self, solver: Any) -> None:
        self.solver = solver
        self.n, self.dim = solver.n, solver.dim
        self.ops = solver.ops
        self.norm = float(self.n) ** (2 * self.dim)
        self.nshell = n_shells(self.n, self.dim)

    # ------------------------------------------------------------------ helpers
    def _device_state(self, state: Any) -> Any:
        s = self.solver
        torch = s.torch
        if isinstance(state, torch.Tensor) and state.device == s.device and \
                state.dtype == s.cdt and state.is_contiguous():
            t = state
        else:
            t = torch.as_tensor(np.asarray(state) if not isinstance(state, torch.Tensor)
                                else state, device=s.device).to(s.cdt).contiguous()
        if tuple(t.shape) != s.state_shape():
            raise ValueError(f"state shape {tuple(t.shape)} != {s.state_shape()}")
        return t

    def _sums(self, state: Any, klo: float = 0.0, khi: float = -1.0) -> list[float]:
        s = self.solver
        t = self._device_state(state)
        out = (ctypes.c_double * 4)()
        s._check(s.lib.sp_diagnostics(s.handle, _lib.dptr(t), float(klo), float(khi), out,
                                      s._stream()), "sp_diagnostics")
        return list(out)

    # ------------------------------------------------------------------ API
    def energy(self, state: Any) -> float:
        """Kinetic energy <|u|^2>/2."""
        return self._sums(state)[0]

    def enstrophy(self, state: Any) -> float:
        """Enstrophy <|omega|^2>/2."""
        return self._sums(state)[1]

    def palinstrophy(self, state: Any) -> float:
        """<|grad omega|^2>/2 (2D)."""
        return self._sums(state)[2]

    def band_energy(self, state: Any, klo: float, khi: float) -> float:
        """Kinetic energy in klo <= |k| <= khi."""
        return self._sums(state, klo, khi)[3]

    def all(self, state: Any, klo: float = 0.0, khi: float = -1.0) -> dict[str, float]:
        """Energy, enstrophy, palinstrophy and band energy from one reduction pass."""
        e, z, p, b = self._sums(state, klo, khi)
        return {"energy": e, "enstrophy": z, "palinstrophy": p, "band_energy": b}

    def spectrum(self, state: Any) -> tuple[np.ndarray, np.ndarray]:
        """Shell-summed energy spectrum E(k), sum_k E(k) = E."""
        s = self.solver
        t = self._device_state(state)
        out = np.zeros(self.nshell, dtype=np.float64)
        s._check(s.lib.sp_spectrum(s.handle, _lib.dptr(t),
                                   out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                   self.nshell, s._stream()), "sp_spectrum")
        return np.arange(self.nshell), out

    def max_velocity_sum(self, state: Any) -> float:
        """sum_i max|u_i| in physical space (CFL)."""
        return self.max_velocity(state)[0]

    def max_velocity(self, state: Any) -> tuple[float, list[float]]:
        """(sum_i max|u_i|, [max|u_i| per component])."""
        s = self.solver
        t = self._device_state(state)
        tot = ctypes.c_double(0.0)
        per = (ctypes.c_double * 3)()
        s._check(s.lib.sp_max_velocity(s.handle, _lib.dptr(t), ctypes.byref(tot), per,
                                       s._stream()), "sp_max_velocity")
        return tot.value, list(per)[: self.dim]
