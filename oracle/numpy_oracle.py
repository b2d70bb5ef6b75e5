"""ORACLE — test infrastructure only; never imported by the product package.

CPU restatement (NumPy + scipy.fft, fp64 unless asked otherwise) of the reference's correctness
oracle ``NumpySolver`` (src/pyspectral/backends/numpy_ref.py:16-153) and of the host
diagnostics it is checked with (src/pyspectral/diagnostics.py:20-109).  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm may use it, and only
as the checker or the timed CPU baseline.

Scope: the textbook IF-RK4 (Lawson) and explicit RK4 integrators with 2/3-rule dealiasing for
the 2D Basdevant / advective and 3D Basdevant / rotational forms — every form the reference's
oracle evaluates except phase-shift dealiasing, which the device path does not run either.

FFTs: the reference's oracle calls scipy.fft (pocketfft; scipy pinned ``>=1.10`` in the
reference's pyproject.toml:13, 1.18.1 installed here) as ``irfftn(a, s, axes, workers)`` /
``rfftn(a, axes, workers)`` (numpy_ref.py:62-66).  This file makes the same calls.  Parity of
this restatement is pinned by tests/golden (vectors produced by the reference itself, script
tests/golden/make_golden.py) and by the reference's known answers (exact Taylor-Green decay,
forcing e^{At}, inviscid energy conservation, Parseval).
"""

from __future__ import annotations

from typing import Any

import numpy as np
import scipy.fft as sfft


# ------------------------------------------------------------------------------- grid
def spectral_shape(n: int, dim: int) -> tuple[int, ...]:
    """grid.py:13-15."""
    return (n,) * (dim - 1) + (n // 2 + 1,)


def wavenumbers(n: int, dim: int) -> tuple[np.ndarray, ...]:
    """grid.py:18-24: fftfreq integers on full axes, 0..n/2 on the last axis."""
    k = np.fft.fftfreq(n, 1.0 / n)
    kr = np.arange(n // 2 + 1, dtype=np.float64)
    if dim == 2:
        return k[:, None], kr[None, :]
    return k[:, None, None], k[None, :, None], kr[None, None, :]


def k_squared(n: int, dim: int) -> np.ndarray:
    """grid.py:27-33."""
    out = np.zeros(spectral_shape(n, dim))
    for k in wavenumbers(n, dim):
        out = out + k * k
    return out


def dealias_mask(n: int, dim: int) -> np.ndarray:
    """2/3 rule as a cubic truncation, keep 3|k_i| < n on every axis (grid.py:36-50)."""
    m = np.ones(spectral_shape(n, dim), dtype=bool)
    for k in wavenumbers(n, dim):
        m = m & (3.0 * np.abs(k) < n)
    return m


def hermitian_weights(n: int, dim: int) -> np.ndarray:
    """grid.py:53-59."""
    w = np.full(n // 2 + 1, 2.0)
    w[0] = 1.0
    w[-1] = 1.0
    return np.broadcast_to(w.reshape((1,) * (dim - 1) + (-1,)), spectral_shape(n, dim))


# ------------------------------------------------------------------------------- solver
class OracleSolver:
    """NumpySolver restated (numpy_ref.py:16-153) for the 2/3-rule forms.

    Parameters mirror ``Config`` (config.py:12-70): n, dim, nu, alpha, alpha_kmax, force_amp,
    force_klo, force_khi, dtype, form.  ``integrator`` is "ifrk4" (Lawson) or "rk4".
    """

    def __init__(self, n: int, dim: int = 2, nu: float = 1e-3, alpha: float = 0.0,
                 alpha_kmax: float = 0.0, force_amp: float = 0.0, force_klo: float = 0.0,
                 force_khi: float = 0.0, dtype: str = "float64", form: str = "basdevant",
                 integrator: str = "ifrk4", workers: int | None = None) -> None:
        if integrator not in ("ifrk4", "rk4"):
            raise ValueError(integrator)
        forms = ("basdevant", "advective") if dim == 2 else ("basdevant", "rotational")
        if form not in forms:
            raise ValueError(form)
        self.n, self.dim, self.form, self.integrator = n, dim, form, integrator
        self.nu, self.alpha, self.alpha_kmax = nu, alpha, alpha_kmax
        self.force_amp, self.force_klo, self.force_khi = force_amp, force_klo, force_khi
        # numpy_ref.py:35: threads only pay off on large grids
        self.workers = workers if workers is not None else (-1 if n**dim >= 2**16 else 1)
        self.rdt = np.float64 if dtype == "float64" else np.float32
        self.cdt = np.complex128 if dtype == "float64" else np.complex64
        self.k = tuple(k.astype(self.rdt) for k in wavenumbers(n, dim))
        self.k2 = k_squared(n, dim).astype(self.rdt)
        self.inv_k2 = np.where(self.k2 > 0, 1.0 / np.where(self.k2 > 0, self.k2, 1), 0).astype(
            self.rdt)
        self.mask = dealias_mask(n, dim)
        self.s = (n,) * dim
        self.axes = tuple(range(-dim, 0))
        shape = spectral_shape(n, dim) if dim == 2 else (3,) + spectral_shape(n, dim)
        self.state = np.zeros(shape, self.cdt)
        self.t = 0.0
        self.nstep = 0

    @property
    def drag_k2(self) -> float:
        """config.py:59-62."""
        return self.alpha_kmax**2 if self.alpha_kmax > 0 else 1e30

    def set_state(self, state_hat: np.ndarray) -> None:
        """base.py:134-139 (mask on set) + numpy_ref.py:55-56."""
        a = np.asarray(state_hat, dtype=np.complex128)
        self.state = (a * self.mask).astype(self.cdt)

    def get_state(self) -> np.ndarray:
        return np.asarray(self.state, dtype=np.complex128)

    def set_forcing_amplitude(self, amp: float) -> None:
        self.force_amp = float(amp)

    def linear_operator(self, k2: np.ndarray) -> np.ndarray:
        """base.py:114-123."""
        L = -(self.nu * k2)
        if self.alpha != 0.0:
            L = L - (k2 * 0.0 + self.alpha) * (k2 <= self.drag_k2)
        if self.force_amp != 0.0:
            band = (k2 >= self.force_klo**2) * (k2 <= self.force_khi**2)
            L = L + (k2 * 0.0 + self.force_amp) * band
        return L

    def _irfft(self, a: np.ndarray) -> np.ndarray:
        return sfft.irfftn(a, s=self.s, axes=self.axes, workers=self.workers)

    def _rfft(self, a: np.ndarray) -> np.ndarray:
        return sfft.rfftn(a, axes=self.axes, workers=self.workers)

    def nonlinear(self, st: np.ndarray) -> np.ndarray:
        """numpy_ref.py:75-119 without phase shifts."""
        if self.dim == 2:
            kx, ky = self.k
            psi = st * self.inv_k2
            u = self._irfft(1j * ky * psi)
            v = self._irfft(-1j * kx * psi)
            if self.form == "basdevant":
                a = self._rfft(v * v - u * u)
                b = self._rfft(u * v)
                nl = kx * ky * a + (kx * kx - ky * ky) * b
            else:
                wx = self._irfft(1j * kx * st)
                wy = self._irfft(1j * ky * st)
                nl = -self._rfft(u * wx + v * wy)
            return (nl * self.mask).astype(self.cdt)
        k = self.k
        u = self._irfft(st)
        if self.form == "rotational":
            wh = np.stack([1j * (k[1] * st[2] - k[2] * st[1]),
                           1j * (k[2] * st[0] - k[0] * st[2]),
                           1j * (k[0] * st[1] - k[1] * st[0])])
            w = self._irfft(wh)
            c = np.stack([u[1] * w[2] - u[2] * w[1],
                          u[2] * w[0] - u[0] * w[2],
                          u[0] * w[1] - u[1] * w[0]])
            nl = self._rfft(c)
        else:
            q = (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]) / 3.0
            t = self._rfft(np.stack([u[0] * u[0] - q, u[1] * u[1] - q, u[0] * u[1],
                                     u[0] * u[2], u[1] * u[2]]))
            t11, t22, t12, t13, t23 = t
            t33 = -(t11 + t22)
            nl = -1j * np.stack([k[0] * t11 + k[1] * t12 + k[2] * t13,
                                 k[0] * t12 + k[1] * t22 + k[2] * t23,
                                 k[0] * t13 + k[1] * t23 + k[2] * t33])
        nl = nl * self.mask
        div = (k[0] * nl[0] + k[1] * nl[1] + k[2] * nl[2]) * self.inv_k2
        nl = np.stack([nl[i] - k[i] * div for i in range(3)])
        return nl.astype(self.cdt)

    def rhs(self, st: np.ndarray) -> np.ndarray:
        """numpy_ref.py:121-123."""
        return self.nonlinear(st) + (self.linear_operator(self.k2) * st).astype(self.cdt)

    def _step(self, dt: float) -> None:
        """numpy_ref.py:134-153."""
        u0 = self.state
        if self.integrator == "rk4":
            k1 = self.rhs(u0)
            k2 = self.rhs(u0 + 0.5 * dt * k1)
            k3 = self.rhs(u0 + 0.5 * dt * k2)
            k4 = self.rhs(u0 + dt * k3)
            self.state = (u0 + dt / 6.0 * (k1 + 2 * k2 + 2 * k3 + k4)).astype(self.cdt)
            return
        L = self.linear_operator(self.k2)
        E = np.exp(L * dt).astype(self.rdt)
        Eh = np.exp(L * (0.5 * dt)).astype(self.rdt)
        k1 = self.nonlinear(u0)
        k2 = self.nonlinear(Eh * (u0 + 0.5 * dt * k1))
        k3 = self.nonlinear(Eh * u0 + 0.5 * dt * k2)
        k4 = self.nonlinear(E * u0 + dt * Eh * k3)
        self.state = (E * u0 + dt / 6.0 * (E * k1 + 2.0 * Eh * (k2 + k3) + k4)).astype(self.cdt)

    def step(self, dt: float) -> None:
        """base.py:83-87."""
        self._step(dt)
        self.t += dt
        self.nstep += 1

    def advance(self, nsteps: int, dt: float) -> None:
        for _ in range(nsteps):
            self.step(dt)


# ------------------------------------------------------------------------------- diagnostics
class OracleDiagnostics:
    """Host diagnostics (diagnostics.py:20-109), fp64."""

    def __init__(self, n: int, dim: int) -> None:
        self.n, self.dim = n, dim
        self.norm = float(n) ** (2 * dim)
        self.k = wavenumbers(n, dim)
        self.k2 = k_squared(n, dim)
        self.w = hermitian_weights(n, dim) / self.norm
        self.nshell = int(np.floor(np.sqrt(dim) * (n // 2) + 0.5)) + 1

    def _density(self, st: np.ndarray) -> np.ndarray:
        a = np.abs(st) ** 2
        if self.dim == 3:
            a = a.sum(axis=0)
        return a * self.w

    def _energy_density(self, st: np.ndarray) -> np.ndarray:
        d = self._density(st)
        if self.dim == 2:
            inv = (self.k2 > 0) / (self.k2 + (self.k2 == 0))
            return d * inv
        return d

    def energy(self, st: np.ndarray) -> float:
        return 0.5 * float(self._energy_density(st).sum())

    def enstrophy(self, st: np.ndarray) -> float:
        d = self._density(st)
        if self.dim == 3:
            d = d * self.k2
        return 0.5 * float(d.sum())

    def palinstrophy(self, st: np.ndarray) -> float:
        d = self._density(st) * self.k2
        if self.dim == 3:
            d = d * self.k2
        return 0.5 * float(d.sum())

    def band_energy(self, st: np.ndarray, klo: float, khi: float) -> float:
        d = self._energy_density(st)
        band = (self.k2 >= klo * klo) * (self.k2 <= khi * khi)
        return 0.5 * float((d * band).sum())

    def spectrum(self, st: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        d = self._energy_density(st)
        shell = (np.sqrt(self.k2) + 0.5).astype(np.int64).reshape(-1)
        e = np.bincount(shell, 0.5 * d.reshape(-1), self.nshell)
        return np.arange(len(e)), e

    def max_velocity_sum(self, st: np.ndarray) -> float:
        s = (self.n,) * self.dim
        axes = tuple(range(-self.dim, 0))
        if self.dim == 2:
            kx, ky = self.k
            inv = (self.k2 > 0) / (self.k2 + (self.k2 == 0))
            psi = st * inv
            u = sfft.irfftn(psi * ky * 1j, s=s, axes=axes, workers=-1)
            v = sfft.irfftn(psi * kx * (-1j), s=s, axes=axes, workers=-1)
            return float(np.abs(u).max() + np.abs(v).max())
        return float(sum(np.abs(sfft.irfftn(st[i], s=s, axes=axes, workers=-1)).max()
                         for i in range(3)))


def run_fixed(solver: Any, nsteps: int, dt: float) -> np.ndarray:
    """Advance and return the state (convenience for tests)."""
    solver.advance(nsteps, dt)
    return solver.get_state()


def cfl_dt(solver: OracleSolver, diag: OracleDiagnostics, cfl: float, dt_max: float) -> float:
    """simulate.py:31-37: cfl * dx / sum_i max|u_i|, capped at dt_max (dt_max if the bound is
    0 or not finite)."""
    umax = diag.max_velocity_sum(solver.state)
    if not (umax > 0.0) or not np.isfinite(umax):
        return dt_max
    return min(dt_max, cfl * (2.0 * np.pi / solver.n) / umax)


def run_cfl(solver: OracleSolver, t_end: float, *, cfl: float = 0.5, dt_max: float = 0.05,
            cfl_every: int = 10, diag_dt: float | None = None) -> dict[str, Any]:
    """simulate.py:40-96 without forcing control or callbacks: CFL-adaptive steps (dt
    refreshed every cfl_every steps), the step clipped to the next record time and to t_end;
    energy and enstrophy recorded at t = 0, every diag_dt and at t_end."""
    diag = OracleDiagnostics(solver.n, solver.dim)
    out: dict[str, Any] = {"t": [], "energy": [], "enstrophy": [], "steps": 0}

    def record() -> None:
        out["t"].append(solver.t)
        out["energy"].append(diag.energy(solver.state))
        out["enstrophy"].append(diag.enstrophy(solver.state))

    record()
    tol = 1e-12 * max(1.0, t_end)
    next_diag = solver.t + diag_dt if diag_dt else np.inf
    h_cfl = cfl_dt(solver, diag, cfl, dt_max)
    k = 0
    while solver.t < t_end - tol:
        if k % cfl_every == 0 and k > 0:
            h_cfl = cfl_dt(solver, diag, cfl, dt_max)
        solver.step(min(h_cfl, t_end - solver.t, next_diag - solver.t))
        k += 1
        if solver.t >= next_diag - tol:
            record()
            next_diag += diag_dt  # type: ignore[operator]
    if out["t"][-1] < solver.t - tol:
        record()
    out["steps"] = k
    return out
