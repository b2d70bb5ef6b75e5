"""Time-stepping driver with the semantics of the reference's ``simulate.run``
(src/pyspectral/simulate.py:31-96): CFL-adaptive dt re-evaluated every ``cfl_every`` steps,
steps shortened to land exactly on ``t_end``, diagnostics and callback times, constant-power
band forcing ``A = P / (2 E_band)``, and wall-clock chunking.

The device work per step is one engine call (one graph launch); the only device->host reads are
the CFL velocity bound and band energy every ``cfl_every`` steps and the diagnostics records.
"""

from __future__ import annotations

import math
import time
from collections.abc import Callable
from dataclasses import dataclass, field
from typing import Any


@dataclass
class RunResult:
    """History recorded by :func:`run`."""

    t: list[float] = field(default_factory=list)
    energy: list[float] = field(default_factory=list)
    enstrophy: list[float] = field(default_factory=list)
    dt: list[float] = field(default_factory=list)
    steps: int = 0
    wall: float = 0.0
    finished: bool = True

    def as_dict(self) -> dict[str, Any]:
        return {"t": self.t, "energy": self.energy, "enstrophy": self.enstrophy, "dt": self.dt,
                "steps": self.steps, "wall_s": self.wall}


def cfl_dt(solver: Any, cfl: float, dt_max: float) -> float:
    """``cfl * dx / sum_i max|u_i|``, capped at ``dt_max`` (dt_max if the bound is 0 or not
    finite)."""
    umax = solver.diag.max_velocity_sum(solver.state_native())
    if not (umax > 0.0) or not math.isfinite(umax):
        return dt_max
    return min(dt_max, cfl * (2.0 * math.pi / solver.n) / umax)


def run(solver: Any, t_end: float, *, dt: float | None = None, cfl: float = 0.5,
        dt_max: float = 0.05, cfl_every: int = 10, diag_dt: float | None = None,
        target_power: float | None = None,
        callback: Callable[[Any], None] | None = None,
        callback_dt: float | None = None, wall_limit: float | None = None,
        result: RunResult | None = None) -> RunResult:
    """Integrate ``solver`` to ``t_end`` (fixed ``dt`` or CFL-adaptive)."""
    res = result if result is not None else RunResult()
    diag = solver.diag
    cfg = solver.cfg

    def record() -> None:
        st = solver.state_native()
        res.t.append(solver.t)
        res.energy.append(diag.energy(st))
        res.enstrophy.append(diag.enstrophy(st))

    if not res.t:
        record()
    tol = 1e-12 * max(1.0, t_end)
    next_diag = res.t[-1] + diag_dt if diag_dt else math.inf
    next_cb = solver.t + callback_dt if callback_dt else math.inf
    h_cfl = dt if dt is not None else cfl_dt(solver, cfl, dt_max)
    start = time.perf_counter()
    k = 0
    while solver.t < t_end - tol:
        if k % cfl_every == 0:
            if dt is None and k > 0:
                h_cfl = cfl_dt(solver, cfl, dt_max)
            if target_power is not None:
                eb = diag.band_energy(solver.state_native(), cfg.force_klo, cfg.force_khi)
                solver.set_forcing_amplitude(target_power / (2.0 * eb) if eb > 0 else 0.0)
        h = min(h_cfl, t_end - solver.t, next_diag - solver.t, next_cb - solver.t)
        solver.step(h)
        res.dt.append(h)
        k += 1
        if solver.t >= next_diag - tol:
            record()
            next_diag += diag_dt  # type: ignore[operator]
        if callback is not None and solver.t >= next_cb - tol:
            callback(solver)
            next_cb += callback_dt  # type: ignore[operator]
        if wall_limit is not None and time.perf_counter() - start > wall_limit:
            break
    solver.synchronize()
    res.finished = solver.t >= t_end - tol
    res.wall += time.perf_counter() - start
    res.steps += k
    if res.finished and res.t[-1] < solver.t - tol:
        record()
    return res


def run_steps(solver: Any, nsteps: int, *, cfl: float = 0.5, dt_max: float = 0.05,
              cfl_every: int = 10, target_power: float | None = None) -> list[float]:
    """Advance exactly ``nsteps`` CFL-adaptive steps (the benchmark workload: a fixed step
    count rather than a fixed end time); returns the dt of every step."""
    cfg = solver.cfg
    diag = solver.diag
    dts = []
    h = dt_max
    for k in range(nsteps):
        if k % cfl_every == 0:
            h = cfl_dt(solver, cfl, dt_max)
            if target_power is not None:
                eb = diag.band_energy(solver.state_native(), cfg.force_klo, cfg.force_khi)
                solver.set_forcing_amplitude(target_power / (2.0 * eb) if eb > 0 else 0.0)
        solver.step(h)
        dts.append(h)
    return dts


def run_device(solver: Any, t_end: float, *, dt: float | None = None, cfl: float = 0.5,
               dt_max: float = 0.05, cfl_every: int = 10,
               target_power: float | None = None) -> RunResult:
    """:func:`run` without records or callbacks, its loop control on the device
    (``solver.run_to``: CFL bound and forcing amplitude from device reductions, one graph replay
    per ``cfl_every`` steps, one host read per replay).  Same rules, same dt sequence; the
    result holds the start and end records only."""
    res = RunResult()
    diag = solver.diag

    def record() -> None:
        st = solver.state_native()
        res.t.append(solver.t)
        res.energy.append(diag.energy(st))
        res.enstrophy.append(diag.enstrophy(st))

    record()
    solver.synchronize()
    start = time.perf_counter()
    res.steps = solver.run_to(t_end, cfl=cfl, dt_max=dt_max, cfl_every=cfl_every,
                              target_power=target_power, dt=dt)
    solver.synchronize()
    res.wall = time.perf_counter() - start
    res.finished = solver.t >= t_end - 1e-12 * max(1.0, t_end)
    record()
    return res
