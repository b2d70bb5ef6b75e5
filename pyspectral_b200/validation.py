"""Physics validation runs on the device: the 3D Taylor-Green vortex at Re = 1600, the IF-RK4
temporal order and the spectral convergence in n.

Mirrors ``pyspectral.validation.tgv3d`` (src/pyspectral/validation.py:152-200): the run from
u = sin x cos y cos z, v = -cos x sin y cos z, w = 0 with nu = 1/1600 to t_end under
``simulate.run`` (CFL-adaptive dt, records every diag_dt), dissipation eps = 2 nu Z, and its
peak.  The comparison series is passed in (``reference``: a dict with "t" and "dissipation",
e.g. a published 512^3 series or the fp64 oracle's 128^3 run); nothing is read from disk.

``python -m pyspectral_b200.validation --n 512 --dtype float32 --form rotational --out run.json``
"""

from __future__ import annotations

import argparse
import json
from typing import Any

import numpy as np

from pyspectral_b200 import initial, simulate
from pyspectral_b200.config import Config
from pyspectral_b200.registry import make_solver

TGV_NU = 1.0 / 1600.0


def tgv3d(variant: str = "b200/fused-inplace-graph", n: int = 128, t_end: float = 10.0,
          cfl: float = 0.5, dtype: str = "float32", diag_dt: float = 0.1,
          form: str = "rotational", reference: dict[str, Any] | None = None) -> dict[str, Any]:
    """Run the Re = 1600 Taylor-Green vortex and return its history (t, E, Z, eps = 2 nu Z,
    -dE/dt), the dissipation peak and, with ``reference``, the error against that series
    (max |eps - eps_ref| / peak_ref over the reference's time span, peak value and time)."""
    cfg = Config(n=n, dim=3, nu=TGV_NU, dtype=dtype, form=form)
    s = make_solver(variant, cfg)
    s.set_state(initial.to_spectral(initial.taylor_green_3d(n), 3))
    res = simulate.run(s, t_end, cfl=cfl, dt_max=0.05, diag_dt=diag_dt)
    t = np.array(res.t)
    e = np.array(res.energy)
    z = np.array(res.enstrophy)
    eps = 2.0 * TGV_NU * z
    i = int(np.argmax(eps))
    out: dict[str, Any] = {
        "variant": variant, "n": n, "dtype": dtype, "form": s.form, "cfl": cfl,
        "diag_dt": diag_dt, "t_end": t_end, "steps": res.steps, "wall_s": res.wall,
        "t": t.tolist(), "energy": e.tolist(), "enstrophy": z.tolist(),
        "dissipation_2nuZ": eps.tolist(), "dissipation_dEdt": (-np.gradient(e, t)).tolist(),
        "peak_value": float(eps[i]), "peak_time": float(t[i]),
    }
    if reference is not None:
        out.update(compare_dissipation(t, eps, reference))
    return out


def compare_dissipation(t: np.ndarray, eps: np.ndarray, reference: dict[str, Any]) -> dict[str, float]:
    """Error of a dissipation history against a reference series (validation.py:181-198)."""
    tr, er = np.asarray(reference["t"], float), np.asarray(reference["dissipation"], float)
    sel = t <= tr.max()
    peak = float(er.max())
    i = int(np.argmax(eps))
    return {
        "max_abs_err_over_peak": float(np.abs(eps[sel] - np.interp(t[sel], tr, er)).max() / peak),
        "ref_peak_value": peak, "ref_peak_time": float(tr[int(np.argmax(er))]),
        "peak_rel_err": float((eps[i] - peak) / peak),
    }


def temporal_convergence(variant: str = "b200/fused-inplace-graph",
                         dts: tuple[float, ...] = (0.04, 0.02, 0.01, 0.005, 0.0025), n: int = 64,
                         nu: float = 0.01, t_end: float = 1.0) -> dict[str, Any]:
    """IF-RK4 self-convergence on a nonlinear 2D flow, fp64 (validation.py:86-100): errors of
    each dt against a run at min(dts)/8 and the least-squares order (slope of log err vs log
    dt; the reference's NumPy path measures 3.99)."""
    w0 = initial.to_spectral(initial.smooth_2d(n), 2)

    def solve(dt: float) -> np.ndarray:
        s = make_solver(variant, Config(n=n, dim=2, nu=nu, dtype="float64"))
        s.set_state(w0)
        s.advance(int(round(t_end / dt)), dt)
        return s.get_state()

    ref = solve(min(dts) / 8)
    errs = [float(np.abs(solve(dt) - ref).max() / np.abs(ref).max()) for dt in dts]
    order = float(np.polyfit(np.log(np.array(dts)), np.log(np.array(errs)), 1)[0])
    return {"variant": variant, "dt": list(dts), "err": errs, "order": order, "n": n, "nu": nu,
            "t_end": t_end}


def pad_spectrum(a: np.ndarray, n_to: int) -> np.ndarray:
    """A 2D r2c spectrum of grid n carried to grid n_to with the same physical amplitudes
    (validation.py:24-35): modes |kx| < m and 0 <= ky < m, m = min(n, n_to) // 2, copied and
    scaled by (n_to / n)^2 for the unnormalised transform; every other mode zero."""
    n = a.shape[-2]
    m = min(n, n_to) // 2
    out = np.zeros((n_to, n_to // 2 + 1), dtype=a.dtype)
    kx = np.r_[0:m, -m + 1:0]
    out[np.ix_(kx % n_to, np.arange(m))] = a[np.ix_(kx % n, np.arange(m))] * (n_to / n) ** 2
    return out


def spatial_convergence(variant: str = "b200/fused-inplace-graph",
                        ns: tuple[int, ...] = (8, 12, 16, 20, 24, 32, 40, 48, 64),
                        n_ref: int = 192, nu: float = 0.02, t_end: float = 0.5,
                        dt: float = 2.5e-3) -> dict[str, Any]:
    """Spectral convergence in n of a smooth, non-band-limited 2D flow, fp64
    (validation.py:103-119): each grid's run to t_end carried to n_ref and compared in physical
    space with the n_ref run (max error / max value)."""

    def solve(n: int) -> np.ndarray:
        s = make_solver(variant, Config(n=n, dim=2, nu=nu, dtype="float64"))
        s.set_state(initial.to_spectral(initial.smooth_2d(n), 2))
        s.advance(int(round(t_end / dt)), dt)
        return s.get_state()

    w_ref = np.fft.irfftn(solve(n_ref), s=(n_ref, n_ref), axes=(0, 1))
    errs = []
    for n in ns:
        w = np.fft.irfftn(pad_spectrum(solve(n), n_ref), s=(n_ref, n_ref), axes=(0, 1))
        errs.append(float(np.abs(w - w_ref).max() / np.abs(w_ref).max()))
    return {"variant": variant, "n": list(ns), "err": errs, "n_ref": n_ref, "nu": nu,
            "t_end": t_end, "dt": dt}


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser(description="3D Taylor-Green vortex, Re = 1600")
    ap.add_argument("--variant", default="b200/fused-inplace-graph")
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--t-end", type=float, default=10.0)
    ap.add_argument("--dtype", default="float32")
    ap.add_argument("--form", default="rotational")
    ap.add_argument("--diag-dt", type=float, default=0.1)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    r = tgv3d(a.variant, a.n, a.t_end, dtype=a.dtype, diag_dt=a.diag_dt, form=a.form)
    print(json.dumps({k: v for k, v in r.items() if not isinstance(v, list)}))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(r, f)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
