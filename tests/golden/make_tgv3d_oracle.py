"""Generate tgv3d_re1600_n128_fp64.json: the fp64 oracle's Taylor-Green run at Re = 1600 on
128^3 (rotational form, 2/3 dealiasing, CFL 0.5, dt_max 0.05, dt refreshed every 10 steps,
records every 0.1) to t = 10 — energy and enstrophy at every record (dissipation = 2 nu Z).

Run from the repository root: ``python tests/golden/make_tgv3d_oracle.py`` (about 27 minutes on
8 cores; 1217 steps).  The device test runs the same schedule and compares every record.
"""

from __future__ import annotations

import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.numpy_oracle import OracleSolver, run_cfl  # noqa: E402

N, NU, T_END, DIAG_DT = 128, 1.0 / 1600.0, 10.0, 0.1


def tgv3d_state(n: int) -> np.ndarray:
    """initial.py:54-63: u = sin x cos y cos z, v = -cos x sin y cos z, w = 0, as rfftn."""
    x = np.arange(n) * (2.0 * np.pi / n)
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    u = np.sin(X) * np.cos(Y) * np.cos(Z)
    v = -np.cos(X) * np.sin(Y) * np.cos(Z)
    w = np.zeros_like(u)
    return np.stack([np.fft.rfftn(c) for c in (u, v, w)])


def main() -> None:
    s = OracleSolver(N, 3, nu=NU, form="rotational")
    s.set_state(tgv3d_state(N))
    t0 = time.perf_counter()
    out = run_cfl(s, T_END, cfl=0.5, dt_max=0.05, cfl_every=10, diag_dt=DIAG_DT)
    out.update({"n": N, "nu": NU, "form": "rotational", "dtype": "float64", "cfl": 0.5,
                "dt_max": 0.05, "cfl_every": 10, "diag_dt": DIAG_DT, "t_end": T_END,
                "seconds": time.perf_counter() - t0})
    path = Path(__file__).with_name("tgv3d_re1600_n128_fp64.json")
    path.write_text(json.dumps(out))
    print(f"{out['steps']} steps in {out['seconds']:.0f} s -> {path.name}")


if __name__ == "__main__":
    main()
