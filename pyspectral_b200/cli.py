"""Command line: ``python -m pyspectral_b200 list|run`` with the options of ``pyspectral
list|run`` (src/pyspectral/cli.py:18-49, 119-173) for this package's variants."""

from __future__ import annotations

import argparse
import sys

import numpy as np

from pyspectral_b200 import initial
from pyspectral_b200.config import Config
from pyspectral_b200.registry import available, make_solver


def _cmd_list(_: argparse.Namespace) -> int:
    for v, ok, why in available():
        flag = "ok " if ok else "-- "
        print(f"{flag} {v.name:36s} {v.description}" + ("" if ok else f"  [{why}]"))
    return 0


def _initial(case: str, n: int, dim: int, seed: int) -> np.ndarray:
    if dim == 2:
        if case == "random-phase":
            return initial.random_phase_2d(n, seed=seed)
        f = {"tgv": initial.taylor_green_2d, "smooth": initial.smooth_2d,
             "random": lambda m: initial.random_2d(m, seed=seed)}[case](n)
    else:
        f = {"tgv": initial.taylor_green_3d,
             "random": lambda m: initial.random_3d(m, seed=seed)}[case](n)
    return initial.to_spectral(f, dim)


def _cmd_run(a: argparse.Namespace) -> int:
    from pyspectral_b200.checkpoint import load_checkpoint, save_checkpoint
    from pyspectral_b200.simulate import run

    cfg = Config(n=a.n, dim=a.dim, nu=a.nu, alpha=a.alpha, dtype=a.dtype, form=a.form)
    s = make_solver(a.backend, cfg)
    prev = None
    if a.resume:
        prev, _ = load_checkpoint(a.resume, s)
    else:
        s.set_state(_initial(a.case, a.n, a.dim, a.seed))
    print(s.describe())
    res = run(s, a.t_end, dt=a.dt, cfl=a.cfl, diag_dt=a.t_end / 10, wall_limit=a.wall_limit,
              result=prev)
    for t, e, z in zip(res.t, res.energy, res.enstrophy, strict=True):
        print(f"t={t:8.4f}  E={e:.8e}  Z={z:.8e}")
    ms = 1e3 * res.wall / max(res.steps, 1)
    print(f"{res.steps} steps in {res.wall:.2f} s ({ms:.3f} ms/step)")
    if a.out:
        save_checkpoint(a.out, s, res)
    return 0 if res.finished else 3


def main(argv: list[str] | None = None) -> int:
    p = argparse.ArgumentParser(prog="pyspectral_b200", description=__doc__)
    sub = p.add_subparsers(dest="cmd", required=True)
    sub.add_parser("list", help="list variants and availability").set_defaults(fn=_cmd_list)
    r = sub.add_parser("run", help="run a simulation and print diagnostics")
    r.add_argument("--backend", default="b200")
    r.add_argument("--dim", type=int, default=2)
    r.add_argument("--n", type=int, default=128)
    r.add_argument("--nu", type=float, default=1e-3)
    r.add_argument("--alpha", type=float, default=0.0)
    r.add_argument("--dtype", default="float64")
    r.add_argument("--form", default="auto")
    r.add_argument("--case", default="random", choices=["tgv", "smooth", "random", "random-phase"])
    r.add_argument("--seed", type=int, default=0)
    r.add_argument("--t-end", type=float, default=1.0)
    r.add_argument("--dt", type=float, default=None)
    r.add_argument("--cfl", type=float, default=0.5)
    r.add_argument("--wall-limit", type=float, default=None)
    r.add_argument("--out", default=None, help="write a checkpoint (.npz) at the end")
    r.add_argument("--resume", default=None, help="continue from a checkpoint")
    r.set_defaults(fn=_cmd_run)
    a = p.parse_args(argv)
    return int(a.fn(a))


if __name__ == "__main__":
    sys.exit(main())
