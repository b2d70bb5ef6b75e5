"""Learned-closure study: filtered forced-DNS data from the batched engine, training, and the
a-posteriori test of the coarse closure run against fine DNS, with DNS as fallback.

No reference counterpart.  The workload (defaults of :class:`StudyConfig`):

* DNS: 2048^2 fp32, nu = 5e-6, constant-power band forcing on 10 <= |k| <= 12 with P = 1e-3,
  drag alpha = 0.1 on |k| <= 2, CFL 0.5.  Runs start from a random-phase field (k0 = 8) with
  energy ``e0``; they are spun up on a 512^2 grid (nu chosen for k_max eta = 1 there), zero-
  padded to 2048^2 with the spectral filter and run on at 2048^2 for ``t_settle`` before use.
* Data: 4000 snapshots from 16 training seeds, advanced together by the batched ensemble
  engine; each snapshot is sharp-spectral-filtered to k <= 85 (the 2/3 cutoff of 256^2) and
  stored as (omega, d omega/dx, d omega/dy, S) with S = F[N(omega)] - N_c(F[omega]).
* Training: 20000 Adam steps at 512 tiles x 128 points = 65536 points per step, for each
  learning rate of a short sweep; the lowest final training loss is kept.
* Coarse runs evaluate the network once per step (first RK stage) and hold its term for the
  other stages (``every_stage=False``), or at every stage.
* Closure variants: the trained network as is; scaled by one a-priori enstrophy-transfer gain
  <omega S_true> / <omega S_model>; scaled per shell so that its mean transfer matches the
  true subgrid transfer shell by shell; that per-shell gain from the forcing band up only.  All
  gains are measured on training snapshots; the variant, then one overall multiplier on its
  gains, then a ramp of the gains toward the cutoff (1 + b x^2, x rising from 0 at
  cutoff_from * 85 to 1 at 85, capped at 1.5 beyond it) are chosen on 8 validation seeds
  (a-posteriori E(k) error), never on the test seeds.
* A-posteriori test on 16 held-out seeds: from the filtered DNS state at t0, a 256^2 run with
  the chosen closure and the 2048^2 DNS advance to t0 + t_eval; E(k) and the enstrophy flux are
  averaged over seeds and over the records from t0 + eval_start on, and compared for
  1 <= k <= 85.  The closure is accepted when max_k |E_les / E_dns - 1| <= err_bound; otherwise
  coarse runs fall back to the DNS (:func:`run_coarse_or_fine`).  A 256^2 run without closure
  is reported beside it, and the wall time of one closure run and of one DNS run to t_eval.
"""

from __future__ import annotations

import dataclasses
import json
import math
import time
from dataclasses import dataclass
from typing import Any

import numpy as np

from pyspectral_b200 import simulate
from pyspectral_b200.closure import (ClosureNet, ClosureSolver, SnapshotPipeline,
                                     filter_spectrum, init_params, nonlinear_term)
from pyspectral_b200.config import Config
from pyspectral_b200.ensemble import Ensemble, nu_for_kmax_eta
from pyspectral_b200.initial import random_phase_2d
from pyspectral_b200.solver import B200FusedSolver, B200Solver


@dataclass
class StudyConfig:
    n_fine: int = 2048
    n_coarse: int = 256
    nu: float = 5e-6
    power: float = 1e-3
    force_klo: float = 10.0
    force_khi: float = 12.0
    alpha: float = 0.1
    alpha_kmax: float = 2.0
    k0: float = 8.0
    e0: float = 5e-3
    cfl: float = 0.5
    dt_max: float = 0.05
    n_spin: int = 512
    t_spin: float = 40.0
    t_settle: float = 5.0
    train_seeds: int = 16
    snapshots: int = 4000
    snap_every: int = 250
    test_seeds: int = 16
    test_seed0: int = 1000
    val_seeds: int = 8
    val_seed0: int = 2000
    t_eval: float = 10.0
    eval_dt: float = 0.5
    eval_start: float = 2.0
    train_steps: int = 20000
    batch_tiles: int = 512
    lr: float = 1e-3
    lr_sweep: tuple[float, ...] = (1e-3, 3e-3, 1e-2)
    # the a-posteriori error is sharp around the calibrated gains (0.75x and 1.5x, or a cutoff
    # ramp of +-0.5, already double it on validation): fine steps near 1
    gain_sweep: tuple[float, ...] = (0.5, 0.75, 0.9, 0.95, 1.05, 1.1, 1.5, 2.0)
    cutoff_sweep: tuple[float, ...] = (-0.3, -0.15, -0.05, 0.05, 0.15, 0.3)
    cutoff_from: float = 0.7
    every_stage: bool = False
    lr_min: float = 1e-5
    warmup: int = 200
    clip: bool = False
    err_bound: float = 0.10

    @property
    def k_check(self) -> int:
        """Largest wavenumber kept by the coarse grid's 2/3 mask (85 for 256^2)."""
        return (self.n_coarse - 1) // 3

    @classmethod
    def small(cls) -> StudyConfig:
        """A minutes-free configuration that exercises every stage (tests, smoke runs)."""
        return cls(n_fine=256, n_coarse=128, nu=2e-4, n_spin=128, t_spin=2.0, t_settle=0.5,
                   train_seeds=2, snapshots=24, snap_every=10, test_seeds=2, val_seeds=1, t_eval=1.0,
                   eval_dt=0.25, eval_start=0.25, train_steps=120, batch_tiles=32, warmup=10)


def forced_config(sc: StudyConfig, n: int, nu: float) -> Config:
    return Config(n=n, dim=2, nu=nu, alpha=sc.alpha, alpha_kmax=sc.alpha_kmax,
                  force_klo=sc.force_klo, force_khi=sc.force_khi, dtype="float32")


def _k_force(sc: StudyConfig) -> float:
    return 0.5 * (sc.force_klo + sc.force_khi)


# ---------------------------------------------------------------------- data generation
def _advance(ens: Ensemble, sc: StudyConfig, t_end: float, chunk: int = 200) -> None:
    """Advance every member (per-member CFL dt, constant-power forcing) to at least t_end."""
    while ens.t.min() < t_end:
        ens.run_steps(chunk, cfl=sc.cfl, dt_max=sc.dt_max, target_power=sc.power)
        if not np.all(np.isfinite(ens.diagnostics()[:, 0])):
            raise FloatingPointError("ensemble member diverged")


def fine_states(sc: StudyConfig, seeds: list[int]) -> list[Any]:
    """Statistically developed fine-grid states (device complex64) for the given seeds: spin-up
    on n_spin, padded to n_fine, then t_settle on n_fine (batched engine throughout)."""
    nu_spin = nu_for_kmax_eta(sc.n_spin, sc.power, _k_force(sc)) if sc.n_spin < sc.n_fine else sc.nu
    spin = Ensemble([forced_config(sc, sc.n_spin, max(nu_spin, sc.nu)) for _ in seeds])
    spin.set_states([random_phase_2d(sc.n_spin, k0=sc.k0, seed=s, energy=sc.e0) for s in seeds])
    _advance(spin, sc, sc.t_spin)
    up = [filter_spectrum(spin.state_native(i).contiguous(), sc.n_fine) for i in range(len(seeds))]
    del spin
    fine = Ensemble([forced_config(sc, sc.n_fine, sc.nu) for _ in seeds])
    fine.set_states([u.cpu().numpy() for u in up])
    _advance(fine, sc, sc.t_settle)
    return [fine.state_native(i).clone() for i in range(len(seeds))]


def collect_snapshots(sc: StudyConfig, net: ClosureNet, pipe: SnapshotPipeline,
                      states: list[Any]) -> dict[str, float]:
    """Advance the training runs together and add sc.snapshots filtered snapshots to the bank."""
    t0 = time.perf_counter()
    ens = Ensemble([forced_config(sc, sc.n_fine, sc.nu) for _ in states])
    ens.set_states([s.cpu().numpy() for s in states])
    per = math.ceil(sc.snapshots / len(states))
    taken = 0
    for _ in range(per):
        ens.run_steps(sc.snap_every, cfl=sc.cfl, dt_max=sc.dt_max, target_power=sc.power)
        for i in range(len(states)):
            if taken < sc.snapshots:
                pipe.add(ens.state_native(i))
                taken += 1
    net.torch.cuda.synchronize()
    return {"snapshots": taken, "dns_steps": ens.nstep, "t_span": float(ens.t.mean()),
            "seconds": time.perf_counter() - t0}


def train(sc: StudyConfig, net: ClosureNet, seed: int = 0) -> dict[str, Any]:
    """sc.train_steps Adam steps from the same initialisation for each learning rate of
    sc.lr_sweep (or sc.lr alone); the network with the lowest final training loss is kept."""
    net.fit_scales(clip=sc.clip)
    runs = []
    best: tuple[float, np.ndarray] | None = None
    for lr in (sc.lr_sweep or (sc.lr,)):
        net.set_params(init_params(seed))
        net.set_adam(lr=lr, lr_min=sc.lr_min, total_steps=sc.train_steps, warmup=sc.warmup)
        net.torch.cuda.synchronize()
        t0 = time.perf_counter()
        losses = net.train(sc.train_steps, batch_tiles=sc.batch_tiles, seed=seed)
        sec = time.perf_counter() - t0
        w = max(1, min(100, len(losses) // 10))
        run = {"lr": lr, "seconds": sec, "ms_per_step": 1e3 * sec / max(1, sc.train_steps),
               "loss_first": float(losses[:w].mean()), "loss_last": float(losses[-w:].mean())}
        runs.append(run)
        if np.isfinite(run["loss_last"]) and (best is None or run["loss_last"] < best[0]):
            best = (run["loss_last"], net.params())
    if best is not None:
        net.set_params(best[1])
    chosen = min(runs, key=lambda r: r["loss_last"] if np.isfinite(r["loss_last"]) else np.inf)
    return {"steps": sc.train_steps, "points_per_step": sc.batch_tiles * 128, "runs": runs,
            "lr": chosen["lr"], "seconds": chosen["seconds"], "ms_per_step": chosen["ms_per_step"],
            "loss_first": chosen["loss_first"], "loss_last": chosen["loss_last"]}


# ---------------------------------------------------------------------- diagnostics
class FluxMeter:
    """Shell energy spectrum and enstrophy flux Pi_Z(k) = -sum_{|k'| <= k} T_Z(k'),
    T_Z(k) = sum over shell k of w Re(conj(omega_k) N_k) / n^4 (w: r2c Hermitian weight)."""

    def __init__(self, solver: B200Solver, kmax: int) -> None:
        torch = solver.torch
        self.solver, self.kmax, self.n = solver, kmax, solver.n
        n = self.n
        kx = torch.fft.fftfreq(n, 1.0 / n, device=solver.device)[:, None]
        ky = torch.arange(n // 2 + 1, device=solver.device, dtype=kx.dtype)[None, :]
        k = torch.sqrt(kx * kx + ky * ky)
        self.shell = (k + 0.5).long().flatten()
        w = torch.full((n // 2 + 1,), 2.0, device=solver.device, dtype=torch.float64)
        w[0] = 1.0
        w[-1] = 1.0
        self.w = w[None, :].expand(n, -1).flatten()
        self.nshell = int(self.shell.max()) + 1
        self.keep = ((3 * kx.abs() < n) & (3 * ky < n)).to(torch.float32)
        self.kx, self.ky = kx, ky

    def transfer(self, state: Any, nl: Any) -> np.ndarray:
        torch = self.solver.torch
        d = (state.conj() * nl).real.to(torch.float64).flatten() * self.w
        t = torch.bincount(self.shell, weights=d, minlength=self.nshell) / float(self.n) ** 4
        return t[: self.kmax + 1].cpu().numpy()

    def flux(self, state: Any, nl: Any) -> np.ndarray:
        return -np.cumsum(self.transfer(state, nl))

    def spectrum(self, state: Any) -> np.ndarray:
        return self.solver.diag.spectrum(state)[1][: self.kmax + 1]

    def closure_term(self, net: ClosureNet, state: Any) -> Any:
        """mask * FFT(S) of the network's subgrid term for a coarse spectral state."""
        torch = self.solver.torch
        w = state * self.keep
        spec = torch.stack([w, 1j * self.kx * w, 1j * self.ky * w])
        fields = torch.fft.irfft2(spec, s=(self.n, self.n)).to(torch.float32)
        S = net.infer(fields)
        return torch.fft.rfft2(S) * self.keep


@dataclass
class RunRecord:
    spectra: list[np.ndarray] = dataclasses.field(default_factory=list)
    fluxes: list[np.ndarray] = dataclasses.field(default_factory=list)
    times: list[float] = dataclasses.field(default_factory=list)
    steps: int = 0
    wall: float = 0.0
    finite: bool = True


def _record_run(solver: Any, meter: FluxMeter, nl_of: Any, sc: StudyConfig) -> RunRecord:
    rec = RunRecord()

    def cb(s: Any) -> None:
        if s.t + 1e-9 < sc.eval_start:
            return
        st = s.state_native()
        if not bool(s.torch.isfinite(st).all()):
            rec.finite = False
            return
        rec.times.append(s.t)
        rec.spectra.append(meter.spectrum(st))
        rec.fluxes.append(meter.flux(st, nl_of(st)))

    res = simulate.run(solver, sc.t_eval, cfl=sc.cfl, dt_max=sc.dt_max, target_power=sc.power,
                       callback=cb, callback_dt=sc.eval_dt)
    rec.steps, rec.wall = res.steps, res.wall
    return rec


def _timed_run(solver: Any, state: Any, sc: StudyConfig) -> tuple[float, int]:
    """Wall time of one run to t_eval with the run loop's control on the device (CFL and
    constant-power forcing every 10 steps, simulate.run_device); the chunk graph is captured by
    a short untimed run first."""
    solver.set_state(state)
    solver.run_to(1e-6, cfl=sc.cfl, dt_max=sc.dt_max, target_power=sc.power)
    solver.set_state(state)
    solver.t = 0.0
    solver.synchronize()
    res = simulate.run_device(solver, sc.t_eval, cfl=sc.cfl, dt_max=sc.dt_max,
                              target_power=sc.power)
    return res.wall, res.steps


@dataclass
class Variant:
    name: str
    gain: np.ndarray  # per-shell gain of the closure term

    def describe(self) -> dict[str, Any]:
        return {"name": self.name, "gain": [round(float(g), 4) for g in self.gain]}


def transfer_spectra(net: ClosureNet, max_entries: int = 256) -> tuple[np.ndarray, np.ndarray]:
    """Shell sums of the enstrophy transfer Re(conj(omega_k) S_k) of the true and of the modelled
    subgrid term over (part of) the bank (training snapshots)."""
    torch = net.torch
    n = net.n
    kx = torch.fft.fftfreq(n, 1.0 / n, device=net.device)[:, None]
    ky = torch.arange(n // 2 + 1, device=net.device, dtype=kx.dtype)[None, :]
    shell = (torch.sqrt(kx * kx + ky * ky) + 0.5).long().flatten()
    w = torch.full((n // 2 + 1,), 2.0, device=net.device, dtype=torch.float64)
    w[0] = 1.0
    w[-1] = 1.0
    w = w[None, :].expand(n, -1).flatten()
    t_true = torch.zeros(net.nshell, dtype=torch.float64, device=net.device)
    t_pred = torch.zeros_like(t_true)
    count = net.bank_count
    for i in np.unique(np.linspace(0, count - 1, min(count, max_entries)).round().astype(int)):
        e = torch.from_numpy(net.bank_entry(int(i))).to(net.device)
        pred = net.infer(e[:3])
        om = torch.fft.rfft2(e[0].double())
        for acc, s in ((t_true, e[3]), (t_pred, pred)):
            d = (om.conj() * torch.fft.rfft2(s.double())).real.flatten() * w
            acc += torch.bincount(shell, weights=d, minlength=net.nshell)[: net.nshell]
    return t_true.cpu().numpy(), t_pred.cpu().numpy()


def _ratio_gain(t_true: np.ndarray, t_pred: np.ndarray) -> np.ndarray:
    """t_true / t_pred in [0, 3]; 0 where the two disagree in sign; 0 for the mean (shell 0)."""
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.where(t_true * t_pred > 0, t_true / np.where(t_pred != 0, t_pred, 1.0), 0.0)
    g = np.clip(r, 0.0, 3.0).astype(np.float32)
    g[0] = 0.0
    return g


def calibrate(sc: StudyConfig, net: ClosureNet) -> list[Variant]:
    """The closure variants, every gain measured on training snapshots:
    mse         the trained network as is;
    calibrated  one gain: total true subgrid enstrophy transfer / modelled transfer;
    shell       per shell, modelled transfer matched to the true transfer in that shell;
    shell_band  the per-shell gain from the forcing band up, 0 below;
    smooth      per shell from transfers summed over +-3 neighbouring shells;
    flux        per shell from the cumulative transfers (the enstrophy fluxes) up to it."""
    t_true, t_pred = transfer_spectra(net)
    kc = sc.k_check
    ones = np.ones(net.nshell, np.float32)
    tot_p = t_pred[1: kc + 1].sum()
    scalar = float(t_true[1: kc + 1].sum() / tot_p) if tot_p != 0 else 1.0
    scalar = scalar if scalar > 0 else 1.0
    shell = _ratio_gain(t_true, t_pred)
    band = shell.copy()
    band[: int(sc.force_klo)] = 0.0
    box = np.ones(7)
    smooth = _ratio_gain(np.convolve(t_true, box, "same"), np.convolve(t_pred, box, "same"))
    flux = _ratio_gain(np.cumsum(t_true), np.cumsum(t_pred))
    return [Variant("mse", ones), Variant("calibrated", ones * np.float32(scalar)),
            Variant("shell", shell), Variant("shell_band", band), Variant("smooth", smooth),
            Variant("flux", flux)]


def _dns_records(sc: StudyConfig, pipe: SnapshotPipeline, states: list[Any]) -> list[RunRecord]:
    meter = FluxMeter(pipe.fine, sc.k_check)
    out = []
    for st in states:
        dns = B200FusedSolver(forced_config(sc, sc.n_fine, sc.nu))
        dns.set_state(st)
        out.append(_record_run(dns, meter, lambda s: nonlinear_term(pipe.fine, s), sc))
    return out


def _coarse_records(sc: StudyConfig, pipe: SnapshotPipeline, states: list[Any],
                    net: ClosureNet | None) -> list[RunRecord]:
    meter = FluxMeter(pipe.coarse, sc.k_check)
    cfg = forced_config(sc, sc.n_coarse, sc.nu)
    out = []
    for st in states:
        wbar = filter_spectrum(st, sc.n_coarse)
        if net is None:
            s = B200Solver(cfg)
            nl = lambda x: nonlinear_term(pipe.coarse, x)  # noqa: E731
        else:
            s = ClosureSolver(cfg, net, every_stage=sc.every_stage)
            nl = lambda x: nonlinear_term(pipe.coarse, x) + meter.closure_term(net, x)  # noqa: E731
        s.set_state(wbar)
        out.append(_record_run(s, meter, nl, sc))
    return out


def _mean(recs: list[RunRecord], key: str) -> np.ndarray | None:
    if not recs or not all(r.finite for r in recs):
        return None
    rows = [a for r in recs for a in getattr(r, key)]
    return np.mean(rows, axis=0) if rows else None


def _compare(recs: list[RunRecord], dns: list[RunRecord]) -> dict[str, Any]:
    e_dns, f_dns = _mean(dns, "spectra"), _mean(dns, "fluxes")
    e, f = _mean(recs, "spectra"), _mean(recs, "fluxes")
    if e is None or e_dns is None:
        return {"finite": False}
    rel = np.abs(e[1:] / e_dns[1:] - 1.0)
    fl = np.linalg.norm(f[1:] - f_dns[1:]) / np.linalg.norm(f_dns[1:])
    return {"finite": True, "e_err_max": float(rel.max()), "e_err_mean": float(rel.mean()),
            "e_err_argmax_k": int(1 + rel.argmax()), "flux_err_l2": float(fl),
            "spectrum": e.tolist(), "flux": f.tolist()}


def _apply(net: ClosureNet, v: Variant) -> None:
    net.set_shell_gain(v.gain)


def select_variant(sc: StudyConfig, net: ClosureNet, pipe: SnapshotPipeline,
                   val_states: list[Any]) -> tuple[Variant, dict[str, Any]]:
    """The variant with the smallest a-posteriori E(k) error on the validation seeds."""
    dns = _dns_records(sc, pipe, val_states)
    report: dict[str, Any] = {}
    variants = calibrate(sc, net)
    best: tuple[float, Variant] | None = None
    for v in variants:
        _apply(net, v)
        cmp = _compare(_coarse_records(sc, pipe, val_states, net), dns)
        report[v.name] = {k: x for k, x in cmp.items() if k not in ("spectrum", "flux")}
        if cmp.get("finite") and (best is None or cmp["e_err_max"] < best[0]):
            best = (cmp["e_err_max"], v)
    chosen = best[1] if best is not None else variants[0]
    # one overall multiplier on the chosen gain profile, also chosen on the validation seeds
    for a in sc.gain_sweep:
        v = Variant(f"{chosen.name}*{a:g}", chosen.gain * np.float32(a))
        _apply(net, v)
        cmp = _compare(_coarse_records(sc, pipe, val_states, net), dns)
        report[v.name] = {k: x for k, x in cmp.items() if k not in ("spectrum", "flux")}
        if cmp.get("finite") and best is not None and cmp["e_err_max"] < best[0]:
            best = (cmp["e_err_max"], v)
    chosen = best[1] if best is not None else variants[0]
    # the gains near the cutoff, where the resolved spectrum is most sensitive to the closure
    ramp = cutoff_ramp(sc, net.nshell)
    for b in sc.cutoff_sweep:
        v = Variant(f"{chosen.name}+cut{b:g}",
                    np.maximum(chosen.gain * (1.0 + np.float32(b) * ramp), 0).astype(np.float32))
        _apply(net, v)
        cmp = _compare(_coarse_records(sc, pipe, val_states, net), dns)
        report[v.name] = {k: x for k, x in cmp.items() if k not in ("spectrum", "flux")}
        if cmp.get("finite") and best is not None and cmp["e_err_max"] < best[0]:
            best = (cmp["e_err_max"], v)
    chosen = best[1] if best is not None else variants[0]
    _apply(net, chosen)
    return chosen, report


def cutoff_ramp(sc: StudyConfig, nshell: int) -> np.ndarray:
    """x^2 per shell, x = (k - k0) / (kc - k0) clipped to [0, 1.5], k0 = cutoff_from * kc."""
    kc = float(sc.k_check)
    k0 = sc.cutoff_from * kc
    x = np.clip((np.arange(nshell, dtype=np.float64) - k0) / max(kc - k0, 1e-9), 0.0, 1.5)
    return (x * x).astype(np.float32)


def evaluate(sc: StudyConfig, net: ClosureNet, pipe: SnapshotPipeline,
             states: list[Any]) -> dict[str, Any]:
    """A-posteriori comparison of closure runs (and plain coarse runs) with the DNS."""
    dns = _dns_records(sc, pipe, states)
    les_cmp = _compare(_coarse_records(sc, pipe, states, net), dns)
    plain_cmp = _compare(_coarse_records(sc, pipe, states, None), dns)
    e_dns, f_dns = _mean(dns, "spectra"), _mean(dns, "fluxes")
    # one DNS run and one closure run to t_eval, no records: the wall-time comparison
    dns_wall, dns_steps = _timed_run(B200FusedSolver(forced_config(sc, sc.n_fine, sc.nu)),
                                     states[0], sc)
    les_wall, les_steps = _timed_run(
        ClosureSolver(forced_config(sc, sc.n_coarse, sc.nu), net, every_stage=sc.every_stage),
        filter_spectrum(states[0], sc.n_coarse), sc)
    accepted = bool(les_cmp.get("finite") and les_cmp["e_err_max"] <= sc.err_bound)
    return {
        "k": list(range(sc.k_check + 1)),
        "dns_spectrum": None if e_dns is None else e_dns.tolist(),
        "dns_flux": None if f_dns is None else f_dns.tolist(),
        "closure": les_cmp, "no_closure": plain_cmp,
        "records_per_run": len(dns[0].times) if dns else 0,
        "dns_wall_s": dns_wall, "dns_steps": dns_steps, "les_wall_s": les_wall,
        "les_steps": les_steps, "wall_ratio": dns_wall / les_wall if les_wall > 0 else None,
        "err_bound": sc.err_bound, "accepted": accepted,
    }


def a_priori_correlation(net: ClosureNet, pipe: SnapshotPipeline, states: list[Any]) -> float:
    """Correlation of predicted and true subgrid terms on held-out snapshots (bank entries
    appended after training)."""
    torch = net.torch
    num = den_a = den_b = 0.0
    for st in states:
        pipe.add(st)
        e = net.bank_entry(net.bank_count - 1)
        pred = net.infer(torch.from_numpy(e[:3]).to(net.device)).cpu().numpy().astype(np.float64)
        true = e[3].astype(np.float64)
        num += float((pred * true).sum())
        den_a += float((pred * pred).sum())
        den_b += float((true * true).sum())
    return num / math.sqrt(den_a * den_b) if den_a > 0 and den_b > 0 else 0.0


# ---------------------------------------------------------------------- fallback
def run_coarse_or_fine(net: ClosureNet | None, accepted: bool, sc: StudyConfig, state_fine: Any,
                       t_end: float) -> tuple[Any, str]:
    """Advance a fine-grid state to t_end: with the closure on the coarse grid when it passed
    its a-posteriori test, else with the fine-grid DNS (the fallback).  Returns the solver and
    which path ran ("closure" or "dns")."""
    if net is not None and accepted:
        s = ClosureSolver(forced_config(sc, sc.n_coarse, sc.nu), net, every_stage=sc.every_stage)
        s.set_state(filter_spectrum(state_fine, sc.n_coarse))
        path = "closure"
    else:
        s = B200FusedSolver(forced_config(sc, sc.n_fine, sc.nu))
        s.set_state(state_fine)
        path = "dns"
    simulate.run(s, t_end, cfl=sc.cfl, dt_max=sc.dt_max, target_power=sc.power)
    return s, path


# ---------------------------------------------------------------------- the whole study
def run_study(sc: StudyConfig, seed: int = 0, log: Any = None) -> dict[str, Any]:
    def say(msg: str) -> None:
        if log is not None:
            print(msg, file=log, flush=True)

    out: dict[str, Any] = {"config": dataclasses.asdict(sc)}
    t0 = time.perf_counter()
    train_seeds = list(range(sc.train_seeds))
    test_seeds = [sc.test_seed0 + i for i in range(sc.test_seeds)]
    tr = fine_states(sc, train_seeds)
    out["t_data_spinup_s"] = time.perf_counter() - t0
    say(f"training runs spun up in {out['t_data_spinup_s']:.1f} s")
    net = ClosureNet(sc.n_coarse, sc.snapshots + min(4, sc.test_seeds))
    pipe = SnapshotPipeline(net, sc.n_fine)
    out["data"] = collect_snapshots(sc, net, pipe, tr)
    say(f"data: {out['data']}")
    del tr
    out["train"] = train(sc, net, seed)
    say(f"train: {out['train']}")
    t1 = time.perf_counter()
    va = fine_states(sc, [sc.val_seed0 + i for i in range(sc.val_seeds)])
    variant, out["validation"] = select_variant(sc, net, pipe, va)
    out["variant"] = variant.describe()
    out["t_validation_s"] = time.perf_counter() - t1
    say(f"validation: {out['validation']}")
    say(f"chosen variant: {variant.name}")
    del va
    t1 = time.perf_counter()
    te = fine_states(sc, test_seeds)
    out["t_test_spinup_s"] = time.perf_counter() - t1
    out["a_priori_corr"] = a_priori_correlation(net, pipe, te[: min(4, len(te))])
    say(f"a-priori correlation {out['a_priori_corr']:.3f}")
    out["evaluation"] = evaluate(sc, net, pipe, te)
    ev = out["evaluation"]
    say(f"closure: {dict((k, v) for k, v in ev['closure'].items() if k not in ('spectrum', 'flux'))}")
    say(f"no closure: {dict((k, v) for k, v in ev['no_closure'].items() if k not in ('spectrum', 'flux'))}")
    say(f"wall DNS {ev['dns_wall_s']:.3f} s / closure {ev['les_wall_s']:.4f} s = {ev['wall_ratio']:.1f}x; "
        f"accepted={ev['accepted']}")
    out["total_s"] = time.perf_counter() - t0
    out["net"] = net
    return out


def kernel_demo(n: int = 256, batch_tiles: int = 512, steps: int = 3) -> dict[str, float]:
    """A few launches of every closure kernel on random data (the small case the kernel
    profiles are captured on): training steps at a full batch, field inferences, and coarse
    closure steps in both update modes."""
    import torch

    rng = np.random.default_rng(0)
    net = ClosureNet(n, 4)
    net.load_bank(rng.normal(size=(4, 4, n, n)).astype(np.float32))
    net.set_params(init_params(0))
    net.fit_scales()
    net.set_adam(total_steps=max(steps, 1), warmup=0)
    losses = net.train(steps, batch_tiles=batch_tiles)
    f = torch.from_numpy(rng.normal(size=(3, n, n)).astype(np.float32)).to(net.device)
    for _ in range(steps):
        net.infer(f)
    cfg = forced_config(StudyConfig(), n, 5e-6)
    for every in (False, True):
        s = ClosureSolver(cfg, net, every_stage=every)
        s.set_state(random_phase_2d(n, k0=8.0, seed=1, energy=5e-3))
        for _ in range(steps):
            s.step(1e-3)
        s.synchronize()
    torch.cuda.synchronize()
    return {"loss_last": float(losses[-1]) if len(losses) else float("nan")}


def main(argv: list[str] | None = None) -> int:
    import argparse
    import sys

    ap = argparse.ArgumentParser(description="learned-closure study (data, training, a-posteriori test)")
    ap.add_argument("--small", action="store_true", help="the reduced configuration")
    ap.add_argument("--out", default=None, help="JSON report path")
    ap.add_argument("--save-net", default=None, help="npz path for the trained network")
    ap.add_argument("--set", nargs="*", default=[], help="StudyConfig overrides key=value")
    ap.add_argument("--kernels", action="store_true",
                    help="only launch every closure kernel a few times on random data")
    a = ap.parse_args(argv)
    if a.kernels:
        print(json.dumps(kernel_demo()))
        return 0
    sc = StudyConfig.small() if a.small else StudyConfig()
    for kv in a.set:
        key, val = kv.split("=", 1)
        typ = type(getattr(sc, key))
        if typ is bool:
            setattr(sc, key, val.lower() in ("1", "true", "yes"))
        elif typ is tuple:
            setattr(sc, key, tuple(float(x) for x in val.split(",") if x))
        else:
            setattr(sc, key, typ(val))
    res = run_study(sc, log=sys.stdout)
    net = res.pop("net")
    if a.save_net:
        net.save(a.save_net)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
