#!/usr/bin/env python
"""Benchmark of the IF-RK4 pseudo-spectral step on B200 (one JSON line on stdout, rank 0).

Default workload (``decay2d-8192-fp32``): 2D decaying turbulence on 8192^2 in fp32 — random-
phase vorticity (seed 0, k0 = 12, E = 0.5, E(k) ~ k^4 exp(-2 (k/k0)^2)), nu = 2e-6, 2/3
dealiasing, CFL 0.5 with dt re-evaluated every 10 steps, as ``simulate.run`` does.  A step is
one IF-RK4 step (4 stages x [C2R, phys, R2C, post]) of that run; the CFL reductions every 10
steps are inside the timed region.  Synthetic data only; every field (268 MB) is larger than
L2 (126 MB), so no L2 flush is needed between steps.

Reported beside the throughput (Mpts/s = n^2 / t_step):
  * pct_fft_roofline — the reference's roofline (src/pyspectral/benchmark.py:413-443):
    (4 t_fft_stage + pointwise_bytes / B_copy) / t_step, with t_fft_stage the faster of the
    standalone batched C2R+R2C of one stage through this library's cuFFT plans (in place) and
    through torch.fft (out of place), both measured here, and B_copy the copy bandwidth
    measured here;
  * roofline — the engine's dominant own kernel against the measured HBM peak;
  * cpu_baseline — the fp64/fp32 NumPy/SciPy oracle timed on this host's cores;
  * e2e — the same run through the public API from a host state to a host state.

``--impl reference`` times the reference algorithm's CPU implementation (the oracle port of
pyspectral's NumpySolver) on the same workload instead, on rank 0 only.
"""

from __future__ import annotations

import argparse
import gc
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

WORKLOADS = {
    # the decaying-turbulence headline: 8192^2 fp32, CFL 0.5, 200 steps in the full run
    "decay2d-8192-fp32": dict(n=8192, dim=2, dtype="float32", nu=2e-6, form="basdevant",
                              ic="random_phase", k0=12.0, seed=0, energy=0.5, cfl=0.5),
    # the same flow on 4096^2 (profiling captures that must stay small)
    "decay2d-4096-fp32": dict(n=4096, dim=2, dtype="float32", nu=8e-6, form="basdevant",
                              ic="random_phase", k0=12.0, seed=0, energy=0.5, cfl=0.5),
    # plain 2D Taylor-Green: 256^2 fp64, nu=1e-2, fixed dt=1e-3
    "tgv2d-256-fp64": dict(n=256, dim=2, dtype="float64", nu=1e-2, form="basdevant",
                           ic="tgv2d", dt=1e-3),
    # 3D Taylor-Green Re=1600, 512^3 fp32, CFL 0.5
    "tgv3d-512-fp32-rotational": dict(n=512, dim=3, dtype="float32", nu=1 / 1600,
                                      form="rotational", ic="tgv3d", cfl=0.5),
    "tgv3d-512-fp32-basdevant": dict(n=512, dim=3, dtype="float32", nu=1 / 1600,
                                     form="basdevant", ic="tgv3d", cfl=0.5),
    # the same flow on 256^3 (profiling captures that must stay small; > 0.7 GB per stage)
    "tgv3d-256-fp32-basdevant": dict(n=256, dim=3, dtype="float32", nu=1 / 1600,
                                     form="basdevant", ic="tgv3d", cfl=0.5),
    # the same flow on 1024^3 with the lean-memory engine (per-field plans), a few steps
    "tgv3d-1024-fp32-lean": dict(n=1024, dim=3, dtype="float32", nu=1 / 1600,
                                 form="rotational", ic="tgv3d", cfl=0.5, big=True),
    # 256 forced runs of uneven size advanced together: 64 each at 128^2 .. 1024^2, fp32
    "ensemble-4x64-fp32": dict(ensemble=True, sizes=(128, 256, 512, 1024), per_size=64,
                               dtype="float32", dim=2, form="basdevant", k0=8.0, power=1e-3,
                               klo=10.0, khi=12.0, alpha=0.1, alpha_kmax=2.0, cfl=0.5),
    # learned-closure 256^2 LES against 2048^2 forced DNS (data, training, a-posteriori test)
    "closure-les-256": dict(closure=True, n=256, n_fine=2048, dtype="float32", dim=2),
}
PUBLISHED_MPTS = {"decay2d-8192-fp32": 547.0}  # reference, RTX 3070 Laptop, fused-inplace
FALLBACK_HBM_GBS = 6650.0


# ----------------------------------------------------------------------------- helpers
def dist_env() -> tuple[int, int, int]:
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


class Replicas:
    """Plumbing of ``--gpus N``: one process per GPU, each running its own replica of the
    workload (the step does not shard).  The only collectives are a barrier around the timed
    region and the max of the per-rank times; ``nccl`` on the GPU box, ``gloo`` in CPU tests."""

    def __init__(self, backend: str = "nccl", device: object = None) -> None:
        self.rank, self.world, self.local = dist_env()
        self.pg = None
        self.device = device
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            kw = {"device_id": device} if backend == "nccl" and device is not None else {}
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300), **kw)
            self.pg = dist

    def barrier(self) -> None:
        if self.pg is not None:
            self.pg.barrier()

    def max(self, x: float) -> float:
        """Max of a float over all ranks (every rank calls it, in the same order)."""
        if self.pg is None:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64,
                         device=self.device if self.device is not None else "cpu")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        if self.pg is not None:
            self.pg.destroy_process_group()
            self.pg = None


def aggregate_mpts(world: int, points_per_replica: float, seconds_per_step: float) -> float:
    """Whole-job throughput: every replica advances its own grid in the (max) step time."""
    return world * points_per_replica / seconds_per_step / 1e6


def make_config(w: dict):
    from pyspectral_b200 import Config

    return Config(n=w["n"], dim=w["dim"], nu=w["nu"], dtype=w["dtype"], form=w["form"])


def make_ic(w: dict):
    from pyspectral_b200 import initial

    if w["ic"] == "random_phase":
        return initial.random_phase_2d(w["n"], k0=w["k0"], seed=w["seed"], energy=w["energy"])
    if w["ic"] == "tgv2d":
        return initial.to_spectral(initial.taylor_green_2d(w["n"]), 2)
    return initial.to_spectral(initial.taylor_green_3d(w["n"]), 3)


def traffic_model(n: int, dim: int, form: str, dtype: str) -> dict:
    """Minimal bytes per step (src/pyspectral/benchmark.py:43-55): every FFT reads and writes
    its data once, phys reads/writes each physical field once, the spectral kernel reads the
    transformed products, state and accumulator and writes accumulator/state and next inputs."""
    from pyspectral_b200.config import fft_split

    sr = 8 if dtype == "float64" else 4
    sc = 2 * sr
    npts = float(n) ** dim
    nmodes = float(n) ** (dim - 1) * (n // 2 + 1)
    ni, nf = fft_split(dim, form)
    ncomp = 1 if dim == 2 else 3
    fft = 4 * (ni + nf) * (nmodes * sc + npts * sr)
    phys = 4 * (ni + nf) * npts * sr
    post = (4 * (nf + ncomp + ni) + 7 * ncomp) * nmodes * sc
    return {"fft_bytes": fft, "pointwise_bytes": phys + post, "total_bytes": fft + phys + post,
            "points": npts, "modes": nmodes, "ffts_per_step": 4 * (ni + nf)}


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:  # noqa: BLE001
            pass
    return {}


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples every 200 ms while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int) -> None:
        self.index = index
        self.proc = None
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self) -> None:
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:  # noqa: BLE001
            self.proc = None

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:  # noqa: BLE001
            self.proc.kill()
        self.file.flush()
        rows = [r.split(",") for r in Path(self.file.name).read_text().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
                power.append(float(r[3]))
            except ValueError:
                continue
            for name, flag in zip(names, r[5:9], strict=False):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "power_w_max": max(power), "samples": len(sm), "reasons": sorted(reasons)}


def event_time_ms(fn, reps: int) -> float:
    """Median CUDA-event time of fn() on the current stream."""
    import torch

    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.median(ts)


def copy_bandwidth_gbs(nbytes: int = 1 << 30) -> float:
    """Device copy bandwidth (read + write counted), best of 10 (benchmark.py:99-116)."""
    import torch

    a = torch.empty(nbytes // 4, dtype=torch.float32, device="cuda")
    b = torch.empty_like(a)
    for _ in range(3):
        b.copy_(a)
    best = min(event_time_ms(lambda: b.copy_(a), 1) for _ in range(10))
    del a, b
    torch.cuda.empty_cache()
    return 2 * nbytes / (best * 1e-3) / 1e9


def tgv3d_device(n: int, dtype) -> "torch.Tensor":  # noqa: F821
    """The 3D Taylor-Green state built on the device: its only modes are (+-1, +-1, +-1), whose
    coefficients are those of the 8^3 transform scaled by (n/8)^3 (no n^3 host arrays)."""
    import torch

    from pyspectral_b200 import initial

    small = initial.to_spectral(initial.taylor_green_3d(8), 3) * (n / 8.0) ** 3
    out = torch.zeros((3, n, n, n // 2 + 1), dtype=dtype, device="cuda")
    for i in (1, 7):
        for j in (1, 7):
            out[:, i if i == 1 else n - 1, j if j == 1 else n - 1, 1] = torch.from_numpy(
                small[:, i, j, 1]).to(dtype).to(out.device)
    return out


def ours_big3d(args, w: dict) -> int:
    """A 3D grid too large for the usual set of solvers side by side (1024^3): one lean solver
    is timed, then its phases; the e2e pass reuses it (host state in and out) when the host has
    the memory; the one-step error against the fp64 lean engine is computed on the device with
    the fp32 solver freed first."""
    import psutil
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    comm = Replicas("nccl", torch.device("cuda", local))
    barrier, max_over_ranks = comm.barrier, comm.max

    from pyspectral_b200 import _lib
    from pyspectral_b200.registry import make_solver

    variant = "b200/fused-inplace-lean"
    cfg = make_config(w)
    n = w["n"]
    ic = tgv3d_device(n, torch.complex64)
    s = make_solver(variant, cfg)
    s.set_state(ic)
    run_workload(s, w, args.warmup)
    torch.cuda.synchronize()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = s.kernel_launches
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    run_workload(s, w, args.steps)
    ev1.record()
    ev1.synchronize()
    barrier()
    clk = clocks.stop()
    launches = s.kernel_launches - l0
    ms_step = max_over_ranks(ev0.elapsed_time(ev1)) / args.steps
    npts = float(n) ** 3
    value = aggregate_mpts(world, npts, ms_step * 1e-3)

    # per-phase device times of a middle stage (state garbage afterwards)
    t_fft = event_time_ms(lambda: (s.run_phase(0), s.run_phase(2)), 5)
    t_phys = event_time_ms(lambda: s.run_phase(1), 5)
    t_post = event_time_ms(lambda: s.run_phase(3, 1), 5)
    tm = traffic_model(n, 3, w["form"], w["dtype"])
    bcopy = copy_bandwidth_gbs()
    t_roof_ms = 4 * t_fft + tm["pointwise_bytes"] / (bcopy * 1e9) * 1e3
    ninv, nfwd, nmodes = s.n_inv, s.n_fwd, tm["modes"]
    post_bytes = (nfwd + 2 * 3 + 3 + ninv) * nmodes * 8
    phys_bytes = (ninv + nfwd) * nmodes * 8
    kernels = {"k_post3d<stage 1>": (t_post, post_bytes), "k_phys": (t_phys, phys_bytes)}
    kname = max(kernels, key=lambda k: kernels[k][0])
    k_ms, k_bytes = kernels[kname]
    hbm = measured_peaks().get("hbm_gbs")
    achieved = k_bytes / (k_ms * 1e-3) / 1e9

    # end to end through the public API on the same solver, if the host can hold the state
    state_bytes = s.u0.nbytes
    solver_bytes = sum(t.nbytes for t in (s.u0, s.acc, s.W, s.aux))
    e2e = None
    if psutil.virtual_memory().available > 8 * state_bytes:
        host_ic = ic.cpu().numpy()
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        s.set_state(host_ic)
        run_workload(s, w, args.steps)
        out = s.get_state()
        e2e_s = max_over_ranks(time.perf_counter() - t0)
        del out, host_ic
        e2e = {"value": world * npts * args.steps / e2e_s / 1e6, "unit": "Mpts/s",
               "h2d_bytes_per_step": state_bytes / args.steps,
               "d2h_bytes_per_step": state_bytes / args.steps,
               "what": "set_state(host) + K steps + get_state(host), wall clock"}
    else:
        e2e = {"value": None, "unit": "Mpts/s", "h2d_bytes_per_step": state_bytes / args.steps,
               "d2h_bytes_per_step": state_bytes / args.steps,
               "what": "skipped: host memory below 8x the state"}

    # one CFL step against the fp64 lean engine, compared on the device
    s.set_state(ic)
    h = min(0.05, w["cfl"] * (2 * math.pi / n) / s.diag.max_velocity_sum(s.state_native()))
    s.step(h)
    ua = s.state_native().clone()
    del s
    ic = None
    gc.collect()  # the solver's diagnostics refer back to it
    torch.cuda.empty_cache()
    rel_err = None
    try:  # the fp64 lean engine at 1024^3 holds about 100 GB more
        b = make_solver(variant, cfg.with_(dtype="float64"))
        b.set_state(tgv3d_device(n, torch.complex128))
        b.step(h)
        ub = b.state_native()
        num = max(float((ua[c].to(torch.complex128) - ub[c]).abs().max()) for c in range(3))
        rel_err = num / float(ub.abs().max())
        del b, ub
    except (torch.OutOfMemoryError, _lib.EngineError) as e:  # reported, not fatal: the
        # timed numbers stand (an EngineError is e.g. cuFFT failing to plan for lack of memory)
        print(f"one-step fp64 check skipped: {type(e).__name__}: {e}", file=sys.stderr)
    del ua
    gc.collect()
    torch.cuda.empty_cache()

    line = {
        "metric": "Mpts/s/RK4 step", "value": value, "unit": "Mpts/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": args.workload, "n": n, "dim": 3, "form": w["form"],
                   "nu": w["nu"], "variant": variant, "cfl": w["cfl"],
                   "parallelism": "replicas" if world > 1 else "single", "l2": l2_note(w)},
        "pct_fft_roofline": 100.0 * t_roof_ms / ms_step,
        "fft_roofline": {"t_fft_stage_ms": t_fft, "t_fft_stage_ms_own_plans": t_fft,
                         "t_fft_stage_ms_torch_fft": None,
                         "note": "own per-field plans only (torch.fft at 1024^3 not run)",
                         "t_roofline_step_ms": t_roof_ms, "copy_bw_gbs": bcopy,
                         "pointwise_bytes": tm["pointwise_bytes"],
                         "model_bytes_per_step": tm["total_bytes"],
                         "own_kernels_ms": {k: v[0] for k, v in kernels.items()}},
        "roofline": {"kernel": kname, "bound": "hbm", "achieved": achieved,
                     "peak": hbm or FALLBACK_HBM_GBS, "unit": "GB/s",
                     "frac": achieved / (hbm or FALLBACK_HBM_GBS),
                     "peak_source": "measured" if hbm else "fallback",
                     "algorithmic_bytes_per_launch": k_bytes, "traffic": None},
        "e2e": e2e, "rel_err_one_step_vs_fp64": rel_err, "gpu_launches": launches,
        "clocks": clk,
        "memory_gb": {"fp32_solver_buffers": solver_bytes / 1e9},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    comm.close()
    return 0


def run_workload(s, w: dict, nsteps: int) -> None:
    from pyspectral_b200.simulate import run_steps

    if "dt" in w:
        s.advance(nsteps, w["dt"])
    else:
        run_steps(s, nsteps, cfl=w["cfl"], dt_max=0.05, cfl_every=10)


def fused3d_pass_bytes(n: int, form: str, dtype: str) -> dict:
    """Algorithmic bytes of one launch of each fused 3D pass at a middle RK stage: every
    work-array element a pass reads or writes once (kept modes only), plus the compact state
    and accumulator of the X pass (read the state and accumulator, write the accumulator)."""
    sc = 16 if dtype == "float64" else 8  # one complex
    pr = 2 * sc                           # one Pair (two kz columns)
    km = (n - 1) // 3
    kz, kk = km + 1, 2 * km + 1
    nq = (kz + 3) // 4 * 2  # kz pairs per row, padded to an even count
    nin, nfw = (6, 3) if form == "rotational" else (3, 5)
    return {
        "k3_yinv": n * nin * nq * (kk + n) * pr,
        "k3_z": n * n * (nin + nfw) * kz * sc,
        "k3_yfwd": n * nfw * nq * (n + kk) * pr,
        "k3_x<stage 1>": kk * nq * (nfw + nin) * n * pr + 3 * 3 * kk * kz * kk * sc,
    }


def secondary_line(wname: str, steps: int, warmup: int, local: int,
                   variant: str = "b200/fused-fft-graph") -> dict:
    """A second workload measured inside the same bench run (its own solver, CUDA-event time
    over ``steps`` steps after ``warmup``, its own clock samples): ms/step, Mpts/s, the
    reference's FFT roofline, the roofline of the engine's dominant own kernel, the error of
    one step against the fp64 cuFFT engine, and the cuFFT engine's own ms/step on the same
    workload.  Used for the 512^3 3D Taylor-Green line beside the 2D headline."""
    import torch

    from pyspectral_b200.config import fft_split
    from pyspectral_b200.registry import make_solver

    w = WORKLOADS[wname]
    n, dim = w["n"], w["dim"]
    cfg = make_config(w)
    fused = "fused-fft" in variant

    def timed(v: str, with_clocks: bool):
        sv = make_solver(v, cfg)
        sv.set_state(tgv3d_device(n, torch.complex64) if w["ic"] == "tgv3d" else make_ic(w))
        run_workload(sv, w, warmup)
        torch.cuda.synchronize()
        clocks = ClockSampler(local) if with_clocks else None
        if clocks:
            clocks.start()
        l0 = sv.kernel_launches
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        run_workload(sv, w, steps)
        e1.record()
        e1.synchronize()
        clk = clocks.stop() if clocks else None
        return sv, e0.elapsed_time(e1) / steps, sv.kernel_launches - l0, clk

    s, ms_step, launches, clk = timed(variant, True)
    tm = traffic_model(n, dim, w["form"], w["dtype"])
    sc = 16 if w["dtype"] == "float64" else 8
    ncomp = 1 if dim == 2 else 3
    if fused:
        pb = fused3d_pass_bytes(n, w["form"], w["dtype"])
        kernels = {name: (event_time_ms(lambda ph=ph: s.run_phase(ph, 1), 10), pb[name])
                   for ph, name in enumerate(pb)}
    else:
        t_post = event_time_ms(lambda: s.run_phase(3, 1), 10)
        post_bytes = (s.n_fwd + 2 * ncomp + ncomp + s.n_inv) * tm["modes"] * sc
        kernels = {"k_post3d<stage 1>" if dim == 3 else "k_post2d<stage 1>": (t_post, post_bytes)}
    # the reference's FFT ceiling: the cuFFT engine's standalone stage transforms
    cf, cufft_ms, _, _ = (s, ms_step, 0, None) if not fused else timed("b200/fused-inplace-graph", False)

    def fft_stage() -> None:
        cf.run_phase(0)
        cf.run_phase(2)

    t_fft_own = event_time_ms(fft_stage, 10)
    del cf
    t_fft_torch = torch_fft_stage_ms(w, *fft_split(dim, w["form"]))
    t_fft = min(t_fft_own, t_fft_torch)
    bcopy = copy_bandwidth_gbs()
    t_roof = 4 * t_fft + tm["pointwise_bytes"] / (bcopy * 1e9) * 1e3
    peak = measured_peaks().get("hbm_gbs")
    kname = max(kernels, key=lambda k: kernels[k][0])
    k_ms, k_bytes = kernels[kname]
    achieved = k_bytes / (k_ms * 1e-3) / 1e9
    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        try:
            traffic = json.loads(tf.read_text()).get(wname, {}).get(kname)
        except Exception:  # noqa: BLE001
            traffic = None
    # one step against the fp64 cuFFT engine from the same state
    ic = tgv3d_device(n, torch.complex64) if w["ic"] == "tgv3d" else make_ic(w)
    s.set_state(ic)
    h = w.get("dt") or min(0.05, w["cfl"] * (2 * math.pi / n)
                           / s.diag.max_velocity_sum(s.state_native()))
    s.step(h)
    ua = s.state_native().clone()
    del s, ic
    gc.collect()
    torch.cuda.empty_cache()
    rel_err = None
    try:
        b = make_solver("b200/fused-inplace-graph", cfg.with_(dtype="float64"))
        b.set_state(tgv3d_device(n, torch.complex128) if w["ic"] == "tgv3d" else make_ic(w))
        b.step(h)
        ub = b.state_native()
        rel_err = float((ua.to(ub.dtype) - ub).abs().max()) / float(ub.abs().max())
        del b, ub
    except Exception as e:  # noqa: BLE001  (reported; the timed numbers stand)
        print(f"secondary fp64 check skipped: {type(e).__name__}: {e}", file=sys.stderr)
    del ua
    gc.collect()
    torch.cuda.empty_cache()
    return {
        "workload": wname, "variant": variant, "n": n, "dim": dim, "form": w["form"],
        "dtype": "f32" if w["dtype"] == "float32" else "f64", "steps": steps, "warmup": warmup,
        "ms_per_step": ms_step, "value": float(n) ** dim / (ms_step * 1e-3) / 1e6,
        "unit": "Mpts/s", "pct_fft_roofline": 100.0 * t_roof / ms_step,
        "cufft_engine_ms_per_step": cufft_ms,
        "fft_roofline": {"t_fft_stage_ms": t_fft, "t_fft_stage_ms_own_plans": t_fft_own,
                         "t_fft_stage_ms_torch_fft": t_fft_torch, "t_roofline_step_ms": t_roof,
                         "copy_bw_gbs": bcopy, "pointwise_bytes": tm["pointwise_bytes"]},
        "own_kernels_ms": {k: v[0] for k, v in kernels.items()},
        "roofline": {"kernel": kname, "bound": "hbm", "achieved": achieved,
                     "peak": peak or FALLBACK_HBM_GBS, "unit": "GB/s",
                     "frac": achieved / (peak or FALLBACK_HBM_GBS),
                     "peak_source": "measured" if peak else "fallback",
                     "algorithmic_bytes_per_launch": k_bytes, "traffic": traffic},
        "rel_err_one_step_vs_fp64": rel_err, "gpu_launches": launches, "clocks": clk,
    }


# ----------------------------------------------------------------------------- ensemble
def ensemble_members(w: dict) -> list:
    """The ensemble workload: run i (seed i) of each size class, nu from k_max eta = 1."""
    from pyspectral_b200 import Config
    from pyspectral_b200.ensemble import nu_for_kmax_eta

    kf = 0.5 * (w["klo"] + w["khi"])
    out = []
    for n in w["sizes"]:
        for _ in range(w["per_size"]):
            out.append(Config(n=n, dim=2, nu=nu_for_kmax_eta(n, w["power"], kf),
                              alpha=w["alpha"], alpha_kmax=w["alpha_kmax"],
                              force_klo=w["klo"], force_khi=w["khi"], dtype=w["dtype"]))
    return out


def ensemble_ics(w: dict, members: list) -> list:
    from pyspectral_b200 import initial

    return [initial.random_phase_2d(c.n, k0=w["k0"], seed=i % w["per_size"], energy=0.5)
            for i, c in enumerate(members)]


def time_oracle_ensemble(w: dict) -> dict:
    """One member per size class on the host (oracle port), scaled to the whole ensemble."""
    from oracle.numpy_oracle import OracleSolver
    from pyspectral_b200.ensemble import nu_for_kmax_eta

    total_s, pts = 0.0, 0.0
    kf = 0.5 * (w["klo"] + w["khi"])
    for n in w["sizes"]:
        from pyspectral_b200 import initial

        s = OracleSolver(n, 2, nu=nu_for_kmax_eta(n, w["power"], kf), alpha=w["alpha"],
                         alpha_kmax=w["alpha_kmax"], force_amp=0.1, force_klo=w["klo"],
                         force_khi=w["khi"], dtype=w["dtype"])
        s.set_state(initial.random_phase_2d(n, k0=w["k0"], seed=0))
        s.step(1e-4)
        t0 = time.perf_counter()
        for _ in range(2):
            s.step(1e-4)
        total_s += w["per_size"] * (time.perf_counter() - t0) / 2
        pts += w["per_size"] * float(n) ** 2
    return {"sec_per_step": total_s, "mpts": pts / total_s / 1e6, "cores": os.cpu_count() or 1}


L2_BYTES = 126 * 2**20


def l2_note(w: dict) -> str:
    """Whether the bytes a step moves (traffic model) exceed L2 (then no flush between steps)."""
    tb = traffic_model(w["n"], w["dim"], w["form"], w["dtype"])["total_bytes"]
    fb = (w["n"] ** w["dim"]) * (8 if w["dtype"] == "float64" else 4)
    if tb / 4 > L2_BYTES:  # every RK stage alone streams more than L2 holds
        return (f"inputs larger than L2 ({fb / 1e6:.0f} MB per field, {tb / 4e9:.2f} GB per "
                f"stage), no flush")
    return (f"working set fits in L2 ({tb / 4e6:.1f} MB per stage), not flushed between steps "
            f"(a parity case, not a headline number)")


def torch_fft_stage_ms(w: dict, ninv: int, nfwd: int) -> float:
    """One stage's batched inverse + forward transforms through torch.fft, out of place (the
    second standalone FFT ceiling: the roofline uses the faster of this and the own plans)."""
    import torch

    cdt = torch.complex64 if w["dtype"] == "float32" else torch.complex128
    rdt = torch.float32 if w["dtype"] == "float32" else torch.float64
    n, dim = w["n"], w["dim"]
    phys = (n,) * dim
    spec = (n,) * (dim - 1) + (n // 2 + 1,)
    axes = tuple(range(-dim, 0))
    qi = torch.zeros((ninv,) + spec, dtype=cdt, device="cuda")
    ri = torch.empty((ninv,) + phys, dtype=rdt, device="cuda")
    rf = torch.zeros((nfwd,) + phys, dtype=rdt, device="cuda")
    qf = torch.empty((nfwd,) + spec, dtype=cdt, device="cuda")

    def stage() -> None:
        torch.fft.irfftn(qi, s=phys, dim=axes, out=ri)
        torch.fft.rfftn(rf, dim=axes, out=qf)

    for _ in range(3):
        stage()
    t = event_time_ms(stage, 15)
    del qi, ri, rf, qf
    torch.cuda.empty_cache()
    return t


def ensemble_fft_stage_ms(w: dict, counts: dict | None = None) -> float:
    """Standalone batched cuFFT time of one RK stage for every class (2 C2R + 2 R2C per member,
    batched over the class, through torch.fft), summed over the classes; ``counts`` = members
    per size (default: the workload's)."""
    import torch

    cdt = torch.complex64 if w["dtype"] == "float32" else torch.complex128
    rdt = torch.float32 if w["dtype"] == "float32" else torch.float64
    tot = 0.0
    for n in w["sizes"]:
        m = w["per_size"] if counts is None else counts.get(n, 0)
        if m == 0:
            continue
        b = 2 * m
        q = torch.zeros((b, n, n // 2 + 1), dtype=cdt, device="cuda")
        r = torch.zeros((b, n, n), dtype=rdt, device="cuda")

        def stage() -> None:
            torch.fft.irfftn(q, s=(n, n), dim=(-2, -1), out=r)
            torch.fft.rfftn(r, dim=(-2, -1), out=q)

        for _ in range(3):
            stage()
        tot += event_time_ms(stage, 10)
        del q, r
    torch.cuda.empty_cache()
    return tot


def ours_ensemble(args, w: dict) -> int:
    """The ensemble workload.  Under torchrun the members are partitioned over the ranks by
    balanced grid points (sharding.partition_by_points) and each GPU advances its share: the
    value is all members' points over the slowest rank's step time (scaling "strong")."""
    import torch

    from pyspectral_b200.sharding import Comm, ShardedEnsemble

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    comm = Replicas("nccl", dev)
    members = ensemble_members(w)
    ics = ensemble_ics(w, members)
    se = ShardedEnsemble(members, comm=Comm(dev))
    ens = se.ens
    counts = {n: sum(1 for i in se.local if members[i].n == n) for n in w["sizes"]}
    se.set_states(ics)
    se.run_steps(args.warmup, cfl=w["cfl"], target_power=w["power"])
    torch.cuda.synchronize()
    comm.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = ens.kernel_launches if ens is not None else 0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    se.run_steps(args.steps, cfl=w["cfl"], target_power=w["power"])
    ev1.record()
    ev1.synchronize()
    comm.barrier()
    clk = clocks.stop()
    launches = (ens.kernel_launches - l0) if ens is not None else 0
    ms_step = comm.max(ev0.elapsed_time(ev1)) / args.steps
    pts = sum(float(c.n) ** 2 for c in members)
    value = pts / (ms_step * 1e-3) / 1e6
    # end to end: host states in, K steps, host states out (this rank's members)
    e2 = ShardedEnsemble(members, comm=Comm(dev))
    e2.set_states(ics)
    torch.cuda.synchronize()
    comm.barrier()
    t0 = time.perf_counter()
    e2.set_states(ics)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    e2.run_steps(args.steps, cfl=w["cfl"], target_power=w["power"])
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    outs = e2.ens.get_states() if e2.ens is not None else []
    t3 = time.perf_counter()
    e2e_s = comm.max(t3 - t0)
    e2e_parts = {"set_states_s": comm.max(t1 - t0), "steps_s": comm.max(t2 - t1),
                 "get_states_s": comm.max(t3 - t2)}
    state_bytes = sum(c.u0.nbytes for c in e2.ens.classes) if e2.ens is not None else 0
    state_bytes = int(comm.max(float(state_bytes)) * world)
    del e2, outs
    torch.cuda.empty_cache()
    # FFT roofline of the reference's definition for this rank's members; the job's is the
    # slowest rank's
    t_fft_stage = ensemble_fft_stage_ms(w, counts)
    bcopy = copy_bandwidth_gbs()
    pw = sum(counts[n] * traffic_model(n, 2, "basdevant", w["dtype"])["pointwise_bytes"]
             for n in w["sizes"])
    t_roof = comm.max(4 * t_fft_stage + pw / (bcopy * 1e9) * 1e3)
    line = {
        "metric": "Mpts/s/RK4 step", "value": value, "unit": "Mpts/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "strong" if world > 1 else "weak",
        "vs_baseline": None,
        "dtype": "f32" if w["dtype"] == "float32" else "f64", "data": "synthetic",
        "config": {"workload": args.workload, "sizes": list(w["sizes"]),
                   "runs_per_size": w["per_size"], "members": len(members),
                   "forcing": f"constant power P={w['power']} on {w['klo']}<=|k|<={w['khi']}",
                   "drag": f"alpha={w['alpha']} on |k|<={w['alpha_kmax']}",
                   "nu": "k_max eta = 1 (nu_for_kmax_eta)", "cfl": w["cfl"],
                   "engine": ("work list: per RK stage one persistent row-pass and one "
                              f"column-pass launch over every class, {ens.worklist}-thread CTAs"
                              if ens is not None and ens.worklist else
                              "sp_batch per size class, one sp_group graph (a branch per class)"),
                   "tiles": {str(c.n): c.tile for c in ens.classes} if ens is not None else {},
                   "tile_source": "TileTuner (CUDA-event timing of each candidate, JSON cache)"
                   if ens is not None and ens.tuner is not None else "default",
                   "parallelism": (f"members partitioned over {world} ranks by grid points"
                                   if world > 1 else "single")},
        "pct_fft_roofline": 100.0 * t_roof / ms_step,
        "fft_roofline": {"t_roofline_step_ms": t_roof, "copy_bw_gbs": bcopy,
                         "t_fft_stage_ms_local_classes": t_fft_stage, "pointwise_bytes_local": pw},
        "e2e": {"value": pts * args.steps / e2e_s / 1e6, "unit": "Mpts/s",
                "h2d_bytes_per_step": state_bytes / args.steps,
                "d2h_bytes_per_step": state_bytes / args.steps,
                "what": "set_states(host) + K steps + get_states (every member), wall clock",
                "parts": e2e_parts},
        "gpu_launches": launches, "clocks": clk,
        "autotune": None if ens is None or ens.tuner is None else {
            k: dict(v) for k, v in ens.tuner.report.items()},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = time_oracle_ensemble(w)
        line["cpu_baseline"] = {"value": r["mpts"], "unit": "Mpts/s", "cores": r["cores"],
                                "kind": "port", **host_info(),
                                "sample": "2 IF-RK4 steps of one member per size class (oracle "
                                          "port, scipy.fft workers=-1), times 64 members"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    comm.close()
    return 0


def ensemble_secondary(wname: str, steps: int, warmup: int, local: int) -> dict:
    """The uneven-ensemble workload measured inside the default bench run on one GPU: the
    autotuned Ensemble stepped with per-member CFL dt and constant-power forcing, CUDA-event
    ms/step over ``steps`` steps after ``warmup``, its own clock samples, the aggregate FFT
    roofline (batched cuFFT of every class + pointwise bytes at the copy bandwidth) and the
    tuner's choices."""
    import torch

    from pyspectral_b200.ensemble import Ensemble

    w = WORKLOADS[wname]
    members = ensemble_members(w)
    ens = Ensemble(members)
    ens.set_states(ensemble_ics(w, members))
    ens.run_steps(warmup, cfl=w["cfl"], target_power=w["power"])
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = ens.kernel_launches
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    ens.run_steps(steps, cfl=w["cfl"], target_power=w["power"])
    ev1.record()
    ev1.synchronize()
    clk = clocks.stop()
    ms_step = ev0.elapsed_time(ev1) / steps
    launches = ens.kernel_launches - l0
    pts = sum(float(c.n) ** 2 for c in members)
    engine = ("work list" if ens.worklist else "per-class launches, one group graph")
    tiles = {str(c.n): c.tile for c in ens.classes}
    report = None if ens.tuner is None else {k: dict(v) for k, v in ens.tuner.report.items()}
    del ens
    gc.collect()
    torch.cuda.empty_cache()
    t_fft_stage = ensemble_fft_stage_ms(w)
    bcopy = copy_bandwidth_gbs()
    pw = sum(w["per_size"] * traffic_model(n, 2, "basdevant", w["dtype"])["pointwise_bytes"]
             for n in w["sizes"])
    t_roof = 4 * t_fft_stage + pw / (bcopy * 1e9) * 1e3
    return {
        "workload": wname, "sizes": list(w["sizes"]), "runs_per_size": w["per_size"],
        "dtype": "f32" if w["dtype"] == "float32" else "f64", "steps": steps, "warmup": warmup,
        "ms_per_step": ms_step, "value": pts / (ms_step * 1e-3) / 1e6, "unit": "Mpts/s",
        "pct_fft_roofline": 100.0 * t_roof / ms_step, "t_roofline_step_ms": t_roof,
        "engine": engine, "tiles": tiles, "autotune": report, "gpu_launches": launches,
        "clocks": clk,
    }


def ours_closure(args, w: dict) -> int:
    """The learned-closure workload: the whole study (batched 2048^2 DNS data, training,
    validation, a-posteriori test on held-out seeds) on one GPU; the headline is the wall-time
    speed-up of the 256^2 closure run over the 2048^2 DNS to the same end time, with the E(k)
    error against that DNS stated beside it."""
    import torch

    from pyspectral_b200 import closure_les as cl

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if rank != 0:
        return 0
    sc = cl.StudyConfig()
    clocks = ClockSampler(local)
    clocks.start()
    res = cl.run_study(sc)
    clk = clocks.stop()
    net = res.pop("net")
    ev = res["evaluation"]
    # the dominant closure kernel: one inference over the 256^2 field, CUDA events
    f = torch.randn(3, sc.n_coarse, sc.n_coarse, device="cuda")
    for _ in range(3):
        net.infer(f)
    reps = 50
    out = torch.empty(sc.n_coarse, sc.n_coarse, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st = torch.cuda.current_stream()
    torch.cuda.synchronize()
    e0.record(st)
    for _ in range(reps):
        net.infer(f, out, sync=False)
    e1.record(st)
    e1.synchronize()
    net.check()
    t_inf = e0.elapsed_time(e1) / reps
    flop = sc.n_coarse ** 2 * 2.0 * (75 * 64 + 64 * 64 + 64 * 64 + 64)
    peaks = measured_peaks()
    tflops = flop / (t_inf * 1e-3) / 1e12
    peak = peaks.get("bf16_tflops", 1590.0)
    les_ms = 1e3 * ev["les_wall_s"] / max(1, ev["les_steps"])
    cmp = ev["closure"]
    line = {
        "metric": "closure-LES speed-up over 2048^2 DNS to t_end (E(k) error stated)",
        "value": ev["wall_ratio"], "unit": "x", "n_gpus": 1, "steps": ev["les_steps"],
        "warmup": 1, "ms_per_step": les_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 flow, bf16 network (fp32 accumulation)",
        "data": "synthetic (seeded random-phase forced runs)",
        "config": {"workload": args.workload, "n_coarse": sc.n_coarse, "n_fine": sc.n_fine,
                   "nu": sc.nu, "forcing": f"P={sc.power} on {sc.force_klo}<=|k|<={sc.force_khi}",
                   "drag": f"alpha={sc.alpha} on |k|<={sc.alpha_kmax}", "t_end": sc.t_eval,
                   "snapshots": sc.snapshots, "train_steps": sc.train_steps,
                   "points_per_step": sc.batch_tiles * 128, "test_seeds": sc.test_seeds,
                   "closure_update": "every stage" if sc.every_stage else "first stage of each step"},
        "closure": {"e_err_max_k_le_85": cmp.get("e_err_max"), "e_err_mean": cmp.get("e_err_mean"),
                    "flux_err_l2": cmp.get("flux_err_l2"), "err_bound": sc.err_bound,
                    "accepted": ev["accepted"], "variant": res["variant"]["name"],
                    "no_closure_e_err_max": ev["no_closure"].get("e_err_max"),
                    "a_priori_corr": res["a_priori_corr"], "dns_wall_s": ev["dns_wall_s"],
                    "les_wall_s": ev["les_wall_s"], "dns_steps": ev["dns_steps"],
                    "train_ms_per_step": res["train"]["ms_per_step"],
                    "data_seconds": res["data"]["seconds"], "study_seconds": res["total_s"]},
        "roofline": {"bound": "tensor", "kernel": "k_infer (256^2, 3 tcgen05 layers)",
                     "achieved": tflops, "peak": peak, "unit": "TFLOP/s", "frac": tflops / peak,
                     "traffic": None, "flop_per_launch": flop, "launch_ms": t_inf},
        "e2e": {"value": ev["wall_ratio"], "unit": "x", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0,
                "what": "wall clock of simulate.run_device (CFL and constant-power control on "
                        "the device, one host read per 10 steps) to t_end for both runs"},
        "gpu_launches": int(net.kernel_launches), "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- CPU side
def time_oracle(w: dict, warmup: int, steps: int) -> dict:
    """The oracle port of the reference's NumpySolver on this host (all cores via
    scipy.fft workers=-1 for large grids): seconds per IF-RK4 step of the workload."""
    from oracle.numpy_oracle import OracleDiagnostics, OracleSolver

    ic = make_ic(w)
    s = OracleSolver(w["n"], w["dim"], nu=w["nu"], dtype=w["dtype"], form=w["form"])
    s.set_state(ic)
    if "dt" in w:
        dt = w["dt"]
    else:
        umax = OracleDiagnostics(w["n"], w["dim"]).max_velocity_sum(s.get_state())
        dt = min(0.05, w["cfl"] * (2 * math.pi / w["n"]) / umax)
    for _ in range(warmup):
        s.step(dt)
    t0 = time.perf_counter()
    for _ in range(steps):
        s.step(dt)
    sec = (time.perf_counter() - t0) / steps
    return {"sec_per_step": sec, "mpts": float(w["n"]) ** w["dim"] / sec / 1e6,
            "cores": os.cpu_count() or 1}


def host_info() -> dict:
    """The CPU model and the NumPy / SciPy versions the CPU baseline ran with."""
    import numpy
    import scipy

    model = None
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"cpu_model": model, "numpy": numpy.__version__, "scipy": scipy.__version__}


def reference_arm(args, w: dict) -> int:
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    warm = min(args.warmup, 1)
    steps = max(1, min(args.steps, 3))
    r = time_oracle(w, warm, steps)
    sample = (f"{steps} IF-RK4 step(s) of the {args.workload} workload after {warm} warm-up "
              f"step(s); NumPy + scipy.fft (pocketfft) with workers=-1 on {r['cores']} host "
              f"threads; oracle port of pyspectral NumpySolver")
    line = {
        "metric": "Mpts/s/RK4 step", "value": r["mpts"], "unit": "Mpts/s", "impl": "reference",
        "n_gpus": world, "steps": steps, "warmup": warm, "ms_per_step": r["sec_per_step"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if w["dtype"] == "float32" else "f64", "data": "synthetic",
        "config": {"workload": args.workload, "n": w["n"], "dim": w["dim"], "form": w["form"],
                   "nu": w["nu"], "l2": "inputs larger than L2"},
        "cpu_baseline": {"value": r["mpts"], "unit": "Mpts/s", "cores": r["cores"],
                         "kind": "port", **host_info(), "sample": sample},
        "e2e": {"value": r["mpts"], "unit": "Mpts/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- GPU side
def ours(args, w: dict) -> int:
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    comm = Replicas("nccl", torch.device("cuda", local))
    barrier, max_over_ranks = comm.barrier, comm.max

    from pyspectral_b200.registry import make_solver

    cfg = make_config(w)
    ic = make_ic(w)
    s = make_solver(args.variant, cfg)
    s.set_state(ic)
    run_workload(s, w, args.warmup)
    torch.cuda.synchronize()
    barrier()

    # ---- timed region: K steps of the run on device-resident state
    clocks = ClockSampler(local)
    clocks.start()
    l0 = s.kernel_launches
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    barrier()
    ev0.record()
    run_workload(s, w, args.steps)
    ev1.record()
    ev1.synchronize()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    launches = s.kernel_launches - l0
    t_ms = max_over_ranks(ev0.elapsed_time(ev1))
    ms_step = t_ms / args.steps
    npts = float(w["n"]) ** w["dim"]
    value = aggregate_mpts(world, npts, ms_step * 1e-3)

    # ---- end to end through the public API: host state in, K steps, host state out
    s2 = make_solver(args.variant, cfg)
    s2.set_state(ic)  # first load allocates the pinned staging buffer; not timed
    run_workload(s2, w, 1)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    s2.set_state(ic)
    run_workload(s2, w, args.steps)
    out = s2.get_state()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = world * npts * args.steps / e2e_s / 1e6
    state_bytes = s2.u0.nbytes
    cfl_reads = math.ceil(args.steps / 10) * 24 if "dt" not in w else 0
    del s2, out
    torch.cuda.empty_cache()

    # ---- error of one step against the fp64 engine (itself pinned to the fp64 oracle)
    rel_err = None
    if w["dtype"] == "float32":
        a = make_solver(args.variant, cfg)
        b = make_solver("b200/fused-inplace-graph", cfg.with_(dtype="float64"))
        a.set_state(ic)
        b.set_state(ic)
        h = w.get("dt") or min(0.05, w["cfl"] * (2 * math.pi / w["n"])
                               / b.diag.max_velocity_sum(b.state_native()))
        a.step(h)
        b.step(h)
        ra, rb = a.get_state(), b.get_state()
        rel_err = float(abs(ra - rb).max() / abs(rb).max())
        del a, b, ra, rb
        torch.cuda.empty_cache()

    # ---- per-phase device times (state garbage afterwards: nothing reads it).  The FFT
    # ceiling of the reference's roofline is always the batched cuFFT C2R + R2C of one stage.
    fused = "fused-fft" in args.variant
    cf = make_solver("b200/fused-inplace-graph", cfg) if fused else s
    if fused:
        cf.set_state(ic)
        cf.step(1e-6)

    def fft_stage() -> None:
        cf.run_phase(0)
        cf.run_phase(2)

    t_fft_own = event_time_ms(fft_stage, 15)
    sc = 16 if w["dtype"] == "float64" else 8
    ncomp = 1 if w["dim"] == 2 else 3
    tm = traffic_model(w["n"], w["dim"], w["form"], w["dtype"])
    if fused and w["dim"] == 3:
        pb = fused3d_pass_bytes(w["n"], w["form"], w["dtype"])
        kernels = {name: (event_time_ms(lambda ph=ph: s.run_phase(ph, 1), 15), pb[name])
                   for ph, name in enumerate(pb)}
        del cf
    elif fused:
        n = w["n"]
        kc = (n + 2) // 3
        kept_rows = 2 * ((n - 1) // 3) + 1
        t_row = event_time_ms(lambda: s.run_phase(0), 15)
        t_col = event_time_ms(lambda: s.run_phase(3, 1), 15)
        row_bytes = 2 * n * kc * 2 * sc          # read + write the (n x kc) pair array
        col_bytes = 2 * n * kc * 2 * sc + 3 * kept_rows * kc * sc  # + state, acc r/w
        # the streamed persistent column pass runs single runs of n = 2048..8192 (fp64 <= 4096)
        streamed = (bool(s.lib.sp_column_streaming()) and 2048 <= n
                    and n <= (4096 if w["dtype"] == "float64" else 8192))
        cname = "k_col_stream<stage 1>" if streamed else "k_col_pass<stage 1>"
        kernels = {"k_row_pass": (t_row, row_bytes), cname: (t_col, col_bytes)}
        del cf
    else:
        t_phys = event_time_ms(lambda: s.run_phase(1), 15)
        t_post = event_time_ms(lambda: s.run_phase(3, 1), 15)
        ninv, nfwd = s.n_inv, s.n_fwd
        # post kernel of a middle stage: reads nfwd products + state + accumulator, writes the
        # accumulator and the ninv next-stage inputs
        post_bytes = (nfwd + 2 * ncomp + ncomp + ninv) * tm["modes"] * sc
        phys_bytes = (ninv + nfwd) * tm["modes"] * sc  # padded real fields, read + write
        kernels = {("k_post2d<stage 1>" if w["dim"] == 2 else "k_post3d<stage 1>"):
                   (t_post, post_bytes), "k_phys": (t_phys, phys_bytes)}
    from pyspectral_b200.config import fft_split

    t_fft_torch = torch_fft_stage_ms(w, *fft_split(w["dim"], w["form"]))
    t_fft_stage = min(t_fft_own, t_fft_torch)  # the fastest standalone stage transforms
    bcopy = copy_bandwidth_gbs()
    t_roof_ms = 4 * t_fft_stage + tm["pointwise_bytes"] / (bcopy * 1e9) * 1e3
    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs")
    kname = max(kernels, key=lambda k: kernels[k][0])  # dominant own kernel
    k_ms, k_bytes = kernels[kname]
    achieved = k_bytes / (k_ms * 1e-3) / 1e9
    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        try:
            traffic = json.loads(tf.read_text()).get(args.workload, {}).get(kname)
        except Exception:  # noqa: BLE001
            traffic = None

    line = {
        "metric": "Mpts/s/RK4 step", "value": value, "unit": "Mpts/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak",
        "vs_baseline": (value / PUBLISHED_MPTS[args.workload]
                        if args.workload in PUBLISHED_MPTS and world == 1 else None),
        "dtype": "f32" if w["dtype"] == "float32" else "f64", "data": "synthetic",
        "config": {"workload": args.workload, "n": w["n"], "dim": w["dim"], "form": w["form"],
                   "nu": w["nu"], "variant": args.variant, "cfl": w.get("cfl"),
                   "dt": w.get("dt"), "parallelism": "replicas" if world > 1 else "single",
                   "l2": l2_note(w)},
        "pct_fft_roofline": 100.0 * t_roof_ms / ms_step,
        "fft_roofline": {"t_fft_stage_ms": t_fft_stage, "t_fft_stage_ms_own_plans": t_fft_own,
                         "t_fft_stage_ms_torch_fft": t_fft_torch,
                         "t_roofline_step_ms": t_roof_ms,
                         "copy_bw_gbs": bcopy, "pointwise_bytes": tm["pointwise_bytes"],
                         "model_bytes_per_step": tm["total_bytes"],
                         "effective_gbs": tm["total_bytes"] / (ms_step * 1e-3) / 1e9,
                         "own_kernels_ms": {k: v[0] for k, v in kernels.items()}},
        "roofline": {"kernel": kname, "bound": "hbm", "achieved": achieved,
                     "peak": hbm or FALLBACK_HBM_GBS, "unit": "GB/s",
                     "frac": achieved / (hbm or FALLBACK_HBM_GBS),
                     "peak_source": "measured" if hbm else "fallback",
                     "algorithmic_bytes_per_launch": k_bytes, "traffic": traffic},
        "e2e": {"value": e2e_value, "unit": "Mpts/s",
                "h2d_bytes_per_step": state_bytes / args.steps,
                "d2h_bytes_per_step": (state_bytes + cfl_reads) / args.steps,
                "what": "set_state(host) + K steps + get_state(host), wall clock"},
        "rel_err_one_step_vs_fp64": rel_err,
        "gpu_launches": launches,
        "clocks": clk,
    }
    if world == 1 and args.workload == "decay2d-8192-fp32" and not args.no_secondary:
        # the 3D Taylor-Green step at 512^3 beside the 2D headline, timed in the same run
        line["secondary"] = secondary_line("tgv3d-512-fp32-basdevant", 10, 3, local)
        # and the 256-member uneven ensemble (64 runs each of 128^2 .. 1024^2)
        line["secondary_ensemble"] = ensemble_secondary("ensemble-4x64-fp32", 20, 3, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = time_oracle(w, 1, 1)
        line["cpu_baseline"] = {
            "value": r["mpts"], "unit": "Mpts/s", "cores": r["cores"], "kind": "port", **host_info(),
            "sample": f"1 IF-RK4 step of {args.workload} after 1 warm-up step; oracle port of "
                      f"pyspectral NumpySolver, scipy.fft workers=-1"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    comm.close()
    return 0


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="decay2d-8192-fp32", choices=sorted(WORKLOADS))
    ap.add_argument("--variant", default="auto",
                    help="registry variant; auto = the fused-FFT engine where it runs (n a "
                         "power of two: 2D <= 8192 fp32 / 4096 fp64, 3D <= 512), else the "
                         "cuFFT graph engine")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the 512^3 3D line measured beside the default 2D workload")
    args = ap.parse_args(argv)
    if args.impl == "ours":
        args.warmup = max(args.warmup, 3)  # at least 3 untimed warm-up steps
    w = WORKLOADS[args.workload]
    if w.get("closure"):
        if args.impl == "reference":
            rank, _, _ = dist_env()
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable":
                                  "the reference has no learned closure (its path for this "
                                  "flow is the plain DNS, timed by the decay2d workloads)"}))
            return 0
        return ours_closure(args, w)
    if w.get("ensemble"):
        if args.impl == "reference":
            rank, _, _ = dist_env()
            if rank != 0:
                return 0
            r = time_oracle_ensemble(w)
            print(json.dumps({
                "metric": "Mpts/s/RK4 step", "value": r["mpts"], "unit": "Mpts/s",
                "impl": "reference", "n_gpus": 1, "steps": 2, "warmup": 1,
                "ms_per_step": r["sec_per_step"] * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": args.workload},
                "cpu_baseline": {"value": r["mpts"], "unit": "Mpts/s", "cores": r["cores"],
                                 "kind": "port", **host_info(), "sample": "one member per class, x64"},
                "e2e": {"value": r["mpts"], "unit": "Mpts/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}), flush=True)
            return 0
        return ours_ensemble(args, w)
    if w.get("big"):
        if args.impl == "reference":
            rank, _, _ = dist_env()
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable":
                                  "a 1024^3 step of the NumPy oracle needs about 100 GB of host "
                                  "memory and minutes per step; the 512^3 workloads carry the "
                                  "CPU baseline"}))
            return 0
        return ours_big3d(args, w)
    if args.variant == "auto":
        n = w["n"]
        pow2 = n & (n - 1) == 0 and 16 <= n
        fused_ok = pow2 and (n <= (8192 if w["dtype"] == "float32" else 4096) if w["dim"] == 2
                             else n <= 512)
        args.variant = "b200/fused-fft-graph" if fused_ok else "b200/fused-inplace-graph"
    if args.impl == "reference":
        return reference_arm(args, w)
    return ours(args, w)


if __name__ == "__main__":
    sys.exit(main())
