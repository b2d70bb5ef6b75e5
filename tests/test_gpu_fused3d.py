"""The fused 3D engine (hand-written FFT passes, no cuFFT) against the fp64 oracle and the cuFFT
engine: both forms, both precisions, forcing, drag, dt and amplitude changes mid-run (the
reference's parity protocol, tests/test_backends.py:24-47), the CFL bound and diagnostics, the
device run loop, and the 512^3 Taylor-Green step against fp64.  Tolerances as everywhere:
max|a - b| / max|b| <= 1e-12 (fp64), <= 5e-6 (fp32) against the fp64 oracle."""

from __future__ import annotations

import math

import numpy as np
import pytest

from oracle.numpy_oracle import OracleDiagnostics, OracleSolver
from pyspectral_b200 import Config, initial
from pyspectral_b200.registry import get

pytestmark = pytest.mark.gpu
FUSED = "b200/fused-fft-graph"
TOL = {"float64": 1e-12, "float32": 5e-6}


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def _cfg(n, form, dtype):
    return Config(n=n, dim=3, nu=0.01, alpha=0.5, alpha_kmax=2.0, force_amp=0.3, force_klo=1,
                  force_khi=2.5, dtype=dtype, form=form)


def _oracle(cfg):
    return OracleSolver(cfg.n, 3, nu=cfg.nu, alpha=cfg.alpha, alpha_kmax=cfg.alpha_kmax,
                        force_amp=cfg.force_amp, force_klo=cfg.force_klo,
                        force_khi=cfg.force_khi, form=cfg.resolved_form())


@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("form", ["basdevant", "rotational"])
@pytest.mark.parametrize("n", [16, 32, 64])
def test_fused3d_matches_oracle(n, form, dtype):
    cfg = _cfg(n, form, dtype)
    s = get(FUSED).make(cfg)
    ref = _oracle(cfg)
    ic = initial.to_spectral(initial.random_3d(n, k0=max(2.0, n / 12), seed=n), 3)
    s.set_state(ic)
    ref.set_state(ic)
    s.advance(3, 0.01)
    ref.advance(3, 0.01)
    s.set_forcing_amplitude(0.1)
    ref.set_forcing_amplitude(0.1)
    s.advance(2, 0.007)
    ref.advance(2, 0.007)
    assert rel(s.get_state(), ref.get_state()) < TOL[dtype]


@pytest.mark.parametrize("form", ["basdevant", "rotational"])
def test_fused3d_128_matches_oracle(form):
    cfg = _cfg(128, form, "float64")
    s = get(FUSED).make(cfg)
    ref = _oracle(cfg)
    ic = initial.to_spectral(initial.random_3d(128, k0=8.0, seed=3), 3)
    s.set_state(ic)
    ref.set_state(ic)
    s.step(4e-3)
    ref.step(4e-3)
    s.set_forcing_amplitude(0.1)
    ref.set_forcing_amplitude(0.1)
    s.step(3e-3)
    ref.step(3e-3)
    assert rel(s.get_state(), ref.get_state()) < 1e-12


@pytest.mark.parametrize("form", ["basdevant", "rotational"])
def test_fused3d_cfl_and_diagnostics_match_the_oracle(form):
    n = 32
    cfg = _cfg(n, form, "float64")
    s = get(FUSED).make(cfg)
    ic = initial.to_spectral(initial.random_3d(n, k0=3.0, seed=9), 3)
    s.set_state(ic)
    s.advance(2, 0.01)
    st = s.get_state()
    od = OracleDiagnostics(n, 3)
    d = s.diag
    assert d.max_velocity_sum(s.state_native()) == pytest.approx(od.max_velocity_sum(st),
                                                                 rel=1e-12)
    assert d.energy(s.state_native()) == pytest.approx(od.energy(st), rel=1e-12)
    assert d.enstrophy(s.state_native()) == pytest.approx(od.enstrophy(st), rel=1e-12)
    # stepping after the CFL evaluation is unaffected by it
    ref = _oracle(cfg)
    ref.set_state(st)
    s.step(0.01)
    ref.step(0.01)
    assert rel(s.get_state(), ref.get_state()) < 1e-12


def test_fused3d_one_graph_step_launches_sixteen_kernels():
    s = get(FUSED).make(_cfg(32, "rotational", "float32"))
    s.set_state(initial.to_spectral(initial.random_3d(32, k0=3.0), 3))
    s.step(1e-3)
    before = s.kernel_launches
    s.step(1e-3)
    assert s.kernel_launches - before == 16  # 4 stages x (y inverse, z, y forward, x)


@pytest.mark.parametrize("form", ["basdevant", "rotational"])
def test_fused3d_device_run_loop_matches_host_loop(form):
    """sp_run_to (CFL bound and constant power on the device) = simulate.run's rules."""
    from pyspectral_b200.simulate import run

    n = 32
    cfg = _cfg(n, form, "float64")
    ic = initial.to_spectral(initial.random_3d(n, k0=3.0, seed=2), 3)
    a, b = get(FUSED).make(cfg), get(FUSED).make(cfg)
    a.set_state(ic)
    b.set_state(ic)
    run(a, 0.3, cfl=0.5, target_power=0.05)
    b.run_to(0.3, cfl=0.5, target_power=0.05)
    assert b.nstep == a.nstep and b.t == pytest.approx(a.t, rel=1e-12)
    assert rel(b.get_state(), a.get_state()) < 1e-11


@pytest.mark.parametrize("form", ["basdevant", "rotational"])
def test_fused3d_tgv_512_fp32_one_step_vs_fp64(form):
    """The 512^3 Taylor-Green workload: one CFL step of the fused fp32 engine against the fp64
    cuFFT engine (pinned to the oracle at 1e-12) from the same state: <= 1e-5."""
    import torch

    n = 512
    cfg = Config(n=n, dim=3, nu=1 / 1600, dtype="float32", form=form)
    small = initial.to_spectral(initial.taylor_green_3d(8), 3) * (n / 8.0) ** 3
    ic = torch.zeros((3, n, n, n // 2 + 1), dtype=torch.complex128, device="cuda")
    for i in (1, 7):
        for j in (1, 7):
            ic[:, i if i == 1 else n - 1, j if j == 1 else n - 1, 1] = torch.from_numpy(
                small[:, i, j, 1]).to("cuda")
    f = get(FUSED).make(cfg)
    f.set_state(ic)
    h = 0.5 * (2 * math.pi / n) / f.diag.max_velocity_sum(f.state_native())
    f.step(h)
    got = f.state_native().clone()
    del f
    torch.cuda.empty_cache()
    g = get("b200").make(cfg.with_(dtype="float64"))
    g.set_state(ic)
    g.step(h)
    want = g.state_native()
    err = float((got.to(want.dtype) - want).abs().max() / want.abs().max())
    assert err < 1e-5, err


@pytest.mark.parametrize("dtype,tol", [("float32", 1e-5), ("float64", 1e-12)])
def test_fused3d_512_random_basdevant_one_step_vs_fp64(dtype, tol):
    """n = 512 (one warp per transform in every pass) from a general state: the Taylor-Green
    state has w = 0, so its products u w and v w vanish and the transforms that carry them
    are not checked by it.  One step of the fused engine from a smooth random field against
    the fp64 cuFFT engine from the same state."""
    import torch

    n = 512
    cfg = Config(n=n, dim=3, nu=1e-3, dtype=dtype, form="basdevant")
    gen = torch.Generator(device="cuda").manual_seed(11)
    phys = torch.randn((3, n, n, n), generator=gen, device="cuda", dtype=torch.float64)
    ic = torch.fft.rfftn(phys, dim=(1, 2, 3))
    del phys
    k = torch.fft.fftfreq(n, 1.0 / n, device="cuda", dtype=torch.float64)
    kz = torch.arange(n // 2 + 1, device="cuda", dtype=torch.float64)
    ic *= torch.exp(-(k[:, None, None] ** 2 + k[None, :, None] ** 2 + kz[None, None, :] ** 2)
                    / 200.0) * 1e-3
    f = get(FUSED).make(cfg)
    f.set_state(ic)
    h = 0.5 * (2 * math.pi / n) / f.diag.max_velocity_sum(f.state_native())
    f.step(h)
    got = f.state_native().clone()
    del f
    torch.cuda.empty_cache()
    g = get("b200").make(cfg.with_(dtype="float64"))
    g.set_state(ic)
    g.step(h)
    want = g.state_native()
    err = float((got.to(want.dtype) - want).abs().max() / want.abs().max())
    assert err < tol, err
