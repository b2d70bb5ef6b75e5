"""simulate.run_device (the run loop's control on the GPU, sp_run_to) against the host-driven
simulate.run: same step count and end time, the same states to round-off."""

from __future__ import annotations

import numpy as np
import pytest

from pyspectral_b200 import Config, initial, simulate
from pyspectral_b200.registry import get

pytestmark = pytest.mark.gpu


def _forced(n, dtype, dim=2):
    return Config(n=n, dim=dim, nu=2e-3, alpha=0.1, alpha_kmax=2.0, force_klo=3, force_khi=5,
                  dtype=dtype)


def _pair(variant, cfg, ic):
    a, b = get(variant).make(cfg), get(variant).make(cfg)
    a.set_state(ic)
    b.set_state(ic)
    return a, b


@pytest.mark.parametrize("variant,dtype,tol", [("b200/fused-inplace-graph", "float64", 1e-11),
                                               ("b200/fused-inplace", "float64", 1e-11),
                                               ("b200/fused-fft-graph", "float32", 2e-6)])
def test_device_loop_matches_host_loop_2d(variant, dtype, tol):
    n = 64 if dtype == "float64" else 128
    cfg = _forced(n, dtype)
    ic = initial.random_phase_2d(n, k0=6.0, seed=2, energy=0.05)
    host, dev = _pair(variant, cfg, ic)
    r1 = simulate.run(host, 0.4, cfl=0.5, dt_max=0.02, target_power=1e-3)
    r2 = simulate.run_device(dev, 0.4, cfl=0.5, dt_max=0.02, target_power=1e-3)
    assert r2.steps == r1.steps and r2.finished
    assert dev.t == pytest.approx(host.t, abs=1e-14)
    assert dev.force_amp == pytest.approx(host.force_amp, rel=1e-6)
    a, b = dev.get_state(), host.get_state()
    assert np.abs(a - b).max() <= tol * np.abs(b).max()
    assert r2.energy[-1] == pytest.approx(r1.energy[-1], rel=10 * tol)


def test_device_loop_3d_cfl_only():
    cfg = Config(n=16, dim=3, nu=1e-2, dtype="float64", form="rotational")
    ic = initial.to_spectral(initial.random_3d(16, k0=2.0, seed=1), 3)
    host, dev = _pair("b200/fused-inplace-graph", cfg, ic)
    r1 = simulate.run(host, 0.2, cfl=0.5, dt_max=0.05)
    r2 = simulate.run_device(dev, 0.2, cfl=0.5, dt_max=0.05)
    assert r2.steps == r1.steps
    a, b = dev.get_state(), host.get_state()
    assert np.abs(a - b).max() <= 1e-11 * np.abs(b).max()


def test_device_loop_fixed_dt_is_exact_tgv():
    n = 64
    cfg = Config(n=n, dim=2, nu=1e-2, dtype="float64")
    s = get("b200/fused-inplace-graph").make(cfg)
    ic = initial.to_spectral(initial.taylor_green_2d(n), 2)
    s.set_state(ic)
    steps = s.run_to(0.1, dt=1e-3)
    assert steps == 100 and s.t == pytest.approx(0.1, abs=1e-12)
    want = ic * np.exp(-2 * cfg.nu * 0.1)
    got = s.get_state() * (initial.to_spectral(initial.taylor_green_2d(n), 2) != 0)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    # a second run continues from the end time
    steps = s.run_to(0.15, dt=1e-3)
    assert steps == 50 and s.t == pytest.approx(0.15, abs=1e-12)


def test_device_loop_with_closure_attached():
    from pyspectral_b200.closure import ClosureNet, ClosureSolver, init_params

    n = 128
    net = ClosureNet(n, 1)
    net.set_params(init_params(3))
    cfg = _forced(n, "float32")
    ic = initial.random_phase_2d(n, k0=6.0, seed=5, energy=0.05)
    host, dev = ClosureSolver(cfg, net, every_stage=False), ClosureSolver(cfg, net, every_stage=False)
    host.set_state(ic)
    dev.set_state(ic)
    r1 = simulate.run(host, 0.3, cfl=0.5, dt_max=0.02, target_power=1e-3)
    r2 = simulate.run_device(dev, 0.3, cfl=0.5, dt_max=0.02, target_power=1e-3)
    assert r2.steps == r1.steps
    a, b = dev.get_state(), host.get_state()
    assert np.abs(a - b).max() <= 2e-6 * np.abs(b).max()
