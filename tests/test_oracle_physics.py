"""Known answers of the reference's physics tests (tests/test_reference.py:15-133) checked on
the oracle — the independent pins that do not depend on the reference's code at all."""

from __future__ import annotations

import math

import numpy as np
import pytest

from oracle.numpy_oracle import OracleDiagnostics, OracleSolver, wavenumbers
from pyspectral_b200 import initial


@pytest.mark.parametrize("form", ["basdevant", "advective"])
@pytest.mark.parametrize("dtype,tol", [("float64", 1e-13), ("float32", 2e-6)])
def test_tgv2d_exact_decay(form, dtype, tol):
    s = OracleSolver(16, 2, nu=0.1, dtype=dtype, form=form)
    w0 = initial.to_spectral(initial.taylor_green_2d(16), 2)
    s.set_state(w0)
    s.advance(20, 0.05)
    exact = w0 * math.exp(-2 * 0.1 * 1.0)
    assert np.abs(s.get_state() - exact).max() / np.abs(exact).max() < tol


def test_rk4_is_fourth_order_and_ifrk4_exact():
    dts = (0.2, 0.1, 0.05, 0.025)
    errs, errs_if = [], []
    w0 = initial.to_spectral(initial.taylor_green_2d(16), 2)
    for dt in dts:
        for integ, store in (("rk4", errs), ("ifrk4", errs_if)):
            s = OracleSolver(16, 2, nu=0.5, integrator=integ)
            s.set_state(w0)
            s.advance(int(round(1.0 / dt)), dt)
            ex = w0 * math.exp(-2 * 0.5 * s.t)
            store.append(np.abs(s.get_state() - ex).max() / np.abs(ex).max())
    order = np.polyfit(np.log(dts), np.log(errs), 1)[0]
    assert 3.8 < order < 4.3
    assert max(errs_if) < 1e-13


def test_forms_agree():
    w0 = initial.to_spectral(initial.smooth_2d(32), 2)
    a = OracleSolver(32, 2, nu=0.01, form="basdevant")
    b = OracleSolver(32, 2, nu=0.01, form="advective")
    for s in (a, b):
        s.set_state(w0)
        s.advance(5, 0.01)
    assert np.abs(a.get_state() - b.get_state()).max() < 1e-12 * np.abs(a.get_state()).max()
    u0 = initial.to_spectral(initial.random_3d(16, k0=2), 3)
    a = OracleSolver(16, 3, nu=0.01, form="basdevant")
    b = OracleSolver(16, 3, nu=0.01, form="rotational")
    for s in (a, b):
        s.set_state(u0)
        s.advance(5, 0.01)
    assert np.abs(a.get_state() - b.get_state()).max() < 1e-12 * np.abs(a.get_state()).max()


def test_inviscid_energy_and_divergence():
    n = 16
    u0 = initial.to_spectral(initial.random_3d(n, k0=2), 3)
    s = OracleSolver(n, 3, nu=0.0)
    s.set_state(u0)
    d = OracleDiagnostics(n, 3)
    e0 = d.energy(u0)
    s.advance(10, 0.002)
    u = s.get_state()
    assert abs(d.energy(u) - e0) / e0 < 1e-9
    kx, ky, kz = wavenumbers(n, 3)
    assert np.abs(kx * u[0] + ky * u[1] + kz * u[2]).max() < 1e-10 * np.abs(u).max()


def test_energy_budget_2d():
    n, nu, dt = 32, 0.01, 1e-3
    s = OracleSolver(n, 2, nu=nu)
    s.set_state(initial.to_spectral(initial.smooth_2d(n), 2))
    d = OracleDiagnostics(n, 2)
    e, z = [], []
    for _ in range(3):
        e.append(d.energy(s.state))
        z.append(d.enstrophy(s.state))
        s.step(dt)
    dedt = (e[2] - e[0]) / (2 * dt)
    assert abs(dedt + 2 * nu * z[1]) < 1e-6 * abs(dedt)


def test_tgv3d_initial_diagnostics():
    d = OracleDiagnostics(16, 3)
    u = initial.to_spectral(initial.taylor_green_3d(16), 3)
    assert d.energy(u) == pytest.approx(0.125)
    assert d.enstrophy(u) == pytest.approx(0.375)
    assert d.spectrum(u)[1].sum() == pytest.approx(0.125)


def test_forcing_band_injects_energy():
    n = 32
    s = OracleSolver(n, 2, nu=0.0, force_amp=1.0, force_klo=1, force_khi=1.5)
    w0 = initial.to_spectral(initial.taylor_green_2d(n), 2)
    s.set_state(w0)
    s.advance(10, 0.01)
    assert np.allclose(s.get_state(), w0 * math.exp(0.1), rtol=1e-12, atol=1e-9)


def test_large_scale_drag_only_below_kmax():
    s = OracleSolver(16, 2, nu=0.0, alpha=1.0, alpha_kmax=1.5)
    L = s.linear_operator(s.k2)
    assert L[1, 1] == -1.0
    assert L[2, 0] == 0.0


def test_parseval_hermitian_weights():
    from oracle.numpy_oracle import hermitian_weights

    f = np.random.default_rng(0).standard_normal((16, 16))
    fh = np.fft.rfftn(f)
    assert np.isclose(np.sum(hermitian_weights(16, 2) * np.abs(fh) ** 2) / 16**4, np.mean(f**2))
