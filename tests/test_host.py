"""Host-side logic of the package: configuration, grid conventions, registry and availability,
the solver contract's host checks, initial conditions and the run driver.  CPU only."""

from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest

from pyspectral_b200 import BackendUnavailable, Config, fft_split, ffts_per_stage, initial
from pyspectral_b200 import grid
from pyspectral_b200.registry import REGISTRY, get, make_solver, names
from pyspectral_b200.simulate import run, run_steps

GOLDEN = np.load(Path(__file__).parent / "golden" / "reference_vectors.npz")


# ----------------------------------------------------------------------------- config / grid
def test_config_validation():
    with pytest.raises(ValueError):
        Config(n=7)
    with pytest.raises(ValueError):
        Config(n=16, dim=4)
    with pytest.raises(ValueError):
        Config(n=16, dtype="float16")
    with pytest.raises(ValueError):
        Config(n=16, dim=2, form="rotational")
    with pytest.raises(ValueError):
        Config(n=16, dealias="none")
    c = Config(n=16, dim=3)
    assert c.resolved_form() == "basdevant"
    assert c.drag_k2 == 1e30 and Config(n=16, alpha_kmax=2.0).drag_k2 == 4.0
    assert c.with_(n=32).n == 32


def test_fft_tables():
    assert fft_split(2, "basdevant") == (2, 2)
    assert fft_split(3, "basdevant") == (3, 5)
    assert fft_split(3, "rotational") == (6, 3)
    assert ffts_per_stage(2, "advective") == 5
    assert ffts_per_stage(3, "rotational") == 9


def test_grid_matches_reference_conventions():
    assert grid.spectral_shape(16, 2) == (16, 9)
    assert grid.spectral_shape(16, 3) == (16, 16, 9)
    m = grid.dealias_mask(12, 2)
    assert m[3, 3] and not m[4, 0] and not m[0, 4]
    assert m.sum() == 7 * 4
    assert grid.k_squared(8, 3)[1, 2, 3] == 1 + 4 + 9
    kx, ky = grid.wavenumbers(8, 2)
    assert list(kx.ravel()) == list(np.fft.fftfreq(8, 1 / 8))
    assert grid.n_shells(8192, 2) == 5794
    f = np.random.default_rng(0).standard_normal((16, 16))
    fh = np.fft.rfftn(f)
    assert np.isclose(np.sum(grid.hermitian_weights(16, 2) * np.abs(fh) ** 2) / 16**4,
                      np.mean(f**2))


# ----------------------------------------------------------------------------- initial conditions
def test_initial_conditions_match_reference():
    np.testing.assert_allclose(initial.random_2d(32, k0=4), GOLDEN["ic_random_2d_n32_k4_s0"],
                               rtol=0, atol=1e-12)
    np.testing.assert_allclose(initial.random_3d(16, k0=2), GOLDEN["ic_random_3d_n16_k2_s0"],
                               rtol=0, atol=1e-12)
    np.testing.assert_allclose(initial.smooth_2d(32), GOLDEN["ic_smooth_2d_n32"], atol=1e-14)
    np.testing.assert_allclose(initial.to_spectral(initial.taylor_green_3d(16), 3),
                               GOLDEN["ic_tgv3d_n16_spec"], atol=1e-9)


def test_random_phase_2d_properties():
    from oracle.numpy_oracle import OracleDiagnostics

    n = 64
    w = initial.random_phase_2d(n, k0=6, seed=3, energy=0.5)
    d = OracleDiagnostics(n, 2)
    assert d.energy(w) == pytest.approx(0.5, rel=1e-12)
    # Hermitian: the inverse transform of the half spectrum is real and re-transforms exactly
    f = np.fft.irfftn(w, s=(n, n), axes=(0, 1))
    np.testing.assert_allclose(np.fft.rfftn(f), w, atol=1e-10 * np.abs(w).max())
    # dealiased
    assert np.all(w[~grid.dealias_mask(n, 2)] == 0)
    # fixed amplitude: |w| depends on |k| only
    kx, ky = grid.wavenumbers(n, 2)
    k2 = (kx * kx + ky * ky) * np.ones_like(w.real)
    sel = (k2 == 25) & grid.dealias_mask(n, 2)
    assert np.ptp(np.abs(w[sel])) < 1e-12 * np.abs(w[sel]).max()
    # seeded
    assert np.array_equal(w, initial.random_phase_2d(n, k0=6, seed=3, energy=0.5))
    assert not np.array_equal(w, initial.random_phase_2d(n, k0=6, seed=4, energy=0.5))


# ----------------------------------------------------------------------------- registry
def test_registry_names_and_lookup():
    assert "b200/fused-inplace-graph" in names()
    assert get("b200").name == "b200/fused-inplace-graph"
    assert get("b200/fused-inplace-lean").variant == "fused-inplace-lean"
    with pytest.raises(KeyError):
        get("nope")


def test_unavailable_without_gpu_is_reported_not_raised():
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    for v in REGISTRY:
        ok, why = v.available()
        assert not ok and why
    with pytest.raises(BackendUnavailable):
        make_solver("b200", Config(n=16))


def test_unsupported_options_raise_backend_unavailable():
    from pyspectral_b200.solver import B200Solver

    with pytest.raises(BackendUnavailable):
        B200Solver(Config(n=16, dim=2, form="advective"))
    with pytest.raises(BackendUnavailable):
        B200Solver(Config(n=16, dim=2, dealias="phase-shift"))


# ----------------------------------------------------------------------------- driver
class _OracleAsSolver:
    """The oracle behind the SpectralSolver surface the driver uses (test harness only)."""

    def __init__(self, cfg: Config) -> None:
        from oracle.numpy_oracle import OracleDiagnostics, OracleSolver

        self.cfg = cfg
        self.n = cfg.n
        self._s = OracleSolver(cfg.n, cfg.dim, nu=cfg.nu, alpha=cfg.alpha,
                               alpha_kmax=cfg.alpha_kmax, force_amp=cfg.force_amp,
                               force_klo=cfg.force_klo, force_khi=cfg.force_khi,
                               dtype=cfg.dtype, form=cfg.resolved_form())
        self.diag = OracleDiagnostics(cfg.n, cfg.dim)
        self.amps: list[float] = []

    @property
    def t(self) -> float:
        return self._s.t

    def set_state(self, a):
        self._s.set_state(a)

    def state_native(self):
        return self._s.state

    def step(self, dt):
        self._s.step(dt)

    def set_forcing_amplitude(self, a):
        self.amps.append(a)
        self._s.set_forcing_amplitude(a)

    @property
    def force_amp(self):
        return self._s.force_amp

    @t.setter
    def t(self, value):
        self._s.t = value

    def get_state(self):
        return self._s.get_state()

    def synchronize(self):
        pass


def test_cfl_run_lands_on_t_end():
    s = _OracleAsSolver(Config(n=16, dim=2, nu=0.01, dtype="float64"))
    s.set_state(initial.to_spectral(initial.random_2d(16, k0=3), 2))
    res = run(s, 0.3, cfl=0.5, diag_dt=0.1)
    assert abs(s.t - 0.3) < 1e-12
    assert len(res.t) == 4
    assert res.finished and res.steps == len(res.dt)


def test_constant_power_forcing_control():
    cfg = Config(n=16, dim=2, nu=0.01, force_klo=1, force_khi=2.5, dtype="float64")
    s = _OracleAsSolver(cfg)
    s.set_state(initial.to_spectral(initial.random_2d(16, k0=3), 2))
    run(s, 0.2, dt=0.01, target_power=1e-3, cfl_every=10)
    assert len(s.amps) == 2
    eb = s.diag.band_energy(s.state_native(), 1, 2.5)
    assert eb > 0 and all(a > 0 for a in s.amps)


def test_wall_limit_returns_unfinished():
    s = _OracleAsSolver(Config(n=16, dim=2, nu=0.01, dtype="float64"))
    s.set_state(initial.to_spectral(initial.random_2d(16, k0=3), 2))
    res = run(s, 100.0, dt=0.01, wall_limit=0.0)
    assert not res.finished and res.steps == 1


def test_run_steps_is_cfl_every_10():
    s = _OracleAsSolver(Config(n=16, dim=2, nu=0.01, dtype="float64"))
    s.set_state(initial.to_spectral(initial.random_2d(16, k0=3), 2))
    dts = run_steps(s, 25, cfl=0.5, dt_max=0.05)
    assert len(dts) == 25
    assert len(set(dts[:10])) == 1 and len(set(dts[10:20])) == 1
    assert math.isclose(sum(dts), s.t)


# ----------------------------------------------------------------------------- pyspectral plugin
def _pyspectral_importable() -> bool:
    import importlib.util
    import os
    import sys

    src = os.environ.get("PYSPECTRAL_SRC", "")  # pyspectral's src/ directory, when available
    if importlib.util.find_spec("pyspectral") is None and src and Path(src).exists():
        sys.path.append(src)
    return importlib.util.find_spec("pyspectral") is not None


@pytest.mark.skipif(not _pyspectral_importable(), reason="pyspectral not importable (set PYSPECTRAL_SRC to its src/ directory)")
def test_plugin_registers_into_pyspectral_registry(capsys):
    from pyspectral.backends import REGISTRY as REF, BackendUnavailable as RefUnavailable
    from pyspectral.backends import get as ref_get
    from pyspectral.backends.base import SpectralSolver as RefSolver
    from pyspectral.cli import main as ref_cli
    from pyspectral.config import Config as RefConfig

    from pyspectral_b200.pyspectral_plugin import register

    before = len(REF)
    added = register()
    register()  # idempotent
    try:
        assert len(REF) == before + 4 == before + len(added)
        v = ref_get("b200")
        assert v.name == "b200/fused-inplace-graph"
        cls = v.load()
        assert issubclass(cls, RefSolver)
        ok, why = v.available()
        import torch

        if not torch.cuda.is_available():
            assert not ok and "CUDA" in why
            with pytest.raises(RefUnavailable):
                v.make(RefConfig(n=16))
        assert ref_cli(["list"]) == 0
        assert "b200/fused-inplace-graph" in capsys.readouterr().out
    finally:
        del REF[before:]


@pytest.mark.skipif(not _pyspectral_importable(), reason="pyspectral not importable (set PYSPECTRAL_SRC to its src/ directory)")
def test_plugin_class_raises_pyspectral_unavailable():
    from pyspectral.backends.base import BackendUnavailable as RefUnavailable
    from pyspectral.config import Config as RefConfig

    from pyspectral_b200.pyspectral_plugin import _plugin_class

    cls = _plugin_class("B200Solver")
    with pytest.raises(RefUnavailable):
        cls(RefConfig(n=16, dim=2, form="advective"))


# ----------------------------------------------------------------------------- checkpoint / CLI
def test_checkpoint_roundtrip_and_chunked_resume(tmp_path):
    from pyspectral_b200.checkpoint import load_checkpoint, save_checkpoint

    cfg = Config(n=16, dim=2, nu=0.01, force_klo=1, force_khi=2.5, dtype="float32")
    ic = initial.to_spectral(initial.random_2d(16, k0=3), 2)
    whole = _OracleAsSolver(cfg)
    whole.set_state(ic)
    run(whole, 0.2, dt=0.01, diag_dt=0.05)
    # same run in two chunks through a checkpoint
    a = _OracleAsSolver(cfg)
    a.set_state(ic)
    res = run(a, 0.1, dt=0.01, diag_dt=0.05)
    a.set_forcing_amplitude(0.0)
    ck = save_checkpoint(tmp_path / "ck.npz", a, res)
    z = np.load(ck)
    assert z["state"].dtype == np.complex64 and float(z["t"]) == pytest.approx(0.1)
    b = _OracleAsSolver(cfg)
    prev, _ = load_checkpoint(ck, b)
    assert b.t == pytest.approx(0.1) and prev.t == res.t
    res2 = run(b, 0.2, dt=0.01, diag_dt=0.05, result=prev)
    assert res2.t[-1] == pytest.approx(0.2)
    np.testing.assert_allclose(b.get_state(), whole.get_state(), rtol=0, atol=1e-5)


def test_cli_list_reports_every_variant(capsys):
    from pyspectral_b200.cli import main

    assert main(["list"]) == 0
    out = capsys.readouterr().out
    assert "b200/fused-fft-graph" in out and "b200/fused-inplace-graph" in out


def test_tile_tuner_cache_roundtrip(tmp_path):
    from pyspectral_b200.ensemble import load_tune_cache, save_tune_cache, tune_key

    p = tmp_path / "sub" / "tiles.json"
    assert load_tune_cache(p) == {}
    k = tune_key("NVIDIA B200", 512, True, 64)
    assert k == "NVIDIA B200|n=512|fp64|members=64"
    save_tune_cache(p, {k: {"tile": 2, "ms_per_step": {"1": 1.0, "2": 0.8}}})
    assert load_tune_cache(p)[k]["tile"] == 2
    p.write_text("not json")
    assert load_tune_cache(p) == {}
