"""Batched ensembles of uneven grid sizes against single runs and the oracle (GPU)."""

from __future__ import annotations

import math

import numpy as np
import pytest

from oracle.numpy_oracle import OracleSolver
from pyspectral_b200 import BackendUnavailable, Config, initial
from pyspectral_b200.registry import get

pytestmark = pytest.mark.gpu
FUSED = "b200/fused-fft-graph"


def _members(dtype: str) -> list[Config]:
    out = []
    for n in (32, 64, 128):
        for j in range(2):
            out.append(Config(n=n, dim=2, nu=2e-3 * (1 + j), alpha=0.1, alpha_kmax=2.0,
                              force_amp=0.2 + 0.1 * j, force_klo=3, force_khi=5, dtype=dtype))
    return out


def _ics(members: list[Config]) -> list[np.ndarray]:
    return [initial.random_phase_2d(c.n, k0=c.n / 10, seed=7 + i) for i, c in enumerate(members)]


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_members_equal_single_runs_bit_for_bit(dtype):
    from pyspectral_b200.ensemble import Ensemble

    cfgs = _members(dtype)
    ics = _ics(cfgs)
    ens = Ensemble(cfgs, autotune=False)  # tile 1: the single-run engine's kernels
    ens.set_states(ics)
    dts = [np.array([1e-3 * (1 + 0.1 * i + 0.05 * k) for i in range(len(cfgs))]) for k in range(6)]
    amps = [np.array([0.2 + 0.02 * i + 0.01 * k for i in range(len(cfgs))]) for k in range(6)]
    for k in range(6):
        ens.set_forcing_amplitudes(amps[k])
        ens.step(dts[k])
    for i, c in enumerate(cfgs):
        s = get(FUSED).make(c)
        s.set_state(ics[i])
        for k in range(6):
            s.set_forcing_amplitude(amps[k][i])
            s.step(dts[k][i])
        assert np.array_equal(ens.get_state(i), s.get_state()), i
        assert ens.t[i] == pytest.approx(s.t)


def test_get_states_equals_get_state_of_each_member():
    """get_states (one refresh and one copy per size class) returns every member's state, in
    member order, equal bit for bit to get_state of that member."""
    from pyspectral_b200.ensemble import Ensemble

    cfgs = _members("float32")
    ens = Ensemble(cfgs, autotune=False)
    ens.set_states(_ics(cfgs))
    for k in range(3):
        ens.step(np.array([1e-3 * (1 + 0.1 * i + 0.05 * k) for i in range(len(cfgs))]))
    allst = ens.get_states()
    assert len(allst) == len(cfgs)
    for i in range(len(cfgs)):
        assert allst[i].dtype == np.complex128
        assert np.array_equal(allst[i], ens.get_state(i)), i


def test_set_states_twice_in_a_row_keeps_the_second():
    """set_states stages each class through one pinned host buffer and copies it to the device
    asynchronously: a second call right after the first waits for the first copy before it
    overwrites the buffer, so the members hold the second states (compared with an ensemble
    given only those)."""
    from pyspectral_b200.ensemble import Ensemble

    cfgs = _members("float32")
    ics = _ics(cfgs)
    second = [2.0 * a for a in ics]
    ens = Ensemble(cfgs, autotune=False)
    ens.set_states(ics)
    ens.set_states(second)
    ref = Ensemble(cfgs, autotune=False)
    ref.set_states(second)
    for i, (a, b) in enumerate(zip(ens.get_states(), ref.get_states())):
        assert np.array_equal(a, b), i


def test_batched_diagnostics_and_cfl_match_single_runs():
    from pyspectral_b200.ensemble import Ensemble

    cfgs = _members("float64")
    ics = _ics(cfgs)
    ens = Ensemble(cfgs)
    ens.set_states(ics)
    ens.step(1e-3)
    d = ens.diagnostics(3, 5)
    u = ens.max_velocity_sum()
    for i, c in enumerate(cfgs):
        s = get(FUSED).make(c)
        s.set_state(ics[i])
        s.step(1e-3)
        ref = s.diag.all(s.state_native(), 3, 5)
        np.testing.assert_allclose(d[i], [ref["energy"], ref["enstrophy"], ref["palinstrophy"],
                                          ref["band_energy"]], rtol=1e-12)
        assert u[i] == pytest.approx(s.diag.max_velocity_sum(s.state_native()), rel=1e-12)


def test_small_member_matches_oracle():
    from pyspectral_b200.ensemble import Ensemble

    c = Config(n=32, dim=2, nu=0.01, alpha=0.5, alpha_kmax=2.0, force_amp=0.3, force_klo=1,
               force_khi=2.5, dtype="float64")
    big = Config(n=256, dim=2, nu=1e-3, dtype="float64")
    ic = initial.to_spectral(initial.random_2d(32, k0=4), 2)
    ens = Ensemble([c, big])
    ens.set_states([ic, initial.random_phase_2d(256, k0=8, seed=1)])
    ref = OracleSolver(32, 2, nu=0.01, alpha=0.5, alpha_kmax=2.0, force_amp=0.3, force_klo=1,
                       force_khi=2.5)
    ref.set_state(ic)
    for k in range(5):
        ens.step([0.01, 1e-3])
        ref.step(0.01)
    ens.set_forcing_amplitudes([0.1, 0.0])
    ref.set_forcing_amplitude(0.1)
    for k in range(3):
        ens.step([0.007, 1e-3])
        ref.step(0.007)
    r = ref.get_state()
    assert np.abs(ens.get_state(0) - r).max() / np.abs(r).max() < 1e-12


def test_constant_power_cfl_run_matches_single_run_driver():
    from pyspectral_b200.ensemble import Ensemble
    from pyspectral_b200.simulate import run_steps

    cfgs = [Config(n=n, dim=2, nu=1e-3, alpha=0.1, alpha_kmax=2, force_klo=3, force_khi=5,
                   dtype="float64") for n in (64, 128, 128)]
    ics = _ics(cfgs)
    ens = Ensemble(cfgs)
    ens.set_states(ics)
    hist = ens.run_steps(25, cfl=0.5, target_power=1e-3)
    assert hist.shape == (25, 3) and np.all(hist > 0)
    for i, c in enumerate(cfgs):
        s = get(FUSED).make(c)
        s.set_state(ics[i])
        dts = run_steps(s, 25, cfl=0.5, target_power=1e-3)
        np.testing.assert_allclose(hist[:, i], dts, rtol=1e-12)
        r = s.get_state()
        assert np.abs(ens.get_state(i) - r).max() / np.abs(r).max() < 1e-12


@pytest.mark.parametrize("worklist", [0, 64])
def test_one_graph_step_launch_count(worklist):
    """Per class: 8 launches per class and step; work list: 8 for the whole group (a row pass
    and a column pass per RK stage over every class)."""
    from pyspectral_b200.ensemble import Ensemble

    ens = Ensemble(_members("float32"), autotune=False, worklist=worklist)
    assert ens.worklist == worklist
    ens.set_states(_ics(ens.members))
    ens.step(1e-3)
    before = ens.kernel_launches
    ens.step(1e-3)
    assert ens.kernel_launches - before == (8 if worklist else 8 * len(ens.classes))


def _uneven(dtype):
    return [Config(n=n, dim=2, nu=1e-3 * (1 + 0.3 * j), alpha=0.1, alpha_kmax=2.0,
                   force_amp=0.2 + 0.05 * j, force_klo=3, force_khi=5, dtype=dtype)
            for n in (64, 128, 256, 512, 1024) for j in range(3 if n < 1024 else 1)]


@pytest.mark.parametrize("dtype,mt", [("float32", 64), ("float32", 128), ("float64", 64),
                                      ("float64", 128)])
def test_worklist_group_step_equals_per_class_launches(dtype, mt):
    """The packed work list runs each row and column with the single-run passes' code:
    members equal the per-class launches over dt and amplitude changes, to round-off (the
    kernels are compiled separately and may contract multiply-adds differently)."""
    from pyspectral_b200.ensemble import Ensemble

    cfgs = _uneven(dtype)
    ics = _ics(cfgs)
    a = Ensemble(cfgs, autotune=False, worklist=0)
    b = Ensemble(cfgs, autotune=False, worklist=mt)
    assert b.worklist == mt
    for e in (a, b):
        e.set_states(ics)
    for k in range(4):
        dt = np.array([2e-4 * (1 + 0.1 * i + 0.05 * k) for i in range(len(cfgs))])
        amps = np.array([0.2 + 0.01 * i + 0.02 * k for i in range(len(cfgs))])
        for e in (a, b):
            e.set_forcing_amplitudes(amps)
            e.step(dt)
    tol = 1e-13 if dtype == "float64" else 1e-6
    for i in range(len(cfgs)):
        ra = a.get_state(i)
        assert np.abs(b.get_state(i) - ra).max() <= tol * np.abs(ra).max(), i


def test_worklist_rejects_classes_it_does_not_run():
    from pyspectral_b200.ensemble import Ensemble

    cfgs = [Config(n=2048, dim=2, nu=1e-4, dtype="float32"), Config(n=64, dim=2, nu=1e-3)]
    e = Ensemble(cfgs, autotune=False)
    assert e.worklist == 0  # 2048^2 and a second precision: one launch per class
    with pytest.raises(BackendUnavailable):
        Ensemble(cfgs, autotune=False, worklist=64)


def test_ensemble_rejects_unsupported_members():
    from pyspectral_b200.ensemble import Ensemble

    with pytest.raises(BackendUnavailable):
        Ensemble([Config(n=48, dim=2)])
    with pytest.raises(BackendUnavailable):
        Ensemble([Config(n=32, dim=3)])
    with pytest.raises(ValueError):
        Ensemble([Config(n=32, dim=2, alpha=0.1), Config(n=32, dim=2, alpha=0.2)])
    assert math.isclose(__import__("pyspectral_b200.ensemble", fromlist=["x"]).nu_for_kmax_eta(
        384, 1e-3, 11.0), (121e-3) ** (1 / 3) * (1 / 128) ** 2)


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_every_tile_gives_the_same_members(dtype):
    """The autotuner's choice (sub-blocks per CTA of the fused passes) leaves the arithmetic of
    every sequence alone; separately compiled kernels may contract multiply-adds differently, so
    tiles agree to round-off (bit-identical runs need a fixed tile)."""
    from pyspectral_b200.ensemble import Ensemble

    cfgs = [Config(n=n, dim=2, nu=2e-3, alpha=0.1, alpha_kmax=2.0, force_amp=0.2, force_klo=3,
                   force_khi=5, dtype=dtype) for n in (16, 64, 256, 1024) for _ in range(2)]
    ics = [initial.random_phase_2d(c.n, k0=c.n / 10, seed=3 + i) for i, c in enumerate(cfgs)]
    out = {}
    for tile in (1, 2, 4):
        ens = Ensemble(cfgs, autotune=False)
        for c in ens.classes:
            c.set_tile(tile)
        assert ens.tiles == [tile] * len(ens.classes)
        ens.set_states(ics)
        for k in range(3):
            ens.step(1e-3 * (1 + 0.1 * k))
        out[tile] = [ens.get_state(i) for i in range(len(cfgs))]
    tol = 1e-13 if dtype == "float64" else 2e-6
    for tile in (2, 4):
        for i in range(len(cfgs)):
            ref = out[1][i]
            assert np.abs(out[tile][i] - ref).max() <= tol * np.abs(ref).max(), (tile, i)


def test_autotuner_times_candidates_and_caches(tmp_path, monkeypatch):
    import json

    from pyspectral_b200.ensemble import Ensemble, tune_key

    monkeypatch.setenv("PYSPECTRAL_B200_TUNE_CACHE", str(tmp_path / "tiles.json"))
    cfgs = [Config(n=n, dim=2, nu=2e-3, dtype="float32") for n in (128, 128, 256, 2048)]
    ens = Ensemble(cfgs, autotune=True)
    rep = ens.tuner.report
    data = json.loads((tmp_path / "tiles.json").read_text())
    import torch

    gpu = torch.cuda.get_device_name(0)
    for n, m in ((128, 2), (256, 1)):
        e = data[tune_key(gpu, n, False, m)]
        assert set(e["ms_per_step"]) == {"1", "2", "4"} and e["tile"] in (1, 2, 4)
        assert rep[tune_key(gpu, n, False, m)]["cached"] is False
    assert ens.tiles[-1] == 1  # 2048^2: only tile 1 is compiled
    again = Ensemble(cfgs, autotune=True)
    assert again.tuner.report[tune_key(gpu, 128, False, 2)]["cached"] is True
    assert again.tiles == ens.tiles


def test_sharded_ensemble_on_one_rank_is_the_ensemble():
    from pyspectral_b200.ensemble import Ensemble
    from pyspectral_b200.sharding import ShardedEnsemble

    cfgs = _members("float64")
    ics = _ics(cfgs)
    a, b = Ensemble(cfgs, autotune=False), ShardedEnsemble(cfgs, factory=lambda c: Ensemble(c, autotune=False))
    a.set_states(ics)
    b.set_states(ics)
    for k in range(3):
        dt = np.array([1e-3 * (1 + 0.1 * i + 0.05 * k) for i in range(len(cfgs))])
        a.step(dt)
        b.step(dt)
    np.testing.assert_array_equal(a.diagnostics(3.0, 5.0), b.diagnostics(3.0, 5.0))
    np.testing.assert_array_equal(a.max_velocity_sum(), b.max_velocity_sum())


@pytest.mark.parametrize("count", [1, 2])
def test_large_class_matches_single_runs(count):
    """A 2048^2 size class: one member runs the streamed persistent column pass (as a single
    run does), two members the batched one-column-per-CTA pass; both equal single runs (to
    round-off: separately compiled kernels)."""
    from pyspectral_b200.ensemble import Ensemble

    cfgs = [Config(n=2048, dim=2, nu=1e-4, alpha=0.1, alpha_kmax=2.0, force_amp=0.2 + 0.1 * i,
                   force_klo=4, force_khi=6, dtype="float32") for i in range(count)]
    ics = _ics(cfgs)
    ens = Ensemble(cfgs, autotune=False)
    ens.set_states(ics)
    for _ in range(3):
        ens.step(np.full(count, 2e-4))
    for i, c in enumerate(cfgs):
        s = get(FUSED).make(c)
        s.set_state(ics[i])
        s.advance(3, 2e-4)
        ref = s.get_state()
        assert np.abs(ens.get_state(i) - ref).max() <= 2e-6 * np.abs(ref).max(), i
