"""Learned closure on the CPU: the oracle pinned to the reference's pad_spectrum and to finite
differences of its own loss, the tile hash, bf16 rounding, and the host-side parameter layout."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import closure_oracle as co
from oracle.numpy_oracle import dealias_mask

GOLD = np.load(Path(__file__).parent / "golden" / "reference_vectors.npz")


@pytest.mark.parametrize("key", ["pad_rand2d_32_to_16", "pad_rand2d_16_to_24",
                                 "pad_rand2d_24_to_24", "pad_rand3d_16_to_8",
                                 "pad_rand3d_8_to_12"])
def test_filter_matches_reference_pad_spectrum(key):
    a = GOLD[key + "_in"]
    dim = a.ndim
    n_to = GOLD[key].shape[0]
    np.testing.assert_array_equal(co.filter_spectrum(a, n_to, dim, dealias=False), GOLD[key])


def test_filter_dealias_is_the_target_mask():
    a = GOLD["pad_rand2d_32_to_16_in"]
    plain = co.filter_spectrum(a, 24, 2, dealias=False)
    np.testing.assert_array_equal(co.filter_spectrum(a, 24, 2, dealias=True),
                                  plain * dealias_mask(24, 2))


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.normal(size=4000).astype(np.float32) * 10 ** rng.uniform(-6, 6, 4000),
                        np.float32([1.0, 1 + 2 ** -8, 1 + 3 * 2 ** -8, -1 - 2 ** -8, 0.0])])
    x = x.astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).float().numpy()
    np.testing.assert_array_equal(co.bf16(x), ref)
    assert co.bf16(np.float32([1 + 2 ** -8]))[0] == 1.0           # tie to even
    assert co.bf16(np.float32([1 + 3 * 2 ** -8]))[0] == 1 + 2 ** -6


def _tile_case(seed=0):
    from pyspectral_b200.closure import init_params

    rng = np.random.default_rng(seed)
    fields = rng.normal(size=(3, 128, 128)).astype(np.float32)
    X = co.tile_features(fields, np.float32([0.7, 1.3, 0.9]), 5, 0)
    target = rng.normal(size=co.TILE)
    p = init_params(seed, out_std=1.0).astype(np.float64)
    p[co.BIAS_IN] = 0.1  # non-zero biases so their gradients are exercised
    p[co.WSZ + 3 * co.K + co.BIAS_H] = -0.2
    p[3 * co.WSZ + co.BIAS_H] = 0.05
    return p, X, target


def test_oracle_gradient_matches_finite_differences():
    p, X, target = _tile_case()
    inv = 1.0 / co.TILE

    def loss(q):
        y = co.forward(q, X, exact=True)["y"]
        return float(np.mean((y - target) ** 2))

    g, _ = co.backward(co.forward(p, X, exact=True), target, inv)
    rng = np.random.default_rng(3)
    picks = list(rng.integers(0, co.NPARAM, 40))
    picks += [co.BIAS_IN, co.WSZ + 7 * co.K + co.BIAS_H, 2 * co.WSZ + 11 * co.K + co.BIAS_H,
              3 * co.WSZ + co.BIAS_H, 3 * co.WSZ + 5, 17, co.WSZ + 3]
    h = 1e-6
    for j in picks:
        q1, q2 = p.copy(), p.copy()
        q1[j] += h
        q2[j] -= h
        fd = (loss(q1) - loss(q2)) / (2 * h)
        assert abs(fd - g[j]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (j, fd, g[j])


def test_oracle_gradient_is_zero_on_padding():
    p, X, target = _tile_case(1)
    g, _ = co.backward(co.forward(p.astype(np.float32), X), target.astype(np.float32), 1 / 128)
    W = g[: 3 * co.WSZ].reshape(3, co.H, co.K)
    assert np.all(W[0, :, co.BIAS_IN + 1:] == 0)
    assert np.all(W[1:, :, co.BIAS_H + 1:] == 0)
    assert np.all(g[3 * co.WSZ + co.BIAS_H + 1:] == 0)
    assert np.any(W[0, :, co.BIAS_IN] != 0) and np.any(W[2, :, co.BIAS_H] != 0)


def test_tile_hash_is_deterministic_and_in_range():
    s1 = co.pick_tile(11, 5, np.arange(4096), 37, 256)
    s2 = co.pick_tile(11, 5, np.arange(4096), 37, 256)
    for a, b in zip(s1, s2):
        np.testing.assert_array_equal(a, b)
    snap, row, seg = s1
    assert snap.min() >= 0 and snap.max() < 37
    assert row.min() >= 0 and row.max() < 256
    assert set(np.unique(seg)) == {0, 1}
    counts = np.bincount(snap, minlength=37)
    assert counts.min() > 0.5 * counts.mean()
    other = co.pick_tile(11, 6, np.arange(4096), 37, 256)[1]
    assert np.mean(other == row) < 0.05


def test_adam_first_update_is_lr_times_sign():
    rng = np.random.default_rng(0)
    p = rng.normal(size=100)
    g = rng.normal(size=100)
    q, m, v = co.adam(p, np.zeros(100), np.zeros(100), g, 1, lr=1e-3, total=10**9)
    np.testing.assert_allclose(q, p - 1e-3 * np.sign(g), rtol=0, atol=1e-9)
    assert co.learning_rate(5, 1e-3, 1e-5, 100, 10) == pytest.approx(5e-4)
    assert co.learning_rate(100, 1e-3, 1e-5, 100, 10) == pytest.approx(1e-5)


def test_init_params_layout():
    from pyspectral_b200.closure import NPARAM, init_params

    p = init_params(0)
    assert p.shape == (NPARAM,) == (co.NPARAM,) and p.dtype == np.float32
    W = p[: 3 * co.WSZ].reshape(3, co.H, co.K)
    assert np.all(W[0, :, co.IN:] == 0) and np.all(W[1:, :, co.H:] == 0)
    assert np.all(p[3 * co.WSZ + co.H:] == 0)
    assert np.all(W[0, :, : co.IN] != 0)


def test_snapshot_fields_derivatives():
    n = 32
    x = 2 * np.pi * np.arange(n) / n
    w = np.sin(3 * x)[:, None] * np.cos(2 * x)[None, :]
    wh = np.fft.rfft2(w)
    f = co.snapshot_fields(wh, wh * 0, wh * 0)
    np.testing.assert_allclose(f[0], w, atol=1e-12)
    np.testing.assert_allclose(f[1], 3 * np.cos(3 * x)[:, None] * np.cos(2 * x)[None, :], atol=1e-11)
    np.testing.assert_allclose(f[2], -2 * np.sin(3 * x)[:, None] * np.sin(2 * x)[None, :], atol=1e-11)
    assert np.all(f[3] == 0)


def test_study_config_cutoffs():
    from pyspectral_b200.closure_les import StudyConfig

    sc = StudyConfig()
    assert sc.k_check == 85 and sc.n_fine == 2048 and sc.snapshots == 4000
    assert sc.batch_tiles * 128 == 65536 and sc.train_steps == 20000
    small = StudyConfig.small()
    assert small.k_check == 42 and 3 * small.k_check < small.n_coarse <= 3 * (small.k_check + 1)


def test_cutoff_ramp_rises_from_the_ramp_start_to_the_cutoff():
    from pyspectral_b200.closure_les import StudyConfig, cutoff_ramp

    sc = StudyConfig()
    r = cutoff_ramp(sc, 182)
    kc, k0 = sc.k_check, sc.cutoff_from * sc.k_check
    assert r.dtype == np.float32 and r.shape == (182,)
    assert np.all(r[: int(k0) + 1] == 0)
    assert abs(r[kc] - 1.0) < 1e-6
    assert np.all(np.diff(r) >= 0) and abs(r.max() - 2.25) < 1e-6
