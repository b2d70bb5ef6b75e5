"""Learned closure on the GPU against the oracle: spectral filter, nonlinear term, snapshot bank,
tcgen05 network inference, gradients and Adam, training, and the coarse solver step with the
closure attached."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import closure_oracle as co
from oracle.numpy_oracle import OracleSolver, dealias_mask, spectral_shape

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


def _random_state(n, seed, k0=None, dtype=np.complex128):
    """Masked random spectrum with a Gaussian envelope of width k0."""
    rng = np.random.default_rng(seed)
    shp = spectral_shape(n, 2)
    kx = np.fft.fftfreq(n, 1.0 / n)[:, None]
    ky = np.arange(n // 2 + 1)[None, :]
    k = np.sqrt(kx ** 2 + ky ** 2)
    k0 = k0 or n / 8
    amp = np.exp(-(k / k0) ** 2) * n * n * 0.05
    a = (rng.normal(size=shp) + 1j * rng.normal(size=shp)) * amp
    # a real field's spectrum: round-trip through the physical grid, then mask
    a = np.fft.rfft2(np.fft.irfft2(a, s=(n, n)))
    return (a * dealias_mask(n, 2)).astype(dtype)


def _bank(n, count, seed, target=None):
    """(count, 4, n, n) entries: fields of random smooth states, S random smooth or target(f)."""
    out = []
    for i in range(count):
        w = _random_state(n, seed + i)
        s = _random_state(n, seed + 100 + i)
        f = co.snapshot_fields(w, s, 0 * s).astype(np.float32)
        if target is not None:
            f[3] = target(f)
        out.append(f)
    return np.stack(out)


# ---------------------------------------------------------------------- spectral helpers
@pytest.mark.parametrize("n,n_to,dim,fp64,dealias", [(64, 32, 2, True, True), (32, 48, 2, True, False),
                                                      (128, 64, 2, False, True), (16, 8, 3, True, True),
                                                      (8, 12, 3, False, False)])
def test_filter_spectrum_matches_oracle(n, n_to, dim, fp64, dealias):
    torch = _torch()
    from pyspectral_b200.closure import filter_spectrum

    rng = np.random.default_rng(n + n_to)
    shp = spectral_shape(n, dim)
    a = rng.normal(size=shp) + 1j * rng.normal(size=shp)
    a = a.astype(np.complex128 if fp64 else np.complex64)
    got = filter_spectrum(torch.from_numpy(a).cuda(), n_to, dim, dealias).cpu().numpy()
    want = co.filter_spectrum(a, n_to, dim, dealias)
    if fp64:
        np.testing.assert_array_equal(got, want)
    else:
        np.testing.assert_allclose(got, want, rtol=1e-6, atol=0)


@pytest.mark.parametrize("n,dtype,tol", [(64, "float64", 1e-12), (128, "float32", 1e-5)])
def test_nonlinear_term_matches_oracle(n, dtype, tol):
    torch = _torch()
    from pyspectral_b200.closure import nonlinear_term
    from pyspectral_b200.config import Config
    from pyspectral_b200.solver import B200Solver

    st = _random_state(n, 3)
    s = B200Solver(Config(n=n, dim=2, dtype=dtype))
    cdt = torch.complex128 if dtype == "float64" else torch.complex64
    got = nonlinear_term(s, torch.from_numpy(st).to(cdt).cuda()).cpu().numpy()
    want = OracleSolver(n, 2).nonlinear(st)
    assert np.abs(got - want).max() <= tol * np.abs(want).max()


def test_nonlinear_term_leaves_stepping_intact():
    """sp_nonlinear borrows the work array; the next step must be the one it would have been."""
    torch = _torch()
    from pyspectral_b200.closure import nonlinear_term
    from pyspectral_b200.config import Config
    from pyspectral_b200.solver import B200Solver

    cfg = Config(n=64, dim=2, nu=1e-3, dtype="float64")
    a, b = B200Solver(cfg), B200Solver(cfg)
    st = _random_state(64, 4)
    a.set_state(st)
    b.set_state(st)
    nonlinear_term(a, torch.from_numpy(_random_state(64, 5)).cuda())
    a.step(1e-3)
    b.step(1e-3)
    np.testing.assert_array_equal(a.get_state(), b.get_state())


def test_snapshot_pipeline_matches_oracle():
    torch = _torch()
    from pyspectral_b200.closure import ClosureNet, SnapshotPipeline

    n_f, n_c = 256, 128
    st = _random_state(n_f, 7, k0=40.0)
    net = ClosureNet(n_c, 2)
    pipe = SnapshotPipeline(net, n_f)
    pipe.add(torch.from_numpy(st).to(torch.complex64).cuda())
    assert net.bank_count == 1
    got = net.bank_entry(0)
    fine, coarse = OracleSolver(n_f, 2), OracleSolver(n_c, 2)
    wbar = co.filter_spectrum(st, n_c)
    fnl = co.filter_spectrum(fine.nonlinear(st), n_c)
    want = co.snapshot_fields(wbar, fnl, coarse.nonlinear(wbar))
    for f in range(4):
        err = np.abs(got[f] - want[f]).max() / np.abs(want[f]).max()
        assert err < 2e-5, (f, err)
    # the subgrid term is a real signal here, not round-off
    fnl_phys = np.fft.irfft2(fnl, s=(n_c, n_c))
    assert np.abs(want[3]).max() > 1e-2 * np.abs(fnl_phys).max()


# ---------------------------------------------------------------------- network
def _net_with(n, bank, seed, out_std=1.0, clip=False):
    from pyspectral_b200.closure import ClosureNet, init_params

    net = ClosureNet(n, max(1, bank.shape[0]))
    net.load_bank(bank)
    p = init_params(seed, out_std=out_std)
    rng = np.random.default_rng(seed)
    # non-zero biases, as training produces them
    W = p[: 3 * co.WSZ].reshape(3, co.H, co.K)
    W[0, :, co.BIAS_IN] = rng.normal(0, 0.1, co.H)
    W[1:, :, co.BIAS_H] = rng.normal(0, 0.1, (2, co.H))
    p[3 * co.WSZ + co.BIAS_H] = 0.05
    net.set_params(p)
    std = np.sqrt((bank.astype(np.float64) ** 2).mean(axis=(0, 2, 3)))
    net.set_scales(1.0 / std[:3], float(std[3]), clip)
    return net, p


@pytest.mark.parametrize("clip", [False, True])
def test_inference_matches_oracle(clip):
    torch = _torch()
    n = 128
    bank = _bank(n, 1, 20)
    net, p = _net_with(n, bank, 1, clip=clip)
    got = net.infer(torch.from_numpy(bank[0, :3]).cuda()).cpu().numpy()
    want = co.infer_field(p, bank[0, :3], net.inscale, net.outscale, clip)
    scale = np.abs(want).max()
    diff = np.abs(got - want)
    # bf16 operands: a hidden activation within rounding distance of a bf16 tie may round the
    # other way on the device; such flips stay rare and small
    assert diff.max() <= 2e-2 * scale, diff.max() / scale
    assert diff.mean() <= 2e-4 * scale, diff.mean() / scale
    if clip:
        assert np.all(got * bank[0, 0] <= 0)


def test_gradient_matches_oracle():
    n = 128
    bank = _bank(n, 3, 30)
    net, p = _net_with(n, bank, 2)
    g, loss = net.grad_at(step=2, batch_tiles=20, seed=5)
    want, wloss = co.batch_grad(p, bank, net.inscale, net.outscale, 5, 2, 20)
    assert loss == pytest.approx(wloss, rel=1e-3)
    blocks = [(0, co.WSZ), (co.WSZ, 2 * co.WSZ), (2 * co.WSZ, 3 * co.WSZ),
              (3 * co.WSZ, co.NPARAM)]
    for lo, hi in blocks:
        err = np.linalg.norm(g[lo:hi] - want[lo:hi]) / np.linalg.norm(want[lo:hi])
        assert err < 1e-2, (lo, err)
    # padding columns carry no gradient
    W = g[: 3 * co.WSZ].reshape(3, co.H, co.K)
    assert np.all(W[0, :, co.BIAS_IN + 1:] == 0) and np.all(W[1:, :, co.BIAS_H + 1:] == 0)
    assert np.all(g[3 * co.WSZ + co.BIAS_H + 1:] == 0)


def test_adam_step_matches_oracle():
    n = 128
    bank = _bank(n, 2, 40)
    net, p = _net_with(n, bank, 3)
    net.set_adam(lr=1e-3, lr_min=1e-5, total_steps=100, warmup=0)
    net.train(1, batch_tiles=16, seed=9)
    g = net.grad().astype(np.float64)
    got = net.params()
    want, _, _ = co.adam(p.astype(np.float64), np.zeros(co.NPARAM), np.zeros(co.NPARAM), g, 1,
                         lr=1e-3, lr_min=1e-5, total=100, warmup=0)
    np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-8)
    assert net.step_count == 1


def test_training_learns_a_local_linear_closure():
    n = 128

    def target(f):
        return 0.5 * f[1] - 0.3 * f[2] + 0.2 * f[0] * (np.abs(f[1]).max() / np.abs(f[0]).max())

    bank = _bank(n, 8, 50, target=target)
    net, _ = _net_with(n, bank, 4, out_std=0.1)
    net.set_adam(lr=3e-3, lr_min=1e-4, total_steps=400, warmup=20)
    losses = net.train(400, batch_tiles=64, seed=1)
    assert np.all(np.isfinite(losses))
    assert losses[-20:].mean() < 0.05 * losses[:5].mean(), (losses[:5], losses[-20:])


# ---------------------------------------------------------------------- coarse solver
def _forced_cfg(n):
    from pyspectral_b200.config import Config

    return Config(n=n, dim=2, nu=2e-4, alpha=0.1, alpha_kmax=2, force_amp=0.3, force_klo=3,
                  force_khi=5, dtype="float32")


def test_closure_solver_with_zero_network_is_the_plain_solver():
    from pyspectral_b200.closure import ClosureNet, ClosureSolver
    from pyspectral_b200.solver import B200Solver

    n = 128
    net = ClosureNet(n, 1)
    net.set_params(np.zeros(co.NPARAM, np.float32))
    cfg = _forced_cfg(n)
    a, b = ClosureSolver(cfg, net), B200Solver(cfg)
    st = _random_state(n, 60)
    a.set_state(st)
    b.set_state(st)
    for dt in (2e-3, 1.5e-3, 2e-3, 1e-3, 2e-3):
        a.step(dt)
        b.step(dt)
    a.synchronize()
    sa, sb = a.get_state(), b.get_state()
    assert np.abs(sa - sb).max() <= 1e-6 * np.abs(sb).max()


@pytest.mark.parametrize("every_stage", [True, False])
def test_closure_solver_step_matches_oracle(every_stage):
    from pyspectral_b200.closure import ClosureSolver

    n = 128
    bank = _bank(n, 1, 70)
    net, p = _net_with(n, bank, 5, out_std=0.3)
    net.set_scales(net.inscale, 10.0 * net.outscale)  # a closure term comparable to N
    gain = np.random.default_rng(5).uniform(0.0, 2.0, net.nshell).astype(np.float32)
    net.set_shell_gain(gain)
    kx = np.fft.fftfreq(n, 1.0 / n)[:, None]
    ky = np.arange(n // 2 + 1)[None, :]
    g_modes = gain[(np.sqrt(kx ** 2 + ky ** 2) + 0.5).astype(int)]
    cfg = _forced_cfg(n)
    dev = ClosureSolver(cfg, net, every_stage=every_stage)
    st = _random_state(n, 71)
    dev.set_state(st)

    def closure_term(s):
        fields = co.snapshot_fields(s, 0 * s, 0 * s)[:3].astype(np.float32)
        S = co.infer_field(p, fields, net.inscale, net.outscale, False)
        Sh = np.fft.rfft2(S.astype(np.float64)) * dealias_mask(n, 2) * g_modes
        Sh[0, 0] = 0.0  # the subgrid term carries no mean
        return Sh

    class OracleLES(OracleSolver):
        held = None

        def nonlinear(self, s):
            S = closure_term(s) if every_stage else self.held
            return super().nonlinear(s) + S

        def _step(self, dt):
            # held mode: the network sees the step's initial state only
            self.held = closure_term(self.state)
            super()._step(dt)

    kw = dict(nu=cfg.nu, alpha=cfg.alpha, alpha_kmax=cfg.alpha_kmax, force_amp=cfg.force_amp,
              force_klo=cfg.force_klo, force_khi=cfg.force_khi)
    ora, plain = OracleLES(n, 2, **kw), OracleSolver(n, 2, **kw)
    ora.set_state(st)
    plain.set_state(st)
    dt = 2e-3
    dev.step(dt)
    ora.step(dt)
    plain.step(dt)
    dev.synchronize()
    got, want = dev.get_state(), ora.get_state()
    scale = np.abs(want).max()
    assert np.abs(got - want).max() <= 1e-5 * scale
    # the closure changed the step by far more than that tolerance
    assert np.abs(want - plain.get_state()).max() > 50 * 1e-5 * scale


def test_data_parallel_training_on_one_rank_is_plain_training():
    from pyspectral_b200.sharding import train_data_parallel

    n = 128
    bank = _bank(n, 3, 90)
    a, p = _net_with(n, bank, 7)
    b, _ = _net_with(n, bank, 7)
    for net in (a, b):
        net.set_adam(lr=2e-3, lr_min=1e-4, total_steps=60, warmup=5)
    la = a.train(60, batch_tiles=24, seed=3)  # graph-replayed chunks
    lb = train_data_parallel(b, 60, batch_tiles=24, seed=3)  # split steps, world of one
    np.testing.assert_array_equal(a.params(), b.params())
    np.testing.assert_array_equal(la, lb)
    assert a.step_count == b.step_count == 60
