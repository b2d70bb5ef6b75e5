"""The multi-GPU data planes through a real NCCL process group of one rank on one GPU.

With a process group, the slab exchange (``all_to_all_single``), the sharded ensemble's
diagnostics gather (``all_gather``) and the data-parallel closure training's gradient mean
(``all_reduce``) go through NCCL on device buffers even with a single rank, so these tests run
the code path that several GPUs run, minus the NVLink transfers.  The slab solver is compared
with the fp64 oracle, not only with the single-GPU solver.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle.numpy_oracle import OracleSolver
from pyspectral_b200 import Config, initial

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nccl_group():
    import datetime

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(0)
    store = dist.HashStore()
    dist.init_process_group("nccl", store=store, rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device("cuda", 0))
    try:
        yield dist
    finally:
        torch.cuda.synchronize()
        dist.destroy_process_group()


def _slab_cfg(form, dtype):
    return Config(n=32, dim=3, nu=2e-2, alpha=0.3, alpha_kmax=1.5, force_amp=0.4, force_klo=1,
                  force_khi=2.5, dtype=dtype, form=form)


@pytest.mark.parametrize("dtype,tol", [("float64", 1e-12), ("float32", 5e-6)])
@pytest.mark.parametrize("form", ["basdevant", "rotational"])
def test_slab_solver_over_nccl_matches_oracle(nccl_group, form, dtype, tol):
    """32^3, forcing, drag, a dt change and an amplitude change mid-run (the reference's parity
    protocol, tests/test_backends.py:24-47), every exchange an NCCL all_to_all_single."""
    from pyspectral_b200.slab import SlabSolver

    cfg = _slab_cfg(form, dtype)
    ic = initial.to_spectral(initial.random_3d(32, k0=3.0, seed=4), 3)
    s = SlabSolver(cfg, 0, 1, comm=nccl_group)
    assert s.recv.data_ptr() != s.send.data_ptr()
    ref = OracleSolver(32, 3, nu=cfg.nu, alpha=cfg.alpha, alpha_kmax=cfg.alpha_kmax,
                       force_amp=cfg.force_amp, force_klo=cfg.force_klo, force_khi=cfg.force_khi,
                       form=form)
    s.set_state(ic)
    ref.set_state(ic)
    for k, dt in enumerate((2e-3, 1.5e-3, 2.5e-3)):
        if k == 1:
            s.set_forcing_amplitude(0.7)
            ref.set_forcing_amplitude(0.7)
        s.step(dt)
        ref.step(dt)
    want = ref.get_state()
    got = s.get_state()
    assert np.abs(got - want).max() <= tol * np.abs(want).max()
    assert s.kernel_launches > 0


def test_sharded_ensemble_gathers_over_nccl(nccl_group):
    import torch

    from pyspectral_b200.ensemble import Ensemble
    from pyspectral_b200.sharding import Comm, ShardedEnsemble

    cfgs = [Config(n=n, dim=2, nu=2e-3 * (1 + j), alpha=0.1, alpha_kmax=2.0,
                   force_amp=0.2 + 0.1 * j, force_klo=3, force_khi=5, dtype="float64")
            for n in (32, 64) for j in range(2)]
    ics = [initial.random_phase_2d(c.n, k0=c.n / 10, seed=7 + i) for i, c in enumerate(cfgs)]
    comm = Comm(torch.device("cuda", 0))
    assert comm.dist is not None and comm.world == 1
    a = Ensemble(cfgs, autotune=False)
    b = ShardedEnsemble(cfgs, comm=comm, factory=lambda c: Ensemble(c, autotune=False))
    a.set_states(ics)
    b.set_states(ics)
    for k in range(3):
        dt = np.array([1e-3 * (1 + 0.1 * i + 0.05 * k) for i in range(len(cfgs))])
        a.step(dt)
        b.step(dt)
    np.testing.assert_array_equal(a.diagnostics(3.0, 5.0), b.diagnostics(3.0, 5.0))
    np.testing.assert_array_equal(a.max_velocity_sum(), b.max_velocity_sum())


def test_data_parallel_training_over_nccl_is_plain_training(nccl_group):
    """The gradient mean is an NCCL all_reduce of the library's gradient buffer in place."""
    import torch

    from oracle import closure_oracle as co
    from pyspectral_b200.closure import ClosureNet, init_params
    from pyspectral_b200.sharding import Comm, train_data_parallel

    n = 128
    rng = np.random.default_rng(90)
    bank = rng.normal(0.0, 1.0, (3, 4, n, n)).astype(np.float32)

    def net():
        c = ClosureNet(n, bank.shape[0])
        c.load_bank(bank)
        p = init_params(7)
        W = p[: 3 * co.WSZ].reshape(3, co.H, co.K)
        W[0, :, co.BIAS_IN] = 0.05
        c.set_params(p)
        c.set_scales(np.ones(3), 1.0, False)
        c.set_adam(lr=2e-3, lr_min=1e-4, total_steps=40, warmup=5)
        return c

    a, b = net(), net()
    la = a.train(40, batch_tiles=16, seed=3)
    lb = train_data_parallel(b, 40, batch_tiles=16, seed=3,
                             comm=Comm(torch.device("cuda", 0)))
    np.testing.assert_array_equal(a.params(), b.params())
    np.testing.assert_array_equal(la, lb)
