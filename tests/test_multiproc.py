"""The N > 1 path of bench.py on CPU: two gloo ranks on 127.0.0.1 run replicas, meet at the
barriers, agree on the max of their timings; the reference arm prints on rank 0 only."""

from __future__ import annotations

import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]

WORKER = r"""
import json, os, sys
sys.path.insert(0, {root!r})
import bench
rank = int(os.environ["RANK"])
rep = bench.Replicas("gloo")
rep.barrier()
mx = rep.max(10.0 + rank)            # rank 1 is the slower replica
rep.barrier()
rep.close()
value = bench.aggregate_mpts(rep.world, 8192.0 ** 2, mx * 1e-3)
print(json.dumps({{"rank": rank, "world": rep.world, "max": mx, "value": value}}))
"""


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _launch(code: str, world: int = 2) -> list[subprocess.CompletedProcess]:
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(world), LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, cwd=ROOT,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    out = []
    for p in procs:
        try:
            so, se = p.communicate(timeout=120)
        except subprocess.TimeoutExpired:
            p.kill()
            so, se = p.communicate()
        out.append(subprocess.CompletedProcess(p.args, p.returncode, so, se))
    return out


def test_two_gloo_replicas_agree_on_the_max_time():
    import json

    res = _launch(WORKER.format(root=str(ROOT)))
    for r in res:
        assert r.returncode == 0, r.stderr
    lines = [json.loads(r.stdout.strip().splitlines()[-1]) for r in res]
    assert [d["rank"] for d in lines] == [0, 1]
    assert all(d["world"] == 2 and d["max"] == 11.0 for d in lines)
    # whole-job value: both replicas' points over the slower replica's time
    assert lines[0]["value"] == pytest.approx(2 * 8192.0**2 / 11e-3 / 1e6)


def test_reference_arm_prints_on_rank_zero_only():
    code = (f"import sys; sys.path.insert(0, {str(ROOT)!r}); import bench; "
            "sys.exit(bench.main(['--impl', 'reference', '--workload', 'tgv2d-256-fp64', "
            "'--steps', '1', '--warmup', '1']))")
    res = _launch(code)
    assert all(r.returncode == 0 for r in res), [r.stderr for r in res]
    assert '"impl": "reference"' in res[0].stdout
    assert res[1].stdout.strip() == ""


SHARD_WORKER = r"""
import json, os, sys, datetime
sys.path.insert(0, {root!r})
import numpy as np
import torch.distributed as dist
from pyspectral_b200.config import Config
from pyspectral_b200.sharding import Comm, ShardedEnsemble
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))

class FakeEnsemble:
    # stands in for the batched GPU engine: per-member rows derived from the configs
    def __init__(self, cfgs):
        self.cfgs = cfgs
        self.steps = []
    def set_states(self, states):
        self.states = states
    def step(self, dt):
        self.steps.append(list(dt))
    def diagnostics(self, klo=0.0, khi=-1.0):
        return np.array([[c.n, c.nu, klo, len(self.steps)] for c in self.cfgs])
    def max_velocity_sum(self):
        return np.array([0.5 * c.n for c in self.cfgs])

members = [Config(n=n, dim=2, nu=1e-3 * (i + 1)) for i, n in enumerate([16, 64, 32, 128, 16, 64, 32])]
se = ShardedEnsemble(members, comm=Comm(), factory=FakeEnsemble)
se.set_states([None] * len(members))
se.step(np.arange(len(members)) * 0.1)
d = se.diagnostics(2.0)
u = se.max_velocity_sum()
mine = se.ens.steps[0] if se.ens is not None else []
dist.destroy_process_group()
print(json.dumps({{"rank": int(os.environ["RANK"]), "diag": d.tolist(), "umax": u.tolist(),
                   "local": se.local, "parts": se.parts, "my_dt": mine, "points": se.local_points}}))
"""


def test_sharded_ensemble_gathers_members_in_global_order():
    import json

    from pyspectral_b200.sharding import partition_by_points

    res = _launch(SHARD_WORKER.format(root=str(ROOT)))
    for r in res:
        assert r.returncode == 0, r.stderr
    out = [json.loads(r.stdout.strip().splitlines()[-1]) for r in res]
    sizes = [16, 64, 32, 128, 16, 64, 32]
    parts = partition_by_points(sizes, 2)
    for o in out:
        assert o["parts"] == parts and o["local"] == parts[o["rank"]]
        # every rank sees every member's row, in the global order
        assert [row[0] for row in o["diag"]] == sizes
        assert [row[1] for row in o["diag"]] == pytest.approx([1e-3 * (i + 1) for i in range(7)])
        assert all(row[2] == 2.0 and row[3] == 1 for row in o["diag"])
        assert o["umax"] == [0.5 * n for n in sizes]
        # each rank stepped exactly its own members with their own dt
        assert o["my_dt"] == pytest.approx([0.1 * i for i in parts[o["rank"]]])
    assert out[0]["points"] + out[1]["points"] == sum(n * n for n in sizes)


def test_partition_by_points_is_balanced_and_complete():
    from pyspectral_b200.sharding import partition_by_points

    sizes = [128] * 64 + [256] * 64 + [512] * 64 + [1024] * 64
    for world in (1, 2, 3, 4, 8):
        parts = partition_by_points(sizes, world)
        assert sorted(i for p in parts for i in p) == list(range(len(sizes)))
        loads = [sum(sizes[i] ** 2 for i in p) for p in parts]
        assert max(loads) - min(loads) <= 1024 ** 2  # within one largest member
        assert parts == partition_by_points(sizes, world)
    assert partition_by_points([16, 16], 4) == [[0], [1], [], []]


MEAN_WORKER = r"""
import json, os, sys, datetime
sys.path.insert(0, {root!r})
import torch, torch.distributed as dist
from pyspectral_b200.sharding import Comm
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
r = int(os.environ["RANK"])
t = torch.full((15440,), float(r + 1))
Comm().allreduce_mean_(t)
dist.destroy_process_group()
print(json.dumps({{"rank": r, "lo": float(t.min()), "hi": float(t.max())}}))
"""


def test_gradient_mean_over_two_ranks():
    import json

    res = _launch(MEAN_WORKER.format(root=str(ROOT)))
    for r in res:
        assert r.returncode == 0, r.stderr
    for o in (json.loads(r.stdout.strip().splitlines()[-1]) for r in res):
        assert o["lo"] == o["hi"] == 1.5


EXCHANGE_WORKER = r"""
import json, os, sys, datetime
sys.path.insert(0, {root!r})
import torch, torch.distributed as dist
from pyspectral_b200.slab import exchange_blocks
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
r, P, nb = dist.get_rank(), dist.get_world_size(), 6
send = torch.zeros(P * nb + 5, dtype=torch.uint8)   # spare tail bytes stay untouched
for p in range(P):
    send[p * nb:(p + 1) * nb] = 10 * r + p             # block p is for rank p
recv = torch.full((P * nb + 5,), 255, dtype=torch.uint8)
exchange_blocks(recv, send, nb, P, dist)
dist.destroy_process_group()
print(json.dumps({{"rank": r, "recv": recv.tolist()}}))
"""


def test_slab_exchange_block_convention():
    import json

    res = _launch(EXCHANGE_WORKER.format(root=str(ROOT)))
    for r in res:
        assert r.returncode == 0, r.stderr
    for o in (json.loads(r.stdout.strip().splitlines()[-1]) for r in res):
        me, nb = o["rank"], 6
        for src in range(2):  # block `src` of my recv came from rank src, aimed at me
            assert o["recv"][src * nb:(src + 1) * nb] == [10 * src + me] * nb
        assert o["recv"][2 * nb:] == [255] * 5
