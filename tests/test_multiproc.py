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
