"""The multi-GPU form of the batched workload on CPU: 48 independent instances
split whole across ranks (plan.shard_instances), no exchange between ranks.
Every rank computes the same split on its own; here two and three `gloo`
ranks run as child processes on 127.0.0.1 in place of the NCCL ranks and
gather their shares, which must cover every instance exactly once with
balanced cell counts, and the whole-job value counts all instances over the
slowest rank's time."""
import json
import os
import subprocess
import sys

import pytest

from gsvit_copy_b200 import plan
from tests.test_replicas import ROOT, _env, _free_port, _run

CHILD = r"""
import json, sys
sys.path.insert(0, {root!r})
import torch.distributed as dist
import bench
from gsvit_copy_b200 import plan
r = bench.Replicas("gloo")
cells = [a * b * c for a, b, c in (p["shape"] for p in plan.batch_params(48))]
mine = plan.shard_instances(cells, r.world)[r.rank]
got = [None] * r.world
dist.all_gather_object(got, mine)
ms = r.max(10.0 + r.rank)
r.barrier()
r.close()
print(json.dumps({{"rank": r.rank, "mine": mine, "all": got, "max_ms": ms,
                   "value": sum(cells) * 20 / (ms * 1e-3) / 1e9}}))
"""


def _cells():
    return [a * b * c for a, b, c in (p["shape"] for p in plan.batch_params(48))]


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_split_covers_every_instance_once_and_balances(world):
    cells = _cells()
    shards = plan.shard_instances(cells, world)
    assert len(shards) == world
    flat = sorted(q for s in shards for q in s)
    assert flat == list(range(len(cells)))
    loads = [sum(cells[q] for q in s) for s in shards]
    # longest-processing-time bound: no rank exceeds the mean by more than the largest instance
    assert max(loads) <= sum(cells) / world + max(cells)
    assert all(s == sorted(s) for s in shards)
    assert plan.shard_instances(cells, world) == shards   # deterministic


def test_batch_params_match_batch_scene_shapes():
    ps = plan.batch_params(4)
    scenes = plan.batch_scenes(4, nsteps=10)
    assert [p["shape"] for p in ps] == [(s.xres, s.yres, s.zres) for s in scenes]


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_agree_on_the_split(world):
    port = _free_port()
    procs = [subprocess.Popen([sys.executable, "-c", CHILD.format(root=ROOT)], cwd=ROOT, text=True,
                              stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                              env=_env(RANK=r, LOCAL_RANK=r, WORLD_SIZE=world, MASTER_ADDR="127.0.0.1",
                                       MASTER_PORT=port))
             for r in range(world)]
    outs = _run(procs)
    res = []
    for p, (out, err) in zip(procs, outs):
        assert p.returncode == 0, err[-2000:]
        res.append(json.loads(out.strip().splitlines()[-1]))
    cells = _cells()
    expect = plan.shard_instances(cells, world)
    for d in res:
        assert d["all"] == expect
        assert d["mine"] == expect[d["rank"]]
        assert d["max_ms"] == 10.0 + (world - 1)
        assert abs(d["value"] - sum(cells) * 20 / ((10.0 + world - 1) * 1e-3) / 1e9) < 1e-9
