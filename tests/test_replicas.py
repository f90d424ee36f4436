"""The N-rank path of bench.py on CPU.  The time step does not shard, so an
N-GPU run is N independent replicas (one process per GPU under torchrun) that
share only a barrier around the timed region and the slowest rank's time;
`value` counts every rank's cell updates over that time.  Here two `gloo`
ranks run as child processes on 127.0.0.1 in place of the NCCL ranks."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
sys.path.insert(0, {root!r})
import bench
r = bench.Replicas("gloo")
r.barrier()
m = r.max(1.5 * (r.rank + 1))
v = bench.whole_job_gcells(1e9, 10, r.world, 2.0)
r.barrier()
r.close()
print(json.dumps({{"rank": r.rank, "world": r.world, "max": m, "value": v}}))
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(**kw):
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "LOCAL_RANK", "WORLD_SIZE", "MASTER_ADDR",
                                                            "MASTER_PORT")}
    env.update({k: str(v) for k, v in kw.items()})
    return env


def _run(procs, timeout=180):
    outs = []
    try:
        for p in procs:
            outs.append(p.communicate(timeout=timeout))
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    return outs


def test_two_gloo_replicas_share_barrier_and_slowest_time():
    port = _free_port()
    procs = [subprocess.Popen([sys.executable, "-c", CHILD.format(root=ROOT)], cwd=ROOT, text=True,
                              stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                              env=_env(RANK=r, LOCAL_RANK=r, WORLD_SIZE=2, MASTER_ADDR="127.0.0.1", MASTER_PORT=port))
             for r in (0, 1)]
    outs = _run(procs)
    for p, (out, err) in zip(procs, outs):
        assert p.returncode == 0, err
    lines = [json.loads(out.strip().splitlines()[-1]) for out, _ in outs]
    assert sorted(x["rank"] for x in lines) == [0, 1]
    for x in lines:
        assert x["world"] == 2
        assert x["max"] == 3.0                  # the slower rank's figure reaches both
        assert x["value"] == 10.0               # 1e9 cells x 10 steps x 2 ranks / 2 s


def test_one_rank_initialises_nothing():
    out = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT)], cwd=ROOT, text=True, capture_output=True,
                         env=_env(), timeout=180)
    assert out.returncode == 0, out.stderr
    x = json.loads(out.stdout.strip().splitlines()[-1])
    assert x == {"rank": 0, "world": 1, "max": 1.5, "value": 5.0}


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun the reference arm's other ranks exit 0 without work or output."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                         cwd=ROOT, text=True, capture_output=True, timeout=180,
                         env=_env(RANK=1, LOCAL_RANK=1, WORLD_SIZE=2, MASTER_ADDR="127.0.0.1",
                                  MASTER_PORT=_free_port()))
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == ""


def test_reference_arm_prints_the_contract_line():
    """Rank 0 of the reference arm times GSvit's own CPU code on a bounded
    sample and prints one JSON line with the bench contract's keys."""
    import pytest
    from oracle.pyoracle import reference_available
    if not reference_available():
        pytest.skip("GSvit's CPU build (oracle/_ref) is not built here")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3"], cwd=ROOT, text=True, capture_output=True, timeout=600, env=_env())
    assert out.returncode == 0, out.stderr
    lines = [x for x in out.stdout.strip().splitlines() if x.startswith("{")]
    assert len(lines) == 1
    x = json.loads(lines[0])
    assert x["impl"] == "reference" and x["metric"] == "Gcell-updates/s" and x["unit"] == "Gcell/s"
    assert x["higher_is_better"] is True and x["steps"] == 1 and x["warmup"] == 3 and x["value"] > 0
    cb = x["cpu_baseline"]
    assert cb["value"] == x["value"] and cb["unit"] == x["unit"] and cb["cores"] >= 1
    assert cb["kind"] in ("reference", "port") and cb["sample"]
    assert x["e2e"] == {"value": x["value"], "unit": x["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "workload" in x["config"]
