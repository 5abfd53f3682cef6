"""CPU tests of bench.py's multi-rank logic with the gloo backend, world
size 2: every rank takes the same collective steps, the timed region is the
max over ranks, the job value sums the replicas, and only rank 0 runs and
prints the reference arm."""
import json
import os
import socket
import subprocess
import sys
import textwrap
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run_ranks(code, world=2, timeout=120):
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), PYTHONPATH=str(ROOT))
        procs.append(subprocess.Popen([sys.executable, "-c", textwrap.dedent(code)], env=env, cwd=ROOT,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=timeout)
        assert p.returncode == 0, err
        outs.append(out)
    return outs


def test_max_over_ranks_and_replica_value_with_gloo():
    outs = _run_ranks("""
        import datetime, json, os
        import torch.distributed as dist
        import bench
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
        r = dist.get_rank()
        ms = 10.0 + 5.0 * r          # rank 1 is the slow replica
        worst = bench.reduce_max(dist, ms, "cpu")
        dist.barrier()
        v = bench.replica_throughput(dist.get_world_size(), 67108864, worst)
        print(json.dumps({"rank": r, "worst": worst, "value": v}))
        dist.destroy_process_group()
    """)
    rows = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert {r["rank"] for r in rows} == {0, 1}
    assert all(r["worst"] == 15.0 for r in rows)
    # Two replicas of 67.1 Mpixel each in 15 ms: 8947.8 Mpixel/s for the job.
    assert all(abs(r["value"] - 2 * 67108864 / 0.015 / 1e6) < 1e-6 for r in rows)


def test_reduce_max_without_process_group_is_identity():
    import bench

    assert bench.reduce_max(None, 3.25, "cpu") == 3.25


def test_reference_arm_prints_only_on_rank_zero():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2", PYTHONPATH=str(ROOT))
    p = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "0"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""
