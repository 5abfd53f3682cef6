"""CPU tests of bench.py's multi-rank logic with the gloo backend, world
size 2: every rank takes the same collective steps, the timed region is the
max over ranks, the tile list is partitioned over the ranks by coded bytes
(every tile on exactly one rank), and only rank 0 runs and prints the
reference arm."""
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


def test_tile_list_partition_by_coded_bytes_with_gloo():
    """Two ranks shard a global list of uneven tiles: each encodes its
    round-robin candidates, the coded sizes are all-gathered, both compute
    the same balanced shards; every tile lands on exactly one rank, each
    rank holds exactly the codestreams of its shard, and the ranks' coded
    bytes differ by less than the largest tile."""
    outs = _run_ranks("""
        import datetime, json
        import torch.distributed as dist
        import bench
        from signinum_b200.shard import shard_tiles
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
        n_total = 24
        idx, tiles, summary = shard_tiles(dist, n_total, lambda ix: bench.build_workload("c2", n_total, ix)[0])
        ref = bench.build_workload("c2", n_total, idx)[0]
        same = all(a.codestream == b.codestream for a, b in zip(tiles, ref))
        print(json.dumps({"rank": dist.get_rank(), "idx": idx, "same": same, "summary": summary,
                          "bytes": sum(len(t.codestream) for t in tiles)}))
        dist.destroy_process_group()
    """, timeout=300)
    rows = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    idx = sorted(i for r in rows for i in r["idx"])
    assert idx == list(range(24)), "every tile exactly once"
    assert all(r["same"] for r in rows)
    assert rows[0]["summary"] == rows[1]["summary"], "both ranks agree on the shards"
    loads = rows[0]["summary"]["coded_bytes_per_rank"]
    assert [r["bytes"] for r in sorted(rows, key=lambda r: r["rank"])] == loads
    from signinum_b200 import encode

    largest = max(len(t.codestream) for t in encode.config2(24).tiles)
    assert abs(loads[0] - loads[1]) < largest


def test_balance_by_coded_bytes_bounds_and_determinism():
    import numpy as np

    from signinum_b200.shard import balance_by_coded_bytes

    rng = np.random.default_rng(5)
    for world in (2, 3, 8):
        sizes = [int(x) for x in rng.integers(1, 1 << 20, size=500)]
        shards = balance_by_coded_bytes(sizes, world)
        assert sorted(i for s in shards for i in s) == list(range(500))
        loads = [sum(sizes[i] for i in s) for s in shards]
        assert max(loads) - min(loads) < max(sizes)
        assert shards == balance_by_coded_bytes(sizes, world)
    assert balance_by_coded_bytes([0, 0, 0], 2) == [[0, 2], [1]]
