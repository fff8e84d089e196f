"""bench.py's multi-process path on the CPU: two gloo ranks stand in for two GPUs.  Each
replica solves independently; the job's time is the slowest rank's, taken with one
all-reduce, and the whole-job throughput counts every rank's solves.  The reference arm
under torchrun runs on rank 0 only."""
import json
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = [120.0, 80.0][rank]
    total = bench.max_over_ranks(ms, world, dist, torch, "cpu")
    q.put((rank, total, bench.replicas_value(9, world, total)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, total, value in got:
        assert total == 120.0
        assert value == pytest.approx(2 * 9 / 0.120)


def test_reference_arm_runs_on_rank_zero_only(tmp_path):
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0 and r.stdout.strip() == ""
    # rank 0 alone runs the arm; here on a 4^3 mesh of the same workload, so it takes seconds
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--n", "4"], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    if "unavailable" in line:
        pytest.skip("the reference solver is not built here: " + line["unavailable"])
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "reference"
    assert line["steps"] == 2 * line["processes"] and line["e2e"]["h2d_bytes_per_step"] == 0
