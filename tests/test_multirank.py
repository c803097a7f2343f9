"""The N > 1 path of bench.py on CPU: two gloo ranks stand in for two GPUs.
Each rank runs its own replica, so the only exchange is the max over ranks
of the timed region, and the reference arm runs on rank 0 alone."""
import json
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, values, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out[rank] = bench.reduce_max_over_ranks(values[rank], world, "cpu")
    finally:
        dist.destroy_process_group()


def test_the_slowest_rank_sets_the_time():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_rank, args=(r, world, 29517, [3.5, 7.25], out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert dict(out) == {0: 7.25, 1: 7.25}


def test_whole_job_rate_is_weak_scaling():
    sys.path.insert(0, ROOT)
    import bench
    one = bench.whole_job_gbs(61.44e9, 1, 22.0)
    assert bench.whole_job_gbs(61.44e9, 4, 22.0) == pytest.approx(4 * one)
    assert one == pytest.approx(61.44e9 / 0.022 / 1e9)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "0", "--N", "4096", "--k", "8"], cwd=ROOT, env=env, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""
    env["RANK"] = "0"
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "0", "--N", "4096", "--k", "8"], cwd=ROOT, env=env, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
