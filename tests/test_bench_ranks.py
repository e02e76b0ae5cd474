"""CPU tests of bench.py's multi-rank logic (one rank per GPU on the B200,
run here as world_size-2 gloo ranks): the job time is the max over ranks, the
value aggregates all ranks' replicas, and the reference arm runs on rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, local_ms, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.job_time_ms(local_ms, world, "cpu")
        v = bench.replicas_value(1000, 10, ms, world)
        out.put((rank, ms, v))
    finally:
        dist.destroy_process_group()


def test_job_time_is_max_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, [12.5, 20.0][r], q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, v in got:
        assert ms == 20.0
        assert v == pytest.approx(2 * 1000 * 10 / 20.0e-3)


def test_single_rank_value():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.job_time_ms(7.0, 1, "cpu") == 7.0
    assert bench.replicas_value(512 ** 3, 100, 220.0, 1) == pytest.approx(512 ** 3 * 100 / 0.22)


def test_reference_arm_prints_only_on_rank_0():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_reference_arm_line_on_rank_0_small_grid():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--grid", "32", "32",
                        "32", "--steps", "2", "--warmup", "1"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
    # the same config dict as the repo arm's line for the same grid and GPU count
    sys.path.insert(0, ROOT)
    import bench
    assert line["config"] == bench.solve_config((32, 32, 32), "fp64", 1)
