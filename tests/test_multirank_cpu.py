"""The N > 1 path of bench.py on CPU with two gloo ranks. The single-domain step has no
exchange step, so N GPUs run N independent replicas: the only collective is the
max over ranks of the timed region (the slowest replica bounds the job), and the whole-job
value counts every rank's cells. The reference arm runs on rank 0 alone; other ranks exit
without work."""
import os
import socket
import subprocess
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = [12.5, 20.0][rank]  # rank 1 is the slow replica
        max_ms = bench.max_over_ranks(ms, world)
        q.put((rank, max_ms, bench.job_throughput(world, 1000, 10, max_ms)))
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank_and_count_every_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [20.0, 20.0]
    # 2 ranks x 1000 cells x 10 steps in 20 ms
    assert got[0][2] == pytest.approx(2 * 1000 * 10 / 0.020 / 1e6)


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks(3.25, 1) == 3.25


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""
