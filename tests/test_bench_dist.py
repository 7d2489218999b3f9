"""bench.py's multi-GPU form on the CPU: N independent replicas, one process per rank, joined only by
the barriers around the timed region and the max over ranks of the elapsed time (world size 2 over
gloo, rendezvous on 127.0.0.1).  The reference arm runs on rank 0 alone; other ranks exit at once."""
import multiprocessing as mp
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, port: int, q):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench
    world, r, _ = bench.dist_setup(2, backend="gloo")
    bench.barrier(world)
    slowest = bench.max_over_ranks(10.0 + 5.0 * r, world)  # rank 1 is the slower replica
    bench.barrier(world)
    q.put((r, world, slowest))
    dist.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(600)  # a fresh machine's first torch import can take a minute
    for p in procs:
        if p.is_alive():
            p.kill()
    assert [p.exitcode for p in procs] == [0, 0]
    got = sorted(q.get(timeout=30) for _ in procs)
    assert got == [(0, 2, 15.0), (1, 2, 15.0)]


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    env = dict(os.environ)
    os.environ.pop("WORLD_SIZE", None)
    try:
        assert bench.dist_setup(1, backend="gloo") == (1, 0, 0)
        assert bench.max_over_ranks(3.5, 1) == 3.5
        bench.barrier(1)  # nothing to join
    finally:
        os.environ.clear()
        os.environ.update(env)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""  # rank 0 alone prints the line
