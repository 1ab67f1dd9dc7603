"""The multi-GPU path of bench.py on CPU: two replica ranks over gloo
(127.0.0.1) agree on the slowest rank's time and on the whole-job rate,
and the reference arm on a non-zero rank exits without work or output."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = [12.5, 17.25][rank]  # the second replica is slower
        ms_max = bench.max_over_ranks(ms, world, "cpu")
        rate = bench.replica_rate(world, 200, 16777216, ms_max)
        out.put((rank, ms_max, rate))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[1] for g in got] == [17.25, 17.25]
    expect = 2 * 200 * 3 * 16777216 / (17.25e-3)
    assert all(abs(g[2] - expect) <= 1e-9 * expect for g in got)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
    assert bench.replica_rate(1, 10, 100, 1.0) == 10 * 3 * 100 / 1e-3


def test_reference_arm_on_a_nonzero_rank_is_silent():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
