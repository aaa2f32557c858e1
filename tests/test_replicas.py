"""The replica plumbing of bench.py on CPU (no GPU): two gloo ranks, the slowest rank's time,
the whole-job rate, and the reference arm's other ranks leaving without output."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench

    r, w, dist = bench.init_replicas("gloo", timeout_s=60)
    try:
        slow = bench.max_over_ranks(1.0 + 0.5 * r, dist)  # rank 1 is the slower replica
        out.put((r, w, slow, bench.job_rate(w, 1000, 10, slow)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_replicas_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[:3] for r in res] == [(0, 2, 1.5), (1, 2, 1.5)]
    assert res[0][3] == pytest.approx(2 * 1000 * 10 / 1.5 / 1e6)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench

    env = {k: os.environ.pop(k) for k in ("WORLD_SIZE", "RANK") if k in os.environ}
    try:
        assert bench.init_replicas("gloo")[1:] == (1, None)
        assert bench.max_over_ranks(2.5, None) == 2.5
    finally:
        os.environ.update(env)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1", MASTER_PORT="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0 and r.stdout.strip() == ""
