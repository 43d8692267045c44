"""The multi-GPU path (replicas only) with world_size 2 on the gloo backend:
seeds shifted per rank, the max-over-ranks reduction, the whole-job rate,
and the reference arm's non-zero ranks exiting without work."""
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


def _rank(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    from readdygpu_b200 import replicas
    try:
        assert replicas.env() == (ws, rank, rank)
        assert replicas.init("gloo", timeout_s=60)
        replicas.barrier(cuda_sync=False)
        # every rank sees the slowest rank's time
        m = replicas.max_over_ranks(10.0 + rank)
        boxes = replicas.replica_boxes([((0, 0, 0), (1, 1, 1), (1, 1, 1), 100), ((0, 0, 0), (2, 2, 2), (1, 1, 1), 200)],
                                       rank)
        rate = replicas.job_rate(1000, ws, 50, m / 1e3)
        q.put((rank, m, [b[3] for b in boxes], replicas.replica_seed(11, rank), rate))
    finally:
        replicas.finalize()


def test_two_ranks_gloo():
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(ws))
    assert [g[1] for g in got] == [11.0, 11.0]                      # max over ranks
    assert got[0][2] == [100, 200] and got[1][2] == [100 + 7919, 200 + 7919]
    assert got[0][3] != got[1][3]
    # 2 ranks x 1000 particles x 50 steps over the slowest rank's 11 ms
    assert abs(got[0][4] - 2 * 1000 * 50 / 0.011) < 1e-6 * got[0][4]


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "3", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
