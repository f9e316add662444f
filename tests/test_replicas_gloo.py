"""The N-GPU bench path on CPU: two ranks over gloo (replicas, no data-path
collective) -- the barrier, the max over ranks of a time, and rank 0 alone
reporting; the reference arm's non-zero ranks exit without work."""
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from attract_b200 import replicas

    R = replicas.init("gloo", timeout_s=60)
    replicas.barrier(R)
    t = replicas.max_over_ranks(R, 1.0 + 3.0 * rank)  # each rank's own "time"
    out[rank] = (R.rank, R.world, R.leader, t)
    replicas.finish(R)


def test_two_gloo_ranks_take_the_max_time():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert sorted(res) == [0, 1]
    for r, (rank, w, leader, t) in res.items():
        assert rank == r and w == world and leader == (r == 0)
        assert t == 4.0  # the max over ranks, on every rank


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    from attract_b200 import replicas

    env = {k: os.environ.pop(k) for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK") if k in os.environ}
    try:
        R = replicas.init("gloo")
        assert (R.rank, R.world, R.leader) == (0, 1, True)
        assert replicas.max_over_ranks(R, 2.5) == 2.5
        replicas.barrier(R)
        replicas.finish(R)
    finally:
        os.environ.update(env)


def test_reference_arm_non_leader_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""
