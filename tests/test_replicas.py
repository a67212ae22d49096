"""The multi-GPU (replicas) bookkeeping of bench.py on CPU: two gloo ranks.

Each replica sorts its own data; the job's time is the slowest rank's, taken
with an all-reduce MAX. The GPU run uses NCCL; the reduction is the same."""
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, ROOT)
    import bench

    slowest = bench.max_over_ranks(10.0 + rank)  # each rank's own "ms"
    ok = bench.max_over_ranks(0.0 if rank == 0 else 1.0) == 0.0  # rank 1 failed its check
    q.put((rank, slowest, ok))
    dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == [(0, 11.0, False), (1, 11.0, False)]


def test_max_over_ranks_without_a_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.5) == 3.5


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""
