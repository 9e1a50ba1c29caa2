"""bench.py's multi-replica bookkeeping, run as two gloo ranks on CPU: the
job's time is the slowest replica's and its work is the sum over replicas;
the reference arm runs on rank 0 only and the other ranks leave quietly."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        # rank r: ms = 10 + r, node-steps = 1000 * (r + 1), e2e 20 + r, 500 * (r + 1)
        res = bench.reduce_over_ranks([10.0 + rank, 1000.0 * (rank + 1), 20.0 + rank,
                                       500.0 * (rank + 1)], world, "cpu")
        out.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_reduce_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        assert res[r] == (11.0, 3000.0, 21.0, 1500.0)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "1"], env=env, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
