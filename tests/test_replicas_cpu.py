"""bench.py's multi-rank plumbing on CPU: two gloo ranks, independent
replicas, timings combined as the max over ranks; the reference arm prints
only on rank 0."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    r, w, _, dist = bench.dist_setup(world, backend="gloo")
    ms = 100.0 + 50.0 * r  # rank 1 is the slow one
    mx = bench.max_over_ranks(ms, dist)
    q.put((r, w, mx, bench.replica_rate(w, 5, mx)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
    assert all(p.exitcode == 0 for p in ps)
    out = sorted(q.get(timeout=10) for _ in range(2))
    for r, w, mx, rate in out:
        assert w == 2 and mx == 150.0
        assert abs(rate - 2 * 5 / 0.150) < 1e-9


def test_reference_arm_silent_on_other_ranks():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
