"""The N>1 bench path on CPU: world_size-2 gloo ranks.  bench.py runs one
replica per rank (queries are independent, no data-path collective); the only
collectives are the barriers and the max-over-ranks of the timed region, and
the reference arm runs on rank 0 alone."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        # rank r "took" (r + 1) ms; every rank must see the slowest one
        ms = bench.max_over_ranks(float(rank + 1), dist, "cpu")
        steps, nq = 3, 100
        value = world * nq * steps / (ms / 1e3)
        q.put((rank, ms, value))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert [g[1] for g in got] == [2.0, 2.0]
    assert got[0][2] == got[1][2] == pytest.approx(2 * 100 * 3 / 2e-3)


def test_max_over_ranks_single_process():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(1.5, None, "cpu") == 1.5


def test_reference_arm_nonzero_rank_exits_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
