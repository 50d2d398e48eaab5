"""Multi-process host logic of bench.py on CPU (gloo, world size 2).

The solve does not shard: N GPUs run N independent replicas, each on its own
seeded batch of orientations of the same target, and the job time is the
maximum over ranks.  No data-path collective exists; the only collectives are
the barrier and the max of the timed region."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import sys

    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(dist, 0)
        slowest = bench.max_over_ranks(dist, 1.5 + rank)

        class A:
            n, orient = 8, 2

        prob, b, adia = bench.workload(A, rank)
        q.put((rank, slowest, prob.nat0, b.shape, float(abs(b).sum())))
        bench.barrier(dist, 0)
    finally:
        dist.destroy_process_group()


def test_replicas_max_over_ranks_and_distinct_batches():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        r, slowest, nat0, shape, bsum = q.get(timeout=120)
        out[r] = (slowest, nat0, shape, bsum)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0] == pytest.approx(2.5)  # max over ranks
    assert out[0][1] == out[1][1] and out[0][2] == out[1][2] == (4, 3 * 8 ** 3)  # same target and batch shape
    assert out[0][3] != out[1][3]  # per-rank orientation seeds
