"""The multi-GPU path is replicas only: each rank solves its own batch and the
only collective is the max over ranks of the timings.  Checked here with two
gloo ranks on CPU (127.0.0.1)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = 100.0 + 25.0 * rank                       # rank 1 is the slower replica
    got = bench.max_over_ranks(ms, dist, "cpu")
    seed = bench.replica_seed(2, rank)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, got, seed))


def test_two_gloo_ranks_take_the_max_and_solve_different_batches():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [125.0, 125.0]
    assert out[0][2] != out[1][2]


def test_single_process_has_no_collective():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
