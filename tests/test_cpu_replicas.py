"""The multi-GPU path is replicas (pairs are independent; no data-path
collective): each rank scores its own pairs and the whole-job rate is taken
over the slowest rank.  These run the bench's replica helpers in two gloo
ranks on the CPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ms = 10.0 * (rank + 1)  # rank 1 is the slow one
        slowest = bench.max_over_ranks(ms, dist, "cpu")
        rate = bench.whole_job_rate(world, 64, 5, slowest)
        q.put((rank, bench.replica_offset(rank, 64), slowest, rate))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, off0, s0, v0), (r1, off1, s1, v1) = out
    assert (off0, off1) == (0, 64)          # disjoint pairs per replica
    assert s0 == s1 == 20.0                 # both ranks report the slowest time
    assert v0 == v1 == pytest.approx(2 * 64 * 5 / 0.020)


def test_single_rank_needs_no_collective():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(7.5, None, "cpu") == 7.5
    assert bench.whole_job_rate(1, 64, 20, 132.0) == pytest.approx(64 * 20 / 0.132)
