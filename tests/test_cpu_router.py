"""The multi-GPU job router (turbo-metrics_b200/router.py) on the CPU.

The policy is checked directly (reference-cache affinity, least outstanding
bytes, dropping a rank).  Then three gloo ranks run the real front end and
worker loop with a fake engine that records which jobs it scored: jobs are
routed by affinity and balance, and a rank that leaves between steps has its
jobs of that step routed again to the ranks that are left, so every job is
scored exactly once.  No GPU is involved; the failure is a process that
exits on the host."""
import os
import socket
import sys
import time

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "turbo-metrics_b200")


def _router():
    sys.path.insert(0, PKG)
    import router
    return router


def test_policy_affinity_then_least_outstanding_bytes():
    R = _router()
    pol = R.RoutingPolicy(3)
    big = lambda i, ref: R.Job(i, ref, 1920, 1080, 4)
    small = lambda i, ref: R.Job(i, ref, 128, 128, 1)
    # three new references: an empty rank each, lowest rank first
    assert [pol.pick(big(i, 10 + i)) for i in range(3)] == [0, 1, 2]
    # the same references again: same ranks, whatever the load
    assert [pol.pick(small(3 + i, 10 + i)) for i in range(3)] == [0, 1, 2]
    assert pol.pick(big(6, 10)) == 0
    # a new reference goes to the least loaded rank (rank 0 now has two big jobs)
    assert pol.pick(small(7, 99)) == 1
    # finishing work moves the balance
    pol.done(0, big(0, 10))
    pol.done(0, big(6, 10))
    assert pol.pick(small(8, 100)) == 0
    assert sum(pol.outstanding) == sum(j.nbytes for j in [big(1, 0), big(2, 0), small(3, 0), small(4, 0),
                                                            small(5, 0), small(7, 0), small(8, 0)])


def test_policy_drop_forgets_the_rank():
    R = _router()
    pol = R.RoutingPolicy(3)
    for i in range(6):
        pol.pick(R.Job(i, i % 3, 64, 64, 1))
    assert pol.affinity == {0: 0, 1: 1, 2: 2}
    pol.drop(1)
    assert 1 not in pol.affinity.values()
    picks = [pol.pick(R.Job(10 + i, i % 3, 64, 64, 1)) for i in range(6)]
    assert 1 not in picks
    assert picks[0] == 0 and picks[2] == 2
    pol.drop(0)
    pol.drop(2)
    with pytest.raises(RuntimeError):
        pol.pick(R.Job(99, 5, 8, 8, 1))


class FakeEngine:
    """Scores a job as ref_id * 1000 + candidate index; records what it saw.
    With `leave_at_step`, the rank exits before scoring that step."""

    def __init__(self, rank, leave_at_step=None):
        self.rank, self.leave_at_step, self.step, self.seen = rank, leave_at_step, 0, []

    def score(self, jobs):
        if self.leave_at_step is not None and self.step == self.leave_at_step:
            os._exit(0)  # leaves between steps: nothing of this step was scored
        self.step += 1
        self.seen.extend(j.job_id for j in jobs)
        time.sleep(0.05)
        return {j.job_id: [j.ref_id * 1000.0 + k for k in range(j.n_candidates)] for j in jobs}


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q, leave_rank, leave_step):
    from datetime import timedelta
    import torch.distributed as dist
    R = _router()
    store = dist.TCPStore("127.0.0.1", port, world, rank == 0, timedelta(seconds=60))
    dist.init_process_group("gloo", store=store, rank=rank, world_size=world, timeout=timedelta(seconds=30))
    dist.barrier()  # every rank joined; no collective after this (a rank may leave)
    eng = FakeEngine(rank, leave_step if rank == leave_rank else None)
    if rank != 0:
        R.worker_loop(store, rank, eng, poll_s=60.0)
        q.put(("worker", rank, eng.seen))
        return
    fe = R.FrontEnd(store, world, eng, deadline_s=3.0)
    mk = lambda base: [R.Job(base + i, i % 6, 320 + 16 * (i % 4), 240, 1 + i % 3) for i in range(12)]
    res_a = fe.run_step(mk(0))
    place_a = {jid: fe.placement[jid] for jid in res_a}
    res_b = fe.run_step(mk(100))
    place_b = {jid: fe.placement[jid] for jid in res_b}
    fe.stop()
    q.put(("front", res_a, place_a, res_b, place_b, fe.dropped, sorted(fe.policy.alive), eng.seen))


def test_three_gloo_ranks_affinity_balance_and_a_rank_leaving():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world, leave_rank, leave_step = 3, 2, 1
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q, leave_rank, leave_step)) for r in range(world)]
    for p in procs:
        p.start()
    msgs = [q.get(timeout=120) for _ in range(world - 1)]  # the leaving rank reports nothing
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    front = [m for m in msgs if m[0] == "front"][0]
    _, res_a, place_a, res_b, place_b, dropped, alive, seen0 = front
    # every job scored exactly once, with its engine's answer
    for base, res in ((0, res_a), (100, res_b)):
        assert sorted(res) == [base + i for i in range(12)]
        for i in range(12):
            assert res[base + i] == [(i % 6) * 1000.0 + k for k in range(1 + i % 3)]
    # step A: all three ranks took work; a reference's jobs share one rank
    assert set(place_a.values()) == {0, 1, 2}
    for i in range(6):
        assert place_a[i] == place_a[i + 6]
    # step B: rank 2 scored front-end step 0 and left at step 1; its jobs of
    # step 1 went, in step 2, to the ranks that are left
    assert dropped == [(1, 2)] and alive == [0, 1]
    assert set(place_b.values()) <= {0, 1}
    for i in range(12):
        if place_a[i] != 2:
            assert place_b[100 + i] == place_a[i]  # affinity kept for live ranks
    worker1 = [m for m in msgs if m[0] == "worker"][0]
    assert worker1[1] == 1
    scored = sorted(seen0 + worker1[2])
    want = sorted([i for i in range(12) if place_a[i] != 2] + [100 + i for i in range(12)])
    assert scored == want  # ranks 0 and 1 scored each of their jobs once
