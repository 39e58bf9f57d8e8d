"""Multi-GPU host logic on the CPU: world_size-2 gloo process groups run the replica
sharding and the measurement reductions bench.py uses for N GPUs, and the in-process
Router spreads jobs over engines (fakes here) by queued work."""
import os
import socket

import pytest

from tipl_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r, lr, w = replicas.env_rank()
        jobs = list(range(11))
        mine = replicas.shard(jobs, r, w)
        # each rank "times" its share: the job time is the max over ranks
        t = 1.5 + r
        tmax = replicas.max_over_ranks(t, dist)
        total = replicas.sum_over_ranks(len(mine), dist)
        all_jobs = replicas.gather_lists(mine, dist)
        lat = replicas.gather_lists([10.0 * r + k for k in range(len(mine))], dist)
        dist.barrier()
        q.put((r, lr, w, mine, tmax, total, all_jobs, lat))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_sharding_and_reductions():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    (r0, l0, w0, m0, t0, n0, a0, lat0), (r1, l1, w1, m1, t1, n1, a1, lat1) = out
    assert (r0, r1, w0, w1, l0, l1) == (0, 1, 2, 2, 0, 1)
    assert m0 == [0, 2, 4, 6, 8, 10] and m1 == [1, 3, 5, 7, 9]
    assert t0 == t1 == 2.5                      # max over ranks, seen by both
    assert n0 == n1 == 11                       # every job exactly once
    assert a0 == a1 == m0 + m1                  # gathered in rank order
    assert lat0 == lat1 and len(lat0) == 11


def test_single_process_defaults():
    assert replicas.shard(list(range(5)), 0, 1) == list(range(5))
    assert replicas.max_over_ranks(3.0) == 3.0
    assert replicas.gather_lists([1, 2]) == [1, 2]


class _FakeEngine:
    def __init__(self):
        self.jobs = {}
        self.next = 1

    def submit(self, moving, **k):
        jid = self.next
        self.next += 1
        self.jobs[jid] = moving
        return jid

    def wait(self, jid):
        return {"status": 0, "moving": self.jobs.pop(jid)}


def test_router_least_queued_work():
    import numpy as np

    engines = [_FakeEngine(), _FakeEngine()]
    r = replicas.Router(engines)
    big, small = np.zeros(1000), np.zeros(10)
    h1 = r.submit(big)          # engine 0
    h2 = r.submit(small)        # engine 1 (less work)
    h3 = r.submit(small)        # engine 1 again (20 < 1000)
    assert (h1[0], h2[0], h3[0]) == (0, 1, 1)
    assert r.wait(h1)["moving"] is big
    h4 = r.submit(small)        # engine 0 is empty now
    assert h4[0] == 0
    for h in (h2, h3, h4):
        assert r.wait(h)["status"] == 0
    assert r.load == [0.0, 0.0]
