"""Multi-rank host logic on CPU (gloo, world size 2): the beam partition
every rank computes independently must agree across ranks, cover every beam
once and balance the work; step times are reduced as the maximum over ranks
(the bench's rule).  No GPU and no collective on the data path."""
from __future__ import annotations

import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    """A port nothing listens on now (each run gets its own, so a store that
    is still closing from an earlier test cannot collide with it)."""
    import socket
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _worker(rank, world, port, q):
    sys.path.insert(0, os.path.join(ROOT, "astro-accelerate_b200"))
    import torch
    import torch.distributed as dist
    import aa_b200 as aa
    from aa_b200 import workloads as WL
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        beams = WL.multibeam_draw(seed=3, nbeams=12)
        costs = []
        for b in beams:
            s = aa.strategy(b["plan"], b["nchans"], b["nsamp"], b["fch1"], b["foff"], b["tsamp"], b["nbits"],
                            64 << 30)
            costs.append(WL.beam_cost(b, s))
        mine = WL.partition(costs, world)[rank]
        got = [None] * world
        dist.all_gather_object(got, mine)
        t = torch.tensor([float(rank + 1)])
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        q.put((rank, got, costs, float(t)))
    finally:
        dist.destroy_process_group()


def test_partition_agrees_across_ranks_and_covers_every_beam():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    parts = res[0][1]
    assert all(r[1] == parts for r in res)  # every rank computed the same partition
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(12))
    costs = res[0][2]
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) <= sum(loads) / world + max(costs)  # LPT bound
    assert all(r[3] == float(world) for r in res)  # max over ranks


def test_partition_single_rank():
    sys.path.insert(0, os.path.join(ROOT, "astro-accelerate_b200"))
    from aa_b200 import workloads as WL
    assert WL.partition([3.0, 1.0, 2.0], 1) == [[0, 1, 2]]
    assert WL.partition([5.0, 4.0, 3.0, 3.0], 2) == [[0, 3], [1, 2]]


def _queue_worker(rank, world, port, nbeams, die_rank, q):
    """Beams from aa_b200.beamqueue over a TCPStore; rank `die_rank` takes one
    beam and exits without finishing it (a rank that stops mid-beam)."""
    sys.path.insert(0, os.path.join(ROOT, "astro-accelerate_b200"))
    import hashlib
    import time
    from datetime import timedelta

    import torch.distributed as dist
    from aa_b200.beamqueue import BeamQueue

    store = dist.TCPStore("127.0.0.1", port, world, rank == 0, timeout=timedelta(seconds=60))
    bq = BeamQueue(store, nbeams, rank, lease_s=1.5)

    def work(i):
        time.sleep(0.05)
        return hashlib.sha256(f"beam-{i}".encode()).hexdigest()

    if rank == die_rank:
        bq._claim_next()
        os._exit(0)  # stops holding a lease: no done mark, no renewal
    mine = bq.run(work, timeout_s=120)
    results = {i: bq.result(i).decode() for i in range(nbeams)} if rank == 0 else None
    q.put((rank, mine, results, bq.ndone()))
    # keep the store (hosted by rank 0) up until every other live rank has
    # made its last store call
    live = world - (1 if die_rank is not None else 0)
    bq.close()
    if rank == 0:
        while int(store.add("left", 0)) < live - 1:
            time.sleep(0.05)
    else:
        store.add("left", 1)


def _run_queue(world, nbeams, die_rank):
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_queue_worker, args=(r, world, port, nbeams, die_rank, q)) for r in range(world)]
    for p in procs:
        p.start()
    live = world - (1 if die_rank is not None else 0)
    res = [q.get(timeout=300) for _ in range(live)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return sorted(res, key=lambda r: r[0])


def test_beam_queue_every_beam_once():
    import hashlib
    res = _run_queue(world=2, nbeams=10, die_rank=None)
    done = sorted(i for r in res for i in r[1])
    assert done == list(range(10))  # each beam by exactly one rank
    assert all(r[3] == 10 for r in res)
    assert res[0][2] == {i: hashlib.sha256(f"beam-{i}".encode()).hexdigest() for i in range(10)}


def test_beam_queue_recovers_the_beam_of_a_stopped_rank():
    import hashlib
    res = _run_queue(world=3, nbeams=9, die_rank=2)
    done = sorted(i for r in res for i in r[1])
    assert done == list(range(9))  # the stopped rank's beam was taken over, once
    assert res[0][2] == {i: hashlib.sha256(f"beam-{i}".encode()).hexdigest() for i in range(9)}
