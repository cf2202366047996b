"""Multi-process host logic on CPU (gloo, world size 2): the sharding of
independent channels over GPUs and the max / sum reductions bench.py uses
for N > 1 (every rank computes the same shard without communicating; the
time is the slowest rank's, the work the sum of all ranks'), and a rank that
dies between steps: the survivor's next reduction ends with an error within
the process group's timeout instead of waiting for good."""
from __future__ import annotations

import importlib
import os
import socket
import sys

import pytest

from conftest import PKG_NAME, ROOT

W = importlib.import_module(PKG_NAME + ".workloads")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    import torch

    sys.path.insert(0, str(ROOT))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    bench = importlib.import_module("bench")
    w = importlib.import_module(PKG_NAME + ".workloads")
    insts = w.batched_instances(96)
    mine = w.shard(insts, world)[rank]
    # gather every rank's shard
    got = [None] * world
    dist.all_gather_object(got, mine)
    t = bench.max_over_ranks(torch, dist, 10.0 + rank)
    u = bench.sum_over_ranks(torch, dist, float(sum(insts[i].updates_per_step() for i in mine)))
    q.put((rank, got, t, u))
    dist.barrier()
    dist.destroy_process_group()


def test_shard_partitions_and_balances():
    insts = W.batched_instances(96)
    for world in (1, 2, 4, 8):
        parts = W.shard(insts, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(96))
        load = [sum(insts[i].updates_per_step() * insts[i].steps for i in p) for p in parts]
        assert max(load) <= 1.1 * (sum(load) / world) + max(x.updates_per_step() * x.steps for x in insts)


@pytest.mark.timeout(120)
def test_two_ranks_agree_on_shards_and_reduce():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=100) for _ in range(2)]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    insts = W.batched_instances(96)
    expect = W.shard(insts, 2)
    total = float(sum(x.updates_per_step() for x in insts))
    for rank, got, t, u in res:
        assert got == expect
        assert t == 11.0
        assert u == total


def _report(q, item):
    """Put one item and wait until the queue's feeder thread has handed it to
    the pipe: os._exit skips that flush, and an item still in the feeder is lost."""
    q.put(item)
    q.close()
    q.join_thread()


def _dying_worker(rank, world, port, q):
    import time
    from datetime import timedelta

    import torch.distributed as dist
    import torch

    sys.path.insert(0, str(ROOT))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        # a generous rendezvous: under CPU load one rank can start many seconds
        # after the other; the collectives then run in a group with a short
        # timeout, the bound a survivor waits for a lost peer
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=90))
        short = dist.new_group(timeout=timedelta(seconds=5))
        bench = importlib.import_module("bench")
        t = bench.max_over_ranks(torch, dist, 1.0 + rank, group=short)  # one step's reduction, both alive
    except Exception as e:  # reported, so the test fails with the reason instead of a queue timeout
        _report(q, (rank, None, "setup failed: " + repr(e), 0.0))
        os._exit(4)
    if rank == 1:
        _report(q, (rank, t, "leaving", 0.0))
        os._exit(3)  # the rank dies between steps, with nothing in flight
    t0 = time.monotonic()
    try:
        bench.max_over_ranks(torch, dist, 5.0, group=short)
        item = (rank, t, "no error", time.monotonic() - t0)
    except Exception as e:  # gloo reports the lost peer or the timeout
        item = (rank, t, type(e).__name__, time.monotonic() - t0)
    _report(q, item)
    os._exit(0)


@pytest.mark.timeout(300)
def test_lost_rank_ends_the_next_reduction_with_an_error():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dying_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    while len(got) < 2:
        rank, t, msg, waited = q.get(timeout=240)
        assert not msg.startswith("setup failed"), msg
        got[rank] = (t, msg, waited)
    for p in procs:
        p.join(timeout=60)
    assert got[1][:2] == (2.0, "leaving")
    t, err, waited = got[0]
    assert t == 2.0
    assert err != "no error"
    assert [p.exitcode for p in procs] == [0, 3]
    # the survivor's collective ended within the short group's timeout (plus
    # slack for a loaded host), not after waiting for good
    assert waited < 60
