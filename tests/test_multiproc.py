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


def _dying_worker(rank, world, port, q):
    from datetime import timedelta

    import torch.distributed as dist
    import torch

    sys.path.insert(0, str(ROOT))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=5))
    bench = importlib.import_module("bench")
    t = bench.max_over_ranks(torch, dist, 1.0 + rank)  # one step's reduction, both alive
    if rank == 1:
        os._exit(3)  # the rank dies between steps, with nothing in flight
    try:
        bench.max_over_ranks(torch, dist, 5.0)
        q.put((rank, t, "no error"))
    except Exception as e:  # gloo reports the lost peer or the timeout
        q.put((rank, t, type(e).__name__))
    os._exit(0)


@pytest.mark.timeout(120)
def test_lost_rank_ends_the_next_reduction_with_an_error():
    import time

    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dying_worker, args=(r, 2, port, q)) for r in range(2)]
    t0 = time.monotonic()
    for p in procs:
        p.start()
    rank, t, err = q.get(timeout=100)
    for p in procs:
        p.join(timeout=30)
    assert rank == 0 and t == 2.0
    assert err != "no error"
    assert [p.exitcode for p in procs] == [0, 3]
    assert time.monotonic() - t0 < 100
