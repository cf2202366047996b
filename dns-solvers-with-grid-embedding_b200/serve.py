"""Continuous-batching request loop over the batched FP32 engine.

Parametric channel solves (workloads.Instance: grid, wall pattern, Re_tau,
step budget) arrive over time.  The loop admits queued requests, first come
first served, while their device footprint fits the HBM budget; admitted
requests join the resident batch between step groups, so work that arrives
while others are on the GPU overlaps with them; a request whose budget is
spent is retired (its statistics and log read back, its memory released) and
its latency recorded.  Each instance's results depend only on its own
parameters, not on what else is resident (the batch engine's invariance).

There is no counterpart in the reference, which runs one MPI job per channel.
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import workloads


@dataclass
class Record:
    inst: workloads.Instance
    id: int = -1
    bytes: int = 0
    arrival: float = 0.0
    admitted: float = float("nan")
    finished: float = float("nan")
    status: int = 0
    result: dict = field(default_factory=dict)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class Server:
    """Serve a list of requests on one GPU.

    batch: a Batch (or an object with its interface); hbm_budget: bytes the
    resident instances may hold; group: coarse steps per batch.run() between
    admission rounds; sample_every: statistics sampling period in steps;
    max_updates: node updates per coarse step the resident instances may do
    together (None: no bound).  The batched kernels reach their throughput
    with one production-size channel resident (c2, 11 M updates a step, runs
    within 4% of 96 channels' 378 M), so admitting far beyond that only
    shares the GPU among more requests: every one of them then finishes near
    the end of the backlog instead of in arrival order (measured on B200 at 10
    requests/s: p50 99 s unbounded, 62 s at 32 M).  Small drawn channels run
    less efficiently than one large one, so the bound keeps several resident:
    at 32 M the aggregate fell to 26.9 from 28.9 GLUPS; the default, 64 M,
    keeps the throughput.
    """

    def __init__(self, pkg, batch=None, hbm_budget: float = 150e9, group: int = 32, sample_every: int = 20,
                 device: int = 0, max_updates: float | None = 64e6):
        self.pkg = pkg
        self.batch = batch if batch is not None else pkg.Batch(device)
        self.budget = hbm_budget
        self.group = group
        self.sample_every = sample_every
        self.max_updates = max_updates
        self.used = 0
        self.peak_used = 0
        self.active_updates = 0  # node updates per step of the resident requests
        self.updates = 0  # node updates done by retired requests

    def footprint(self, inst) -> int:
        return self.pkg.batch_footprint(inst.params(self.pkg))

    def _retire(self, rec: Record, now: float, status: int | None = None):
        b = self.batch
        info = b.info(rec.id)
        rec.status = int(info.status) if status is None or info.status != 0 else status
        stats, _ = b.stats(rec.id)
        log = b.log(rec.id)
        if rec.status == 0 and len(log):
            rec.result = workloads.solve_result(rec.inst, stats, log, b.geoms[rec.id].zdf)
        rec.result["steps"] = int(info.steps_done)
        self.updates += int(info.steps_done) * int(info.updates_per_step)
        b.remove(rec.id)
        self.used -= rec.bytes
        self.active_updates -= rec.inst.updates_per_step()
        rec.finished = now

    def run(self, requests, clock=time.perf_counter, sleep=time.sleep, deadline: float | None = None):
        """Serve requests (arrival times in seconds from the start); returns
        the records in arrival order.  A request larger than the whole budget
        is rejected with status DNS_ENOMEM.  An instance whose wall shear
        stress turns non-finite is retired at once with DNS_ENAN; the others
        run on unaffected.  With a deadline (seconds from the start), the loop
        ends at the first step-group boundary past it: resident requests are
        retired with DNS_ETIMEOUT (the steps they took are reported), queued
        and later ones get DNS_ETIMEOUT without running."""
        pending = sorted(requests, key=lambda r: r.arrival)
        recs = [Record(inst=r, arrival=r.arrival) for r in pending]
        queue: deque[Record] = deque()
        active: dict[int, Record] = {}
        nxt = 0
        t0 = clock()
        while nxt < len(recs) or queue or active:
            now = clock() - t0
            if deadline is not None and now >= deadline:
                for i in list(active):
                    self._retire(active.pop(i), now, status=self.pkg.DNS_ETIMEOUT)
                for rec in list(queue) + recs[nxt:]:
                    rec.status = self.pkg.DNS_ETIMEOUT
                    rec.finished = now
                break
            while nxt < len(recs) and recs[nxt].arrival <= now:
                queue.append(recs[nxt])
                nxt += 1
            # admission: first come first served while the footprint fits the
            # HBM budget and the work the resident set does per step stays
            # under the bound (a request is always admitted to an idle GPU)
            while queue:
                rec = queue[0]
                rec.bytes = self.footprint(rec.inst)
                if rec.bytes > self.budget:
                    queue.popleft()
                    rec.status = self.pkg.DNS_ENOMEM
                    rec.finished = clock() - t0
                    continue
                if self.used + rec.bytes > self.budget:
                    break
                if (self.max_updates is not None and active and
                        self.active_updates + rec.inst.updates_per_step() > self.max_updates):
                    break
                queue.popleft()
                rec.id = self.batch.add(rec.inst.params(self.pkg), steps=rec.inst.steps, seed=rec.inst.seed,
                                        uc=workloads.UC, amp=workloads.AMP, sample_every=self.sample_every)
                rec.admitted = clock() - t0
                self.used += rec.bytes
                self.active_updates += rec.inst.updates_per_step()
                self.peak_used = max(self.peak_used, self.used)
                active[rec.id] = rec
            if not active:
                if nxt < len(recs):
                    wake = recs[nxt].arrival if deadline is None else min(recs[nxt].arrival, deadline)
                    sleep(max(0.0, wake - (clock() - t0)))
                continue
            self.batch.run(self.group)
            now = clock() - t0
            for i in list(active):
                info = self.batch.info(i)
                if info.remaining == 0 or info.status != 0:
                    self._retire(active.pop(i), now)
        return recs


def serve_one_at_a_time(pkg, requests, clock=time.perf_counter, sleep=time.sleep, sample_every: int = 20,
                        device: int = 0):
    """The baseline the continuous-batching loop is compared with: the same
    requests served one at a time, first come first served, each by the FP64
    plain form on its own channel handle (allocated on arrival at the head of
    the queue, stepped through its whole budget, results read back, freed).
    Latency = completion - arrival on the host clock, as Server.run."""
    recs = [Record(inst=r, arrival=r.arrival) for r in sorted(requests, key=lambda r: r.arrival)]
    t0 = clock()
    for rec in recs:
        now = clock() - t0
        if now < rec.arrival:
            sleep(rec.arrival - now)
        rec.admitted = clock() - t0
        p = rec.inst.params(pkg, precision=pkg.FP64)
        p.device = device
        with pkg.Channel(p) as ch:
            ch.init_seeded(rec.inst.seed, workloads.UC, workloads.AMP)
            ch.set_sampling(sample_every)
            try:
                log = ch.step(rec.inst.steps)
            except pkg.DnsError as e:
                rec.status = e.code
                log = None
            if rec.status == 0:
                stats, _ = ch.stats()
                rec.result = workloads.solve_result(rec.inst, stats, log, ch.geom.zdf)
            rec.result["steps"] = int(rec.inst.steps)
        rec.finished = clock() - t0
    return recs


def latency_summary(recs) -> dict:
    lat = np.array([r.latency for r in recs if r.status == 0])
    if lat.size == 0:
        return {"p50_s": None, "p99_s": None, "completed": 0}
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "completed": int(lat.size),
            "failed": int(sum(1 for r in recs if r.status != 0))}


def fifo_latencies(arrivals, services) -> np.ndarray:
    """Latencies of a single server taking requests one at a time, first come
    first served: finish_i = max(arrival_i, finish_{i-1}) + service_i (a
    model, used by the host tests to check serve_one_at_a_time's clock)."""
    fin = 0.0
    out = []
    for a, s in zip(arrivals, services):
        fin = max(a, fin) + s
        out.append(fin - a)
    return np.array(out)
