"""Host logic of the batched and served forms (no GPU): the seeded workload
draws, the result quantities, and the continuous-batching request loop driven
against a stand-in batch on a virtual clock."""
from __future__ import annotations

import importlib

import numpy as np
import pytest

from conftest import PKG_NAME

W = importlib.import_module(PKG_NAME + ".workloads")
S = importlib.import_module(PKG_NAME + ".serve")


def test_batched_draw_is_seeded_and_in_range():
    a = W.batched_instances(96)
    b = W.batched_instances(96)
    assert [(x.nx, x.ny, x.nz, x.pattern, x.pitch, x.gas, x.re_tau) for x in a] == \
           [(x.nx, x.ny, x.nz, x.pattern, x.pitch, x.gas, x.re_tau) for x in b]
    for x in a:
        assert x.nx in W.NX_CHOICES and x.ny in W.NY_CHOICES and x.nz in W.NZ_CHOICES
        assert x.pitch in W.PITCH_CHOICES and 0 < x.gas < x.pitch
        assert 180 <= x.re_tau <= 395 and x.pattern in ("RSLIP", "PSLIP")
        assert 0.4 < x.gas_fraction < 0.95
        assert x.zds == x.ny // 4
        assert x.re_tau_run <= W.dplus_cap(x.ny) * x.height / 2 + 1e-9 and x.re_tau_run <= x.re_tau
    assert {x.pattern for x in a} == {"RSLIP", "PSLIP"}


def test_dean_correlation_round_trip():
    for rt in (180.0, 395.0):
        reb = W.reb_from_retau(rt)
        assert abs(0.175 * (reb / 2) ** (7 / 8) - rt) < 1e-9
    assert 5400 < W.reb_from_retau(180) < 5700


def test_request_stream_poisson():
    r = W.request_stream(rate=20.0, n=4000, seed=1)
    t = np.array([x.arrival for x in r])
    assert np.all(np.diff(t) > 0)
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert abs(gaps.mean() - 1 / 20.0) < 0.05 / 20.0 * 20 ** 0.5  # mean of exponential gaps
    steps = np.array([x.steps for x in r])
    assert steps.min() >= 1000 and steps.max() <= 10000


def test_slip_length_and_drag_reduction():
    # a linear profile U = a (z + b) near both walls has slip length b
    nz = 30
    z = np.zeros(nz)
    for k in range(1, 4):
        z[k] = k - 0.5
        z[nz - 1 - k] = k - 0.5
    stats = np.zeros((14, nz))
    stats[1] = 0.01 * (z + 2.5)
    lo, up = W.slip_length(stats, zdf=9)
    assert abs(lo - 2.5) < 1e-12 and abs(up - 2.5) < 1e-12
    log = np.zeros((10, 9))
    log[:, 2], log[:, 3] = 0.08, 1.0
    cf0 = 0.073 * 6000 ** -0.25
    log[:, 7] = 0.5 * 0.08 ** 2 * cf0 * 0.7  # 30 % below the no-slip value
    cf, dr = W.drag_reduction(log, 6000.0)
    assert abs(dr - 30.0) < 1e-9


class FakeBatch:
    """Stand-in with the Batch interface: each run(n) advances every instance
    with budget left by up to n steps and moves the virtual clock by n ms."""

    def __init__(self, clock, fail_at=None):
        self.clock = clock
        self.inst = {}
        self.geoms = {}
        self.nid = 0
        self.resident_max = 0
        self.fail_at = fail_at or {}  # seed -> step whose wall stress turns non-finite

    def add(self, p, steps, seed, uc, amp, sample_every):
        i = self.nid
        self.nid += 1
        self.inst[i] = dict(steps=steps, done=0, U=p.xdv * p.ydv, status=0, fail=self.fail_at.get(seed))
        self.geoms[i] = type("G", (), {"zdf": p.zds + 1})
        self.resident_max = max(self.resident_max, len(self.inst))
        return i

    def run(self, n):
        self.clock.t += 1e-3 * n
        for v in self.inst.values():
            if v["status"] != 0:
                continue
            v["done"] = min(v["steps"], v["done"] + n)
            if v["fail"] is not None and v["done"] >= v["fail"]:
                # the engine stops the instance after the failing step
                v["done"], v["status"] = v["fail"], -4
        return sum(1 for v in self.inst.values() if v["done"] < v["steps"] and v["status"] == 0)

    def info(self, i):
        v = self.inst[i]
        return type("I", (), {"remaining": 0 if v["status"] else v["steps"] - v["done"], "steps_done": v["done"],
                              "status": v["status"], "updates_per_step": v["U"]})

    def stats(self, i):
        s = np.zeros((14, 20))
        s[1] = np.linspace(0.01, 0.02, 20)
        return s, 5

    def log(self, i):
        x = np.ones((self.inst[i]["done"], 9))
        x[:, 7] = 1e-5
        return x

    def remove(self, i):
        del self.inst[i]


class Clock:
    t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += dt


def _server(pkg, budget, fp, fail_at=None):
    clk = Clock()
    fb = FakeBatch(clk, fail_at)
    srv = S.Server(pkg, batch=fb, hbm_budget=budget, group=32)
    srv.footprint = lambda inst: fp[inst.seed]
    return srv, fb, clk


def test_server_admits_by_footprint_and_overlaps(pkg):
    reqs = W.request_stream(rate=100.0, n=12, seed=3, budget=(200, 400))
    fp = {r.seed: 10 for r in reqs}
    srv, fb, clk = _server(pkg, budget=35, fp=fp)  # at most three resident
    recs = srv.run(reqs, clock=clk, sleep=clk.sleep)
    assert all(r.status == 0 and r.result["steps"] == r.inst.steps for r in recs)
    assert fb.resident_max == 3 and srv.peak_used <= 35 and srv.used == 0
    # requests that arrived while others ran were admitted before those finished
    overl = sum(1 for a in recs for b in recs if a is not b and a.admitted < b.admitted < a.finished)
    assert overl > 0
    assert all(r.admitted >= r.arrival and r.finished > r.admitted for r in recs)
    lat = S.latency_summary(recs)
    assert lat["completed"] == 12 and lat["p99_s"] >= lat["p50_s"] > 0


def test_server_rejects_oversize_and_waits_for_arrivals(pkg):
    reqs = W.request_stream(rate=2.0, n=4, seed=4, budget=(64, 64))
    fp = {r.seed: 10 for r in reqs}
    fp[reqs[1].seed] = 1000
    srv, fb, clk = _server(pkg, budget=100, fp=fp)
    recs = srv.run(reqs, clock=clk, sleep=clk.sleep)
    assert recs[1].status == pkg.DNS_ENOMEM
    assert [r.status for r in recs if r is not recs[1]] == [0, 0, 0]
    # sparse arrivals: each request waits for nobody
    assert all(abs(r.admitted - r.arrival) < 1e-9 for r in recs if r.status == 0)


def test_fifo_model():
    lat = S.fifo_latencies([0.0, 0.5, 0.6], [1.0, 1.0, 1.0])
    np.testing.assert_allclose(lat, [1.0, 1.5, 2.4])


def test_server_retires_a_failed_instance_and_runs_the_rest(pkg):
    """Fault injected on the host: one request's instance reports a
    non-finite wall shear stress mid-run; it is retired with DNS_ENAN and its
    memory released while the co-resident requests finish their budgets."""
    assert pkg.DNS_ENAN == -4
    reqs = W.request_stream(rate=100.0, n=6, seed=5, budget=(300, 300))
    fp = {r.seed: 10 for r in reqs}
    srv, fb, clk = _server(pkg, budget=100, fp=fp, fail_at={reqs[2].seed: 70})
    recs = srv.run(reqs, clock=clk, sleep=clk.sleep)
    bad = recs[2]
    assert bad.status == pkg.DNS_ENAN and bad.result["steps"] == 70 and "cf" not in bad.result
    assert bad.finished < max(r.finished for r in recs)  # retired at once, not at the end
    for r in recs:
        if r is not bad:
            assert r.status == 0 and r.result["steps"] == 300
    assert srv.used == 0 and not fb.inst
    lat = S.latency_summary(recs)
    assert lat["completed"] == 5 and lat["failed"] == 1


def test_server_deadline_times_out_resident_and_queued(pkg):
    """A CPU-side timeout of the request loop: past the deadline the resident
    requests are retired with DNS_ETIMEOUT (their steps so far reported), the
    queued and later ones are not run, and every byte is released."""
    reqs = W.request_stream(rate=50.0, n=10, seed=6, budget=(400, 400))
    fp = {r.seed: 10 for r in reqs}
    srv, fb, clk = _server(pkg, budget=25, fp=fp)  # two resident at a time
    recs = srv.run(reqs, clock=clk, sleep=clk.sleep, deadline=0.9)
    st = [r.status for r in recs]
    # 400 steps at 1 ms a step take ~0.42 s: two pairs finish before 0.9 s
    assert st[:4] == [0, 0, 0, 0]
    assert set(st[4:]) == {pkg.DNS_ETIMEOUT}
    cut = [r for r in recs if r.status == pkg.DNS_ETIMEOUT and r.result]
    assert len(cut) == 2 and all(0 < r.result["steps"] < 400 for r in cut)
    never = [r for r in recs if r.status == pkg.DNS_ETIMEOUT and not r.result]
    assert len(never) == 4 and all(r.admitted != r.admitted for r in never)  # NaN: not admitted
    assert all(r.finished >= 0.9 for r in recs[4:])
    assert srv.used == 0 and not fb.inst


class FakeChannel:
    """Stand-in FP64 channel: step(n) moves the virtual clock by 2 ms a step."""

    def __init__(self, clock, p, fail_seed=None):
        self.clock = clock
        self.geom = type("G", (), {"zdf": p.zds + 1})
        self.fail_seed = fail_seed
        self.seed = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def init_seeded(self, seed, uc, amp):
        self.seed = seed

    def set_sampling(self, every):
        pass

    def step(self, n):
        self.clock.t += 2e-3 * n
        if self.seed == self.fail_seed:
            raise self.err(-4, "fake: NaN wall shear stress")
        x = np.ones((n, 9))
        x[:, 7] = 1e-5
        return x

    def stats(self):
        s = np.zeros((14, 20))
        s[1] = np.linspace(0.01, 0.02, 20)
        return s, 5


def test_one_at_a_time_server_is_first_come_first_served(pkg):
    import types

    clk = Clock()
    reqs = W.request_stream(rate=2.0, n=5, seed=8, budget=(300, 600))
    fail = reqs[3].seed
    fake = types.SimpleNamespace(FP64=pkg.FP64, DnsError=pkg.DnsError, make_params=pkg.make_params,
                                 FORCING_CFR=pkg.FORCING_CFR,
                                 Channel=lambda p: FakeChannel(clk, p, fail_seed=fail))
    FakeChannel.err = pkg.DnsError
    recs = S.serve_one_at_a_time(fake, reqs, clock=clk, sleep=clk.sleep)
    # the same latencies as a single first-come-first-served server with
    # service = 2 ms x budget
    lat = S.fifo_latencies([r.arrival for r in recs], [2e-3 * r.inst.steps for r in recs])
    np.testing.assert_allclose([r.latency for r in recs], lat, rtol=1e-12, atol=1e-12)
    assert recs[3].status == -4 and "cf" not in recs[3].result
    assert all(r.status == 0 and "slip_length" in r.result for r in recs if r is not recs[3])


def test_server_bounds_the_resident_work_per_step(pkg):
    """With the per-step work bound, requests are admitted while the resident
    set's node updates per step stay under it (a request is always admitted
    to an idle GPU), so a backlog completes in arrival order instead of every
    request sharing the GPU until the end."""
    reqs = W.request_stream(rate=1000.0, n=10, seed=9, budget=(300, 300))
    fp = {r.seed: 1 for r in reqs}
    clk = Clock()
    fb = FakeBatch(clk)
    per = max(r.updates_per_step() for r in reqs)
    srv = S.Server(pkg, batch=fb, hbm_budget=1e12, group=32, max_updates=2.5 * per)
    srv.footprint = lambda inst: fp[inst.seed]
    recs = srv.run(reqs, clock=clk, sleep=clk.sleep)
    assert all(r.status == 0 for r in recs)
    least = min(r.updates_per_step() for r in reqs)
    assert fb.resident_max <= int(2.5 * per / least) and fb.resident_max < 10 and srv.active_updates == 0
    fin = [r.finished for r in recs]
    assert fin == sorted(fin)
    # unbounded, all ten are resident at once
    clk2 = Clock()
    fb2 = FakeBatch(clk2)
    srv2 = S.Server(pkg, batch=fb2, hbm_budget=1e12, group=32, max_updates=None)
    srv2.footprint = lambda inst: fp[inst.seed]
    srv2.run(reqs, clock=clk2, sleep=clk2.sleep)
    assert fb2.resident_max == 10
