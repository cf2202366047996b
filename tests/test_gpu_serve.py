"""Served form on the GPU: a request's answer is the same served alone as
served among others that arrive, overlap and leave around it (bit for bit:
the batch engine keeps every instance's arithmetic independent of the mix)."""
from __future__ import annotations

import importlib

import numpy as np
import pytest

from conftest import PKG_NAME, gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]

W = importlib.import_module(PKG_NAME + ".workloads")
S = importlib.import_module(PKG_NAME + ".serve")


def _requests():
    mk = W.Instance
    return [mk(64, 32, 64, "RSLIP", 16, 10, 200.0, seed=11, steps=96, arrival=0.0),
            mk(128, 48, 64, "PSLIP", 24, 12, 300.0, seed=12, steps=40, arrival=0.0),
            mk(64, 32, 96, "PSLIP", 32, 20, 250.0, seed=13, steps=130, arrival=0.05),
            mk(64, 64, 64, "RSLIP", 24, 16, 390.0, seed=14, steps=70, arrival=0.1)]


def test_served_result_same_alone_and_in_mix(pkg):
    reqs = _requests()
    srv = S.Server(pkg, hbm_budget=150e9, group=16, sample_every=4)
    mixed = srv.run(reqs)
    srv.batch.close()
    assert all(r.status == 0 for r in mixed)
    for r in mixed:
        assert r.result["steps"] == r.inst.steps
        assert np.isfinite(r.result["slip_length"]) and np.isfinite(r.result["drag_reduction_pct"])
        assert r.finished > r.admitted >= r.arrival
    # overlap happened: the first request was still resident when a later one was admitted
    assert any(a.admitted < b.admitted < a.finished for a in mixed for b in mixed if a is not b)
    for q in (0, 2):
        alone = S.Server(pkg, hbm_budget=150e9, group=16, sample_every=4)
        one = alone.run([reqs[q]])[0]
        alone.batch.close()
        assert np.array_equal(np.array(one.result["U"]), np.array(mixed[q].result["U"]))
        assert one.result["slip_length"] == mixed[q].result["slip_length"]
        assert one.result["drag_reduction_pct"] == mixed[q].result["drag_reduction_pct"]


def test_server_respects_hbm_budget(pkg):
    reqs = _requests()
    fps = [pkg.batch_footprint(r.params(pkg)) for r in reqs]
    budget = max(fps) + min(fps)  # never more than two resident
    srv = S.Server(pkg, hbm_budget=budget, group=16, sample_every=0)
    recs = srv.run(reqs)
    srv.batch.close()
    assert all(r.status == 0 for r in recs)
    assert srv.peak_used <= budget and srv.used == 0
