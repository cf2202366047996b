"""Host-side arithmetic of the long-run statistics legs (no GPU): window means
from cumulative statistics, batch-means errors, Cf / drag reduction as the
reference's post-processing forms them, and the per-statistic comparison."""
from __future__ import annotations

import importlib
import math

import numpy as np

from conftest import PKG_NAME

W = importlib.import_module(PKG_NAME + ".workloads")


def test_window_means_invert_cumulative_averages():
    rng = np.random.default_rng(3)
    nz = 7
    samples = [rng.normal(size=(14, nz)) for _ in range(12)]
    # cumulative averages after 0, 4, 8, 12 samples (row 0 is z)
    cum = [(np.zeros((14, nz)), 0)]
    for n in (4, 8, 12):
        avg = np.mean(samples[:n], axis=0)
        cum.append((avg, n))
    wm = W.window_means(cum)
    for q, lo in enumerate((0, 4, 8)):
        expect = np.mean(samples[lo:lo + 4], axis=0)
        np.testing.assert_allclose(wm[q][1:10], expect[1:10], rtol=1e-12, atol=1e-13)


def test_batch_mean_and_error():
    m, e = W.batch_mean_and_error([[1.0], [2.0], [3.0], [4.0]])
    assert m[0] == 2.5
    assert math.isclose(e[0], np.std([1, 2, 3, 4], ddof=1) / 2.0)


def test_friction_coefficient_follows_cfriction():
    # rows: time force momentum denst flowrate stup stdown stress pgrad
    nyf, nzs = 16, 20
    log = np.zeros((4, 9))
    log[:, 4] = [1.0, 1.1, 0.9, 1.0]
    log[:, 7] = [2e-4, 3e-4, 1e-4, 2e-4]
    ub = np.mean(log[:, 4]) / ((nyf + 1) * (nzs - 2.0))
    expect = np.mean(log[:, 7] / (0.5 * ub * ub))
    assert math.isclose(W.friction_coefficient(log, nyf, nzs), expect)
    assert math.isclose(W.drag_reduction_vs(0.006, 0.008), 25.0)


def test_compare_runs_flags_large_errors():
    nz = 9
    z = np.linspace(0, 1, nz)
    prof = np.zeros((14, nz))
    prof[1] = 4 * z * (1 - z)
    prof[5] = 1e-3 * np.sin(np.pi * z)
    prof[8] = -1e-4 * np.sin(2 * np.pi * z)
    se = np.full((14, nz), 1e-9)
    ref = {"profiles": prof, "stderr": se, "tau_w": 1e-3, "tau_w_stderr": 1e-6, "cf": 8e-3, "cf_stderr": 1e-6,
           "slip_length": 2.0, "slip_length_stderr": 1e-3}
    same = dict(ref, profiles=prof * (1 + 1e-5))
    assert all(v["ok"] for v in W.compare_runs(same, ref).values())
    off = dict(ref, profiles=prof.copy())
    off["profiles"][5] = prof[5] * 1.01
    res = W.compare_runs(off, ref)
    assert not res["uu"]["ok"] and res["U"]["ok"]
    assert math.isclose(res["uu"]["rel_err"], 0.01, rel_tol=1e-6)
