"""Long-run statistics of the FP32 deviation form against the FP64 plain form
(a short version of the production-channel leg bench.py reports): channel c1
(reference macros xdv 64, ydv 64, zdv 27, zds 8, GR 2) at constant flow rate,
500 warm-up steps, then 1500 steps sampled every step in 5 windows.  Every
statistic must agree within 1e-3 of the profile's scale or within two
batch-means standard errors, as the bench leg's bar."""
from __future__ import annotations

import importlib

import numpy as np
import pytest

from conftest import PKG_NAME, gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]

UB = 0.0866034
C1 = dict(xdv=64, ydv=64, zdv=27, zds=8, gratio=2, Rebs=150.0 * UB * 63, ub=UB, CFL=0.1, pattern=None)
C1_RIDGES = dict(C1, pattern="RSLIP", gyplussize=8, wyplussize=8)


@pytest.mark.parametrize("macros", [C1, C1_RIDGES], ids=["noslip", "ridges"])
def test_fp32_statistics_match_fp64(pkg, macros):
    W = importlib.import_module(PKG_NAME + ".workloads")
    g = pkg.geometry(pkg.make_params(**macros))
    runs = {}
    for prec in ("fp64", "fp32"):
        cum, log, err = W.long_run(pkg, macros, prec, warm=500, windows=5, per=300)
        assert err is None, err
        assert cum[-1][1] - cum[0][1] == 1500
        assert log.shape == (1500, 9) and np.all(np.isfinite(log))
        runs[prec] = W.summarize_run(cum, log, 5, g.nyf, g.nzs, g.zdf, macros["Rebs"])
    cmp = W.compare_runs(runs["fp32"], runs["fp64"])
    bad = {k: v for k, v in cmp.items() if not v["ok"]}
    assert not bad, bad
    # the mean profile carries the flow: its error is far inside the bar
    assert cmp["U"]["rel_err"] < 1e-3
