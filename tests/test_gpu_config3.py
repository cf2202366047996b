"""The superhydrophobic channel at its full size (needs a B200).

Coarse 384 x 192 x 115 in the reference's (xdv, ydv, zdv) with 2:1 fine
blocks 768 x 384 x 16 per wall, Re_tau ~395 (constant flow rate, Reb from
Dean's correlation), with streamwise ridges (pitch 48 fine cells, gas
fraction 0.5) or square posts (pitch 32, gas fraction 0.75): 27.4 M node
updates per coarse step.  The oracle takes seconds per step at this size, so
the FP64 form is held to it over one step (bit-identical with a constant
force, 1e-12 relative with a constant flow rate); over 30 steps the FP32 form
is held to the FP64 form by the FP32 bars of the smaller cases, and the
batched engine to the FP32 channel.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import gpu_available
from test_gpu_parity import GCONST, RTOL_CFR, params_for

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]

SEED, UC, AMP = 42, 0.05, 0.005


@pytest.mark.parametrize("name,mode", [("c3r", "const"), ("c3p", "cfr")])
def test_full_size_step_matches_oracle(pkg, port, ref_configs, name, mode):
    m = ref_configs[name]
    g = pkg.geometry(params_for(pkg, m, mode))
    assert g.updates_per_step == 27_353_088
    ch = pkg.Channel(params_for(pkg, m, mode))
    ch.init_seeded(SEED, UC, AMP)
    o = port.Port(m)
    o.init_seeded(SEED, UC, AMP, GCONST if mode == "const" else 0.0)
    o.set_forcing(mode == "cfr", GCONST if mode == "const" else 0.0)
    ch.step(1)
    o.step(1)
    for lvl in range(3):
        a, b = ch.export_state(lvl), o.export(lvl)
        if mode == "const":
            np.testing.assert_array_equal(a, b, err_msg=f"level {lvl}")
        else:
            np.testing.assert_allclose(a, b, rtol=RTOL_CFR, atol=0, err_msg=f"level {lvl}")
        del a, b
    ha, hb = ch.export_history(), o.history()
    if mode == "const":
        np.testing.assert_array_equal(ha, hb)
    else:
        np.testing.assert_allclose(ha, hb, rtol=RTOL_CFR, atol=1e-13)
    o.close()
    ch.close()


@pytest.mark.parametrize("name", ["c3r", "c3p"])
def test_full_size_fp32_and_batch_track_fp64(pkg, ref_configs, name):
    m = ref_configs[name]
    a = pkg.Channel(params_for(pkg, m, "cfr"))
    a.init_seeded(SEED, UC, AMP)
    p32 = params_for(pkg, m, "cfr")
    p32.precision = pkg.FP32
    b = pkg.Channel(p32)
    b.init_seeded(SEED, UC, AMP)
    la, lb = a.step(30), b.step(30)
    sa = [a.export_state(lvl) for lvl in range(3)]
    sb = [b.export_state(lvl) for lvl in range(3)]
    assert max(np.max(np.abs(x - y)) for x, y in zip(sa, sb)) < 2e-6
    np.testing.assert_allclose(lb[:, 2:5], la[:, 2:5], rtol=1e-5, atol=1e-8)
    pa, pb = a.plane_stats(), b.plane_stats()
    used = slice(1, pa.shape[1] - 1)
    for row, stat in ((0, "U"), (3, "u_rms"), (4, "v_rms"), (5, "w_rms"), (6, "uw"), (7, "rho")):
        scale = np.max(np.abs(pa[row][used])) or 1.0
        assert np.max(np.abs(pa[row][used] - pb[row][used])) / scale < 1e-3, stat
    assert np.all(np.isfinite(la[:, 7])) and np.all(np.isfinite(lb[:, 7]))
    with pkg.Batch() as B:
        i = B.add(params_for(pkg, m, "cfr"), steps=30, seed=SEED, uc=UC, amp=AMP)
        assert B.run(30) == 0
        # the batched engine's kernels (four nodes per thread) round
        # differently from the single-channel FP32 form's: both are held to
        # the FP64 form at the FP32 bar, and to each other at FP32 rounding
        sB = [B.export_state(i, lvl) for lvl in range(3)]
        assert max(np.max(np.abs(x - y)) for x, y in zip(sB, sa)) < 2e-6
        assert max(np.max(np.abs(x - y)) for x, y in zip(sB, sb)) < 5e-7
        np.testing.assert_allclose(B.log(i)[:, 2:5], la[:, 2:5], rtol=1e-5, atol=1e-8)
    a.close()
    b.close()
