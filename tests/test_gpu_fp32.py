"""FP32 deviation-storage form against the FP64 oracle (needs a B200).

The FP32 form stores f_a - w_a in float and collides in FP32, with the
flow-rate reductions and statistics sums in FP64.  It is not bit-identical;
it is held to: populations within 2e-9 after seeding (one float rounding of a
deviation), within 2e-6 after tens of steps, and mean-velocity / Reynolds-
stress profiles within 1e-3 relative of the FP64 oracle.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import gpu_available
from test_gpu_parity import GCONST, c1_force, params_for

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]


def pair32(pkg, port, m, mode, g=GCONST, seed=42, uc=0.05, amp=0.005):
    p = params_for(pkg, m, mode, g)
    p.precision = pkg.FP32
    ch = pkg.Channel(p)
    ch.init_seeded(seed, uc, amp)
    o = port.Port(m)
    o.init_seeded(seed, uc, amp, g if mode == "const" else 0.0)
    o.set_forcing(mode == "cfr", g if mode == "const" else 0.0)
    return ch, o


def max_dev(ch, o):
    return max(np.max(np.abs(ch.export_state(l) - o.export(l))) for l in range(3))


def profile_rel_err(a, b, used):
    scale = np.max(np.abs(b[used])) or 1.0
    return np.max(np.abs(a[used] - b[used])) / scale


@pytest.mark.parametrize("name", ["t_noslip", "t_odd", "c1"])
def test_fp32_seed_is_one_rounding_of_fp64(pkg, port, ref_configs, name):
    ch, o = pair32(pkg, port, ref_configs[name], "cfr")
    assert max_dev(ch, o) < 2e-9
    np.testing.assert_allclose(ch.force(), o.force(), rtol=1e-6, atol=1e-12)


@pytest.mark.parametrize("name,mode", [("t_noslip", "const"), ("t_ridges", "cfr"), ("t_posts", "cfr"),
                                       ("t_span", "const"), ("t_gr4", "cfr"), ("t_gr4f", "cfr"), ("t_odd", "cfr")])
def test_fp32_steps_track_fp64(pkg, port, ref_configs, name, mode):
    ch, o = pair32(pkg, port, ref_configs[name], mode)
    la = ch.step(30)
    lb = o.step(30)
    assert max_dev(ch, o) < 2e-6
    # logged force / momentum / mass / flowrate
    np.testing.assert_allclose(la[:, 2:5], lb[:, 1:4], rtol=1e-5, atol=1e-8)


@pytest.mark.parametrize("mode", ["const", "cfr"])
def test_fp32_config1_statistics_within_1e3(pkg, port, ref_configs, mode):
    """Plain channel 64 x 32 x 64 with 2:1 blocks, 100 steps: mean velocity and
    Reynolds-stress profiles of the FP32 form within 1e-3 relative of FP64."""
    m = ref_configs["c1"]
    g = c1_force(pkg, m)
    ch, o = pair32(pkg, port, m, mode, g=g)
    ch.step(100)
    o.step(100)
    a, b = ch.plane_stats(), o.plane_stats()
    used = slice(1, a.shape[1] - 1)
    for row, name in ((0, "U"), (3, "u_rms"), (4, "v_rms"), (5, "w_rms"), (6, "uw"), (7, "rho")):
        assert profile_rel_err(a[row], b[row], used) < 1e-3, name
    assert max_dev(ch, o) < 1e-5


def test_fp32_restart_roundtrip(pkg, port, ref_configs, tmp_path):
    m = ref_configs["t_ridges"]
    a, _ = pair32(pkg, port, m, "cfr")
    a.step(4)
    a.write_restart(tmp_path, 5)
    p = params_for(pkg, m, "cfr")
    p.precision = pkg.FP32
    b = pkg.Channel(p)
    b.load_restart(tmp_path, 5)
    for lvl in range(3):
        np.testing.assert_allclose(a.export_state(lvl), b.export_state(lvl), atol=1e-15, rtol=0)
    a.step(3)
    b.step(3)
    for lvl in range(3):
        np.testing.assert_allclose(a.export_state(lvl), b.export_state(lvl), atol=1e-7, rtol=0)
