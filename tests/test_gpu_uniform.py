"""Mode -i start on the GPU (needs a B200): a uniform-grid lbf.TTTT interpolated
onto the embedded grids and the interface history built from it.

The FP64 form is bit-identical to the oracle's restatement, which the CPU tests
pin to the unmodified reference main run in mode -i; the FP32 form holds its
populations within 1e-7.  Runs continued from the start follow the oracle as
any other FP64 run does.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import gpu_available
from test_gpu_parity import GCONST, RTOL_CFR, assert_state, params_for

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]

# c1 (64 x 27 x 64 coarse, zds 8) with a uniform grid of 47 wall-normal cells
C1_UNIFORM = dict(xdu=96, ydu=96, zdu=47)


def _macros(ref_configs, name):
    m = dict(ref_configs[name])
    if "xdu" not in m:
        m.update(C1_UNIFORM)
    return m


def _start(pkg, port, m, mode, tmp_path, precision=None, seeds=(1, 2)):
    xu, yu, zu, tstr = int(m["xdu"]), int(m["ydu"]), int(m["zdu"]), int(m["TSTR"])
    first = port.uniform_state(xu, yu, zu, seeds[0])
    port.write_uniform_file(tmp_path / f"lbf.{tstr:04d}", first, port.uniform_state(xu, yu, zu, seeds[1]))
    prm = params_for(pkg, m, mode)
    prm.xdu, prm.ydu, prm.zdu = xu, yu, zu
    if precision is not None:
        prm.precision = precision
    ch = pkg.Channel(prm)
    ch.load_uniform(tmp_path, tstr)
    p = port.Port(m)
    g = GCONST if mode == "const" else 0.0
    p.set_forcing(mode == "cfr", g)
    p.init_uniform(first)
    return ch, p


@pytest.mark.parametrize("name", ["t_noslip", "t_ridges", "c1"])
def test_uniform_start_bit_identical(pkg, port, ref_configs, tmp_path, name):
    ch, p = _start(pkg, port, _macros(ref_configs, name), "cfr", tmp_path)
    assert_state(ch, p, exact=True)
    h = ch.export_history()
    np.testing.assert_array_equal(h[1], h[0])
    np.testing.assert_array_equal(h[2], h[0])
    np.testing.assert_allclose(ch.force(), p.force(), rtol=1e-13, atol=0)
    ch.close()


@pytest.mark.parametrize("name,mode", [("t_noslip", "const"), ("t_ridges", "cfr"), ("t_ridges", "const")])
def test_uniform_start_then_steps(pkg, port, ref_configs, tmp_path, name, mode):
    ch, p = _start(pkg, port, _macros(ref_configs, name), mode, tmp_path)
    la = ch.step(20)
    lb = p.step(20)
    assert_state(ch, p, exact=(mode == "const"), rtol=RTOL_CFR)
    np.testing.assert_allclose(la[:, 1:5], lb[:, 0:4], rtol=1e-11, atol=1e-15)
    ch.close()


def test_uniform_start_fp32(pkg, port, ref_configs, tmp_path):
    ch, p = _start(pkg, port, _macros(ref_configs, "t_ridges"), "cfr", tmp_path, precision=pkg.FP32)
    for lvl in range(3):
        np.testing.assert_allclose(ch.export_state(lvl), p.export(lvl), rtol=0, atol=1e-7)
    np.testing.assert_allclose(ch.export_history(), p.history(), rtol=0, atol=1e-7)
    ch.close()


def test_uniform_start_rejects_short_grid(pkg, port, ref_configs, tmp_path):
    """Stencils that would leave the reference's periodic halo: EINVAL."""
    m = dict(ref_configs["t_ridges"], xdu=4)
    with pytest.raises(pkg.DnsError) as e:
        _start(pkg, port, m, "cfr", tmp_path)
    assert e.value.code == pkg.DNS_EINVAL


def test_uniform_start_missing_file(pkg, ref_configs, tmp_path):
    prm = params_for(pkg, ref_configs["t_ridges"], "cfr")
    ch = pkg.Channel(prm)
    with pytest.raises(pkg.DnsError) as e:
        ch.load_uniform(tmp_path, 7)
    assert e.value.code == pkg.DNS_EIO
    ch.close()
