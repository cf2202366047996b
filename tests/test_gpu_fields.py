"""Field output (the reference's vel_print) from the GPU state (needs a B200).

The FP64 form's vel-* / den-* files are compared byte for byte with the files
the reference's own vel_print writes for the same state (the compiled
reference harness loads the restart this library wrote and calls vel_print);
the FP32 form's within its tolerance."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

from conftest import gpu_available, ref_binary
from test_gpu_parity import GCONST, params_for

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]

FILES = ("vel-c", "den-c", "vel-slf", "den-slf", "vel-suf", "den-suf")


def _reference_fields(exe, src, dst, cntr):
    subprocess.run([str(exe), str(src), str(cntr), str(dst), str(cntr), "0", "const", GCONST.hex(), "0", "1"],
                   check=True, capture_output=True)


@pytest.mark.parametrize("name", ["t_ridges", "t_posts", "c1"])
def test_fields_fp64_match_reference_vel_print(pkg, ref_configs, tmp_path, name):
    exe = ref_binary(name)
    if exe is None:
        pytest.skip("compiled reference not available")
    a, b = tmp_path / "ours", tmp_path / "ref"
    a.mkdir()
    b.mkdir()
    ch = pkg.Channel(params_for(pkg, ref_configs[name], "const"))
    ch.init_seeded(42, 0.05, 0.005)
    ch.step(6)
    ch.write_restart(a, 8)
    ch.write_fields(a, 8)
    ch.close()
    _reference_fields(exe, a, b, 8)
    for fn in FILES:
        x = (a / f"{fn}.0008").read_bytes()
        y = (b / f"{fn}.0008").read_bytes()
        assert len(x) == len(y) and x == y, fn


def test_fields_fp32_within_tolerance(pkg, ref_configs, tmp_path):
    name = "t_ridges"
    exe = ref_binary(name)
    if exe is None:
        pytest.skip("compiled reference not available")
    a, b = tmp_path / "ours", tmp_path / "ref"
    a.mkdir()
    b.mkdir()
    p = params_for(pkg, ref_configs[name], "const")
    p.precision = pkg.FP32
    ch = pkg.Channel(p)
    ch.init_seeded(42, 0.05, 0.005)
    ch.step(6)
    ch.write_restart(a, 8)
    ch.write_fields(a, 8)
    ch.close()
    _reference_fields(exe, a, b, 8)
    for fn in FILES:
        x = np.fromfile(a / f"{fn}.0008")
        y = np.fromfile(b / f"{fn}.0008")
        np.testing.assert_allclose(x, y, rtol=0, atol=1e-7)
