"""Turbulence statistics and kinetic-energy budget on the GPU (needs a B200).

The reference's own offline program (TKE-budget/computations, compiled
unmodified against the single-rank MPI shim into oracle/_ref/<config>/
tke_budget) reads the vel-* / den-* files this library writes; its three
output files are compared with the budget computed on the device from the
live state and from the same files.  The plane means are summed in the
reference's order (bit-identical), the 44 per-plane product sums in another
association than the reference's sequential loops, so every profile is held
to 1e-11 of its own largest magnitude.
"""
from __future__ import annotations

import json
import subprocess

import numpy as np
import pytest

from conftest import ROOT, gpu_available, ref_binary
from test_gpu_parity import GCONST, params_for

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]

GOLDEN = json.loads((ROOT / "tests" / "golden" / "tke_golden.json").read_text())
RTOL = 1e-11


def _reference_budget(pkg, exe, fields_dir, cntr, nz):
    work = fields_dir / "tke"
    work.mkdir()
    subprocess.run([str(exe)], cwd=work, check=True, capture_output=True)
    rows = []
    for name, n in pkg.TKE_FILES:
        a = np.fromfile(work / f"{name}.000.{cntr:04d}")
        assert a.size == n * nz, name
        rows.append(a.reshape(n, nz))
    return np.concatenate(rows), work


def assert_profiles(ours, ref, names, rtol=RTOL):
    for r, name in enumerate(names):
        scale = np.max(np.abs(ref[r]))
        np.testing.assert_allclose(ours[r], ref[r], rtol=0, atol=rtol * scale + 1e-300, err_msg=name)


def _channel(pkg, m, steps, precision=None):
    p = params_for(pkg, m, "const")
    if precision is not None:
        p.precision = precision
    ch = pkg.Channel(p)
    ch.init_seeded(42, 0.05, 0.005)
    ch.step(steps)
    return ch, p


@pytest.mark.parametrize("name,steps", [("t_odd", 6), ("t_gr4", 4), ("c1", 6)])
def test_budget_matches_reference_program(pkg, ref_configs, tmp_path, name, steps):
    exe = ref_binary(name, "tke_budget")
    if exe is None:
        pytest.skip("compiled reference budget program not available")
    m = ref_configs[name]
    cntr = int(m["TSTR"])
    ch, p = _channel(pkg, m, steps)
    ch.write_fields(tmp_path, cntr)
    nz = pkg.geometry(p).nz_profile
    ref, work = _reference_budget(pkg, exe, tmp_path, cntr, nz)
    ours, ufl, vfl = ch.tke_budget(fluct_plane=True)
    assert_profiles(ours, ref, pkg.TKE_NAMES)
    files = pkg.tke_budget_files(p, tmp_path, cntr)
    assert_profiles(files, ref, pkg.TKE_NAMES)
    # the reference main writes the fluctuation plane every 200 unit times
    if cntr % 200 == 0:
        g = pkg.geometry(p)
        for fn, a in (("ufl4", ufl), ("vfl4", vfl)):
            b = np.fromfile(work / f"{fn}.{cntr:04d}").reshape(g.nxf, g.nyf)
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-15)
    # the files this library writes have the reference's names and layout
    out = tmp_path / "ours"
    out.mkdir()
    pkg.write_tke_budget(p, out, cntr, ours, ufl, vfl)
    for fname, n in pkg.TKE_FILES:
        a = np.fromfile(out / f"{fname}.000.{cntr:04d}")
        b = np.fromfile(work / f"{fname}.000.{cntr:04d}")
        assert a.size == b.size
    ch.close()


@pytest.mark.parametrize("case", GOLDEN, ids=lambda c: c["config"])
def test_budget_matches_golden(pkg, ref_configs, case):
    """Against the reference program's output stored in tests/golden (for
    machines without the compiled reference)."""
    m = ref_configs[case["config"]]
    ch, p = _channel(pkg, m, case["steps"])
    ours = ch.tke_budget()
    ref = np.array(case["profiles"])
    assert_profiles(ours, ref, pkg.TKE_NAMES)
    ch.close()


def test_budget_fp32_state_close_to_fp64(pkg, ref_configs):
    """The FP32 form's fields give the same statistics to its precision."""
    m = ref_configs["c1"]
    a, _ = _channel(pkg, m, 6)
    b, _ = _channel(pkg, m, 6, precision=pkg.FP32)
    pa, pb = a.tke_budget(), b.tke_budget()
    for name in ("UAVG", "UTIN", "VTIN", "WTIN", "uw", "DAVG"):
        r = pkg.TKE_NAMES.index(name)
        np.testing.assert_allclose(pb[r], pa[r], rtol=0, atol=1e-4 * np.max(np.abs(pa[r])), err_msg=name)
    a.close()
    b.close()


def test_budget_rejects_small_grids(pkg, ref_configs):
    m = ref_configs["t_noslip"]   # zds = 4: the wall stencils need 5 planes
    ch = pkg.Channel(params_for(pkg, m, "const", GCONST))
    ch.init_seeded(1, 0.05, 0.005)
    with pytest.raises(pkg.DnsError) as e:
        ch.tke_budget()
    assert e.value.code == pkg.DNS_EINVAL
    ch.close()
