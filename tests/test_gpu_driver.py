"""The host driver dns_run against the unmodified reference main program
(needs a B200 and the compiled reference main, oracle/_ref/<config>/ref_main).

Both programs start from the same inputs in their own directories: mode -p
from restart files of counter TSTR, mode -s from rest, mode -i from a
uniform-grid lbf.TSTR.  With ITER = 50 and one coarse step per unit time they
write restart files at counters 100 and 150, field and statistics files at
every counter and the six per-step text logs.  Every such file of the
reference has a counterpart from dns_run with the same name and layout; the
values agree to the constant-flow-rate tolerance (the force is summed in
another order on the device, 1e-12 relative on the populations).  In mode -i
only the start is compared: the reference's inter_init slips (not
reproduced) make the two runs part after it.  tests/test_driver.py makes the
same comparisons on the host, bit for bit, with the channel held by the
oracle.
"""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

from conftest import PKG_NAME, ROOT, gpu_available, ref_binary, write_definitions
from test_gpu_parity import RTOL_CFR, params_for

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]

DRIVER = ROOT / PKG_NAME / "dns_run"
LOGS = ("flowrate.txt", "density.txt", "str-up.txt", "str-do.txt", "w-str.txt", "p-grad.txt")


def _programs(name):
    exe = ref_binary(name, "ref_main")
    if exe is None or not DRIVER.exists():
        pytest.skip("compiled reference main or dns_run not available")
    return exe


def _run_both(exe, m, mode, a, b, extra=()):
    ra = subprocess.run([str(exe), f"-{mode}"], cwd=a, capture_output=True, text=True, timeout=600)
    assert ra.returncode == 0, ra.stderr[-2000:]
    write_definitions(m, b / "definitions.h")
    rb = subprocess.run([str(DRIVER), f"-{mode}", *extra], cwd=b, capture_output=True, text=True, timeout=600)
    assert rb.returncode == 0, rb.stderr[-2000:]


def _close(x, y, rtol, atol, what):
    assert x.shape == y.shape, what
    np.testing.assert_allclose(x, y, rtol=rtol, atol=atol, err_msg=what)


def _compare_dirs(a, b, first_only=False):
    """Every restart, field and statistics file of the reference run (a) has
    a counterpart in b that agrees; the per-step logs agree line by line.
    first_only: contents of what iteration 0 writes (files of counter 100, the
    first log line) only."""
    names = sorted(p.name for p in a.iterdir()
                   if p.name.startswith(("lbf-", "force.", "vel-", "den-", "turb-fld.")))
    assert any(n.startswith("lbf-c.") for n in names) and any(n.startswith("vel-") for n in names)
    for n in names:
        assert (b / n).exists(), n
        if first_only and (not n.endswith((".0100", ".100")) or n.startswith(("lbf-lin.", "lbf-uin."))):
            continue
        x, y = np.fromfile(b / n), np.fromfile(a / n)
        if n.startswith(("lbf-c.", "lbf-slf.", "lbf-suf.")):
            # [ftemp | f]: the first half is the state; the reference's second
            # half is its scratch lattice
            assert x.size == y.size, n
            x, y = x[: x.size // 2], y[: y.size // 2]
            _close(x, y, RTOL_CFR, 0.0, n)
        elif n.startswith(("lbf-lin.", "lbf-uin.", "force.")):
            _close(x, y, RTOL_CFR, 1e-14, n)
        else:
            _close(x, y, 1e-9, 1e-12 * max(1.0, float(np.max(np.abs(y)))), n)
    for n in LOGS:
        la = (a / n).read_text().splitlines()
        lb = (b / n).read_text().splitlines()
        assert len(la) == len(lb) == 51, n
        if first_only:
            la, lb = la[:1], lb[:1]
        ta = [ln.split()[0] for ln in la]
        tb = [ln.split()[0] for ln in lb]
        assert ta == tb, n
        va = np.array([float(ln.split()[1]) for ln in la])
        vb = np.array([float(ln.split()[1]) for ln in lb])
        _close(vb, va, 1e-10, 2e-12, n)
    for n in ("uavg-temp.dat", "uavg-exact-lam.dat")[first_only:]:
        _close(np.loadtxt(b / n), np.loadtxt(a / n), 1e-9, 2e-12, n)


def _dirs(tmp_path):
    a, b = tmp_path / "reference", tmp_path / "driver"
    a.mkdir()
    b.mkdir()
    return a, b


@pytest.mark.parametrize("name", ["t_noslip", "t_ridges"])
def test_mode_p_matches_reference_main(pkg, ref_configs, tmp_path, name):
    exe = _programs(name)
    m = ref_configs[name]
    a, b = _dirs(tmp_path)
    ch = pkg.Channel(params_for(pkg, m, "cfr"))
    ch.init_seeded(42, 0.05, 0.005)
    for d in (a, b):
        ch.write_restart(d, int(m["TSTR"]))
    ch.close()
    _run_both(exe, m, "p", a, b)
    _compare_dirs(a, b)


def test_mode_s_matches_reference_main(ref_configs, tmp_path):
    exe = _programs("t_noslip")
    m = ref_configs["t_noslip"]
    a, b = _dirs(tmp_path)
    _run_both(exe, m, "s", a, b)
    _compare_dirs(a, b)


def test_mode_i_matches_reference_main(port, ref_configs, tmp_path):
    exe = _programs("t_ridges")
    m = ref_configs["t_ridges"]
    a, b = _dirs(tmp_path)
    xu, yu, zu, tstr = int(m["xdu"]), int(m["ydu"]), int(m["zdu"]), int(m["TSTR"])
    first, second = port.uniform_state(xu, yu, zu, 1), port.uniform_state(xu, yu, zu, 2)
    for d in (a, b):
        port.write_uniform_file(d / f"lbf.{tstr:04d}", first, second)
    _run_both(exe, m, "i", a, b)
    # the reference's inter_init fills the interface history with two slips
    # that are not reproduced (test_oracle.py pins them), so the runs part
    # after the start: the start itself and the file set are compared
    _compare_dirs(a, b, first_only=True)


def test_fp32_driver_run_tracks_fp64(pkg, ref_configs, tmp_path):
    """The same mode -p run in the FP32 form: its restart files hold the
    FP64 run's populations, and its logs the FP64 run's values, within the
    FP32 form's bars."""
    if not DRIVER.exists():
        pytest.skip("dns_run not available")
    m = ref_configs["t_ridges"]
    a, b = _dirs(tmp_path)
    ch = pkg.Channel(params_for(pkg, m, "cfr"))
    ch.init_seeded(42, 0.05, 0.005)
    for d in (a, b):
        ch.write_restart(d, int(m["TSTR"]))
        write_definitions(m, d / "definitions.h")
    ch.close()
    for d, extra in ((a, []), (b, ["--fp32"])):
        r = subprocess.run([str(DRIVER), "-p", *extra], cwd=d, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
    for n in ("lbf-c.0150", "lbf-slf.0150", "lbf-suf.0150"):
        x, y = np.fromfile(b / n), np.fromfile(a / n)
        # the FP32 bar after 100 steps of the plain channel (test_gpu_fp32)
        assert np.max(np.abs(x[: x.size // 2] - y[: y.size // 2])) < 1e-5, n
    for n in ("flowrate.txt", "density.txt", "w-str.txt"):
        v64 = np.loadtxt(a / n)[:, 1]
        v32 = np.loadtxt(b / n)[:, 1]
        np.testing.assert_allclose(v32, v64, rtol=0, atol=1e-3 * np.max(np.abs(v64)), err_msg=n)


BUDGET = ROOT / PKG_NAME / "dns_budget"


@pytest.mark.parametrize("name", ["t_odd", "c1"])
def test_budget_program_matches_reference_program(pkg, ref_configs, tmp_path, name):
    """dns_budget and the reference's budget program (TKE-budget/computations,
    compiled unmodified) on the same vel-* / den-* snapshot: the three profile
    files within 1e-11 of each profile's scale (test_gpu_tke.py's bar), the
    fluctuation planes where the counter is a multiple of 200."""
    exe = ref_binary(name, "tke_budget")
    if exe is None or not BUDGET.exists():
        pytest.skip("compiled reference budget program or dns_budget not available")
    m = ref_configs[name]
    cntr = int(m["TSTR"])
    # both programs run in a subdirectory of the run and read its fields from ".."
    ch = pkg.Channel(params_for(pkg, m, "cfr"))
    ch.init_seeded(42, 0.05, 0.005)
    ch.step(6)
    ch.write_fields(tmp_path, cntr)
    ch.close()
    a, b = _dirs(tmp_path)
    subprocess.run([str(exe)], cwd=a, check=True, capture_output=True, timeout=600)
    write_definitions(m, b / "definitions.h", TEND=cntr)
    r = subprocess.run([str(BUDGET)], cwd=b, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    for fname, n in pkg.TKE_FILES:
        x = np.fromfile(b / f"{fname}.000.{cntr:04d}").reshape(n, -1)
        y = np.fromfile(a / f"{fname}.000.{cntr:04d}").reshape(n, -1)
        for row in range(n):
            scale = float(np.max(np.abs(y[row])))
            np.testing.assert_allclose(x[row], y[row], rtol=0, atol=1e-11 * scale + 1e-300, err_msg=f"{fname} {row}")
    if cntr % 200 == 0:
        for fn in ("ufl4", "vfl4"):
            np.testing.assert_allclose(np.fromfile(b / f"{fn}.{cntr:04d}"), np.fromfile(a / f"{fn}.{cntr:04d}"),
                                       rtol=0, atol=1e-15, err_msg=fn)
