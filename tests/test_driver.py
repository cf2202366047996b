"""The host driver dns_run on the host alone (no GPU): argument handling,
parameters read from a reference-style definitions.h, and the output
schedule of the reference main loop (dns-q-mgrd-all-patterns-xyc.c:1254-1381:
restart files every 50 unit times, fields and plane statistics every unit
time, of the pre-step state, under counter TSTR + ss / utime; ITER + 1 or
(TEND - TSTR) utime + 1 loop iterations; the statistics once more at the end)."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

from conftest import PKG_NAME, ROOT, gpu_available, write_definitions

DRIVER = ROOT / PKG_NAME / "dns_run"


def run(args, cwd):
    if not DRIVER.exists():
        pytest.skip("dns_run is not built")
    return subprocess.run([str(DRIVER)] + args, cwd=cwd, capture_output=True, text=True, timeout=120)


@pytest.mark.parametrize("args", [[], ["-x"], ["-pp"], ["p"], ["-p", "-n"], ["-p", "-n", "-3"], ["-i", "--uc", "1"],
                                  ["-s", "--bogus"]])
def test_usage_errors_exit_2(tmp_path, args):
    r = run(args, tmp_path)
    assert r.returncode == 2 and "usage: dns_run" in r.stderr


def expected_plan(tstr, utime, up):
    out = [f"mode p utime {utime} iterations {up + 1} (steps 0..{up})"]
    for ss in range(up + 1):
        if ss % utime == 0:
            if ss % (50 * utime) == 0:
                out.append(f"ss {ss} restart {tstr + ss // utime:04d}")
            out.append(f"ss {ss} fields {tstr + ss // utime:04d} statistics {tstr + ss // utime:03d}")
    out.append(f"end statistics {tstr + (up + 1) // utime:03d}")
    return out


@pytest.mark.parametrize("name,over,n", [("t_noslip", {}, None), ("t_ridges", {}, 120),
                                         ("c1", {"ITER": None, "TSTR": 0, "TEND": 2}, None)])
def test_plan_follows_the_reference_loop(pkg, ref_configs, tmp_path, name, over, n):
    m = dict(ref_configs[name], **over)
    write_definitions(m, tmp_path / "definitions.h")
    r = run(["-p", "--plan"] + (["-n", str(n)] if n is not None else []), tmp_path)
    assert r.returncode == 0, r.stderr
    p = pkg.params_from_definitions(tmp_path / "definitions.h")
    g = pkg.geometry(p)
    # main :439-468
    utime = int((0.5 * (g.nzs - 2.0) / float(m["CFL"])) / m["gratio"])
    assert g.utime == utime >= 1
    up = n if n is not None else (int(m["ITER"]) if m.get("ITER") is not None else (m["TEND"] - m["TSTR"]) * utime)
    assert r.stdout.splitlines() == expected_plan(int(m["TSTR"]), utime, up)


def test_definitions_drive_the_parameters(pkg, ref_configs, tmp_path):
    m = ref_configs["t_ridges"]
    write_definitions(m, tmp_path / "definitions.h")
    p = pkg.params_from_definitions(tmp_path / "definitions.h")
    assert (p.xdv, p.ydv, p.zdv, p.zds, p.gratio, p.TSTR) == (m["xdv"], m["ydv"], m["zdv"], m["zds"],
                                                             m["gratio"], m["TSTR"])
    assert p.pattern == pkg.PATTERN_RSLIP and p.ITER == m["ITER"] and p.fltr == 0


def test_missing_parameters_file(tmp_path):
    r = run(["-p", "-D", "absent.h"], tmp_path)
    assert r.returncode == 1 and "cannot open absent.h" in r.stderr


@pytest.mark.skipif(gpu_available(), reason="checks the failure without a GPU")
def test_without_a_gpu_the_driver_fails_loudly(ref_configs, tmp_path):
    write_definitions(ref_configs["t_noslip"], tmp_path / "definitions.h")
    r = run(["-s"], tmp_path)
    assert r.returncode == 1 and "no CUDA device" in r.stderr
    assert not any(tmp_path.glob("lbf-*")) and not (tmp_path / "flowrate.txt").exists()


# ---- the driver's own work against the unmodified reference main, on the host:
# the channel is held by a fake of the library (tests/fake_dnsembed.c over the
# oracle's restatement, which is bit-identical to the reference), so every file
# the driver writes must equal the reference main's byte for byte (the restart
# files' second half excepted: the reference keeps its scratch lattice there)

@pytest.fixture(scope="module")
def fake_lib(tmp_path_factory):
    if not DRIVER.exists():
        pytest.skip("dns_run is not built")
    d = tmp_path_factory.mktemp("fake")
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-shared", "-fPIC", "-Wall", "-I", str(ROOT / "include"),
                    "-I", str(ROOT / "oracle"), str(ROOT / "tests" / "fake_dnsembed.c"),
                    str(ROOT / "oracle" / "dnsport.c"), "-o", str(d / "libdnsembed.so"), "-ldl", "-lm"],
                   check=True)
    return d


def run_on_fake(fake_lib, args, cwd):
    import os

    env = dict(os.environ, LD_LIBRARY_PATH=str(fake_lib), DNS_FAKE_REAL=str(ROOT / PKG_NAME / "libdnsembed.so"))
    return subprocess.run([str(DRIVER)] + args, cwd=cwd, env=env, capture_output=True, text=True, timeout=300)


def same_files(a, b, first_only=False):
    """first_only: compare the contents of what iteration 0 writes (files of
    counter TSTR, the first log line) and the names of the rest"""
    names = sorted(p.name for p in a.iterdir()
                   if p.name.startswith(("lbf-", "force.", "vel-", "den-", "turb-fld.")) or p.suffix in (".txt", ".dat")
                   and not p.name.startswith(("2dresults", "results")))
    assert len([n for n in names if n.startswith("turb-fld.")]) == 52
    for n in names:
        x, y = (b / n).read_bytes(), (a / n).read_bytes()
        if first_only and n.endswith(".txt"):
            x, y = x.splitlines()[0], y.splitlines()[0]
        elif first_only and not n.endswith((".0100", ".100")):
            continue
        if n.startswith(("lbf-c.", "lbf-slf.", "lbf-suf.")):
            assert len(x) == len(y), n
            x, y = x[: len(x) // 2], y[: len(y) // 2]
        if first_only and n.startswith(("lbf-lin.", "lbf-uin.")):
            continue  # the reference's inter_init slips (see test_oracle.py), not reproduced
        assert x == y, n
    return names


@pytest.mark.parametrize("name,mode", [("t_noslip", "p"), ("t_ridges", "p"), ("t_noslip", "s"), ("t_ridges", "i"),
                                       ("t_gr4f", "p")])
def test_driver_files_equal_reference_main(fake_lib, port, ref_configs, tmp_path, name, mode):
    from conftest import ref_binary

    exe = ref_binary(name, "ref_main")
    if exe is None:
        pytest.skip("compiled reference main not available")
    m = ref_configs[name]
    a, b = tmp_path / "reference", tmp_path / "driver"
    a.mkdir()
    b.mkdir()
    tstr = int(m["TSTR"])
    if mode == "p":
        p = port.Port(m)
        p.init_seeded(42, 0.05, 0.005, 0.0)
        p.set_forcing(True)
        for d in (a, b):
            p.save(d, tstr)
    if mode == "i":
        xu, yu, zu = int(m["xdu"]), int(m["ydu"]), int(m["zdu"])
        first, second = port.uniform_state(xu, yu, zu, 1), port.uniform_state(xu, yu, zu, 2)
        for d in (a, b):
            port.write_uniform_file(d / f"lbf.{tstr:04d}", first, second)
    subprocess.run([str(exe), f"-{mode}"], cwd=a, check=True, capture_output=True)
    write_definitions(m, b / "definitions.h")
    r = run_on_fake(fake_lib, [f"-{mode}"], b)
    assert r.returncode == 0, r.stderr
    # mode -i: the reference's inter_init fills the interface history with
    # two slips that are not reproduced, so the runs part after the start
    names = same_files(a, b, first_only=(mode == "i"))
    assert {"flowrate.txt", "w-str.txt", "p-grad.txt", "uavg-temp.dat", "lbf-c.0150", "force.0150"} <= set(names)
    assert "Total computational time is:" in (b / "report.code").read_text()


def test_non_finite_stress_ends_the_run_as_the_reference_does(fake_lib, port, ref_configs, tmp_path):
    """A NaN population next to the lower wall: both programs stop at the
    first step with exit status 1, after the flow-rate and density logs of
    that step and before its wall-stress logs (wshearstr.c:139-143)."""
    from conftest import ref_binary

    exe = ref_binary("t_noslip", "ref_main")
    if exe is None:
        pytest.skip("compiled reference main not available")
    m = ref_configs["t_noslip"]
    a, b = tmp_path / "reference", tmp_path / "driver"
    a.mkdir()
    b.mkdir()
    p = port.Port(m)
    p.init_seeded(42, 0.05, 0.005, 0.0)
    p.set_forcing(True)
    for d in (a, b):
        p.save(d, 100)
        f = np.fromfile(d / "lbf-slf.0100")
        f[((3 * p.nyf + 3) * p.zdf + 2) * 19 + 5] = np.nan
        f.tofile(d / "lbf-slf.0100")
    ra = subprocess.run([str(exe), "-p"], cwd=a, capture_output=True, text=True)
    write_definitions(m, b / "definitions.h")
    rb = run_on_fake(fake_lib, ["-p"], b)
    assert ra.returncode != 0 and rb.returncode == 1 and "NAN in wall shear stress" in rb.stderr
    for n in ("flowrate.txt", "density.txt"):
        assert (b / n).read_text() == (a / n).read_text() and len((b / n).read_text().splitlines()) == 1
    for n in ("str-up.txt", "str-do.txt", "w-str.txt", "p-grad.txt"):
        assert not (a / n).exists() and not (b / n).exists()


# ---- dns_budget, the budget program (host-only parts)
BUDGET = ROOT / PKG_NAME / "dns_budget"


def test_budget_program_arguments_and_plan(ref_configs, tmp_path):
    if not BUDGET.exists():
        pytest.skip("dns_budget is not built")
    r = subprocess.run([str(BUDGET), "-x"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 2 and "usage: dns_budget" in r.stderr
    m = dict(ref_configs["c1"])
    defs = write_definitions(m, tmp_path / "definitions.h", TSTR=150, TEND=420)
    defs.write_text(defs.read_text() + "#define DT 50\n")
    r = subprocess.run([str(BUDGET), "--plan"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    # budget-no-slip-mgrd.c: tst = TSTR .. TEND step DT, the fluctuation plane when tst % 200 == 0
    assert r.stdout.splitlines() == ["0150 budget", "0200 budget fluctuation-plane", "0250 budget", "0300 budget",
                                     "0350 budget", "0400 budget fluctuation-plane"]


def test_budget_program_reports_a_failed_snapshot(ref_configs, tmp_path):
    """No vel-* / den-* files (and, here, no GPU): status 1, the snapshot named."""
    if not BUDGET.exists():
        pytest.skip("dns_budget is not built")
    write_definitions(ref_configs["t_odd"], tmp_path / "definitions.h", TEND=ref_configs["t_odd"]["TSTR"])
    r = subprocess.run([str(BUDGET)], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 1 and "snapshot 0100" in r.stderr
    assert not any(tmp_path.glob("turb-fld-2d.*"))
