"""The host driver dns_run on the host alone (no GPU): argument handling,
parameters read from a reference-style definitions.h, and the output
schedule of the reference main loop (dns-q-mgrd-all-patterns-xyc.c:1254-1381:
restart files every 50 unit times, fields and plane statistics every unit
time, of the pre-step state, under counter TSTR + ss / utime; ITER + 1 or
(TEND - TSTR) utime + 1 loop iterations; the statistics once more at the end)."""
from __future__ import annotations

import subprocess

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
