"""C ABI surface and host-only logic (no GPU calls)."""
from __future__ import annotations

import ctypes as C
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HEADER = ROOT / "include" / "dns_embed.h"


def declared_symbols():
    txt = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(dns_\w+)\s*\(", txt, re.M)))


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg.lib()
    syms = declared_symbols()
    assert len(syms) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", str(pkg.LIBPATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (dns_\w+)", out))
    missing = [s for s in syms if s not in exported]
    assert not missing, missing
    for s in syms:
        assert getattr(lib, s) is not None


def test_defaults_mirror_reference_definitions(pkg):
    p = pkg.default_params()
    assert (p.xdv, p.ydv, p.zdv, p.zds, p.gratio) == (512, 256, 220, 10, 4)
    assert (p.xdu, p.ydu, p.zdu, p.fltr) == (512, 256, 221, 0)
    assert p.Rebs == 7200.0 and p.ub == 0.0866034 and p.CFL == 0.1
    assert p.pattern == pkg.PATTERN_RSLIP and p.ITER < 0


def test_params_from_definitions_file(pkg, tmp_path):
    src = tmp_path / "definitions.h"
    src.write_text("""
#define Rebs 5533.0
#define ub 0.0866034
#define zdv  83
#define ydv  128
#define xdv  256
#define gratio 2
#define zds 16
#define gyplussize 24
#define wyplussize 24
//#define PSLIP
#define RSLIP
//#define SSLIP
#define XDIM 4
#define YDIM 2
#define NOFLTR
//#define FLTR
//#define ITER 1
#define xdu 384
#define ydu 192
#define zdu 95
""")
    p = pkg.params_from_definitions(src)
    assert (p.xdv, p.ydv, p.zdv, p.zds, p.gratio) == (256, 128, 83, 16, 2)
    assert p.pattern == pkg.PATTERN_RSLIP and p.ITER < 0 and p.Rebs == 5533.0
    assert (p.xdu, p.ydu, p.zdu) == (384, 192, 95) and p.fltr == 0
    src.write_text(src.read_text().replace("#define NOFLTR", "//#define NOFLTR").replace("//#define FLTR",
                                                                                        "#define FLTR"))
    assert pkg.params_from_definitions(src).fltr == 1
    with pytest.raises(pkg.DnsError) as e:
        pkg.params_from_definitions(tmp_path / "missing.h")
    assert e.value.code == pkg.DNS_EIO


def test_geometry_matches_reference_formulas(pkg, port, ref_configs):
    for name in ("t_noslip", "t_gr4", "c1", "c2"):
        m = ref_configs[name]
        p = pkg.make_params(xdv=m["xdv"], ydv=m["ydv"], zdv=m["zdv"], zds=m["zds"], gratio=m["gratio"],
                            Rebs=float(m["Rebs"]), ub=m["ub"], CFL=m["CFL"], pattern=m.get("pattern"))
        g = pkg.geometry(p)
        q = port.Port(m)
        oc, of, nzs = q.params()
        assert g.nzs == nzs and g.omega_c == oc and g.omega_f == of
        gr = m["gratio"]
        assert g.updates_per_step == m["xdv"] * m["ydv"] * m["zdv"] + 2 * gr * (gr * m["xdv"]) * (gr * m["ydv"]) * m["zds"]
    # config 1 / 2 work units quoted by the survey
    p1 = pkg.make_params(xdv=64, ydv=64, zdv=27, zds=8, gratio=2)
    assert pkg.geometry(p1).updates_per_step == 634880
    p2 = pkg.make_params(xdv=256, ydv=128, zdv=83, zds=16, gratio=2)
    assert pkg.geometry(p2).updates_per_step == 11108352


@pytest.mark.parametrize("bad", [dict(gratio=1), dict(zds=2), dict(zdv=3), dict(xdv=2), dict(Rebs=-1.0),
                                 dict(pattern=9), dict(precision=7), dict(fltr=2),
                                 dict(fltr=1),                       # FLTR is defined for gratio 4
                                 dict(fltr=1, gratio=4, zds=6),      # and needs zds >= 7
                                 dict(xdv=1 << 20),                  # 32-bit population offsets
                                 dict(xdv=1 << 14, ydv=1 << 14, zdv=16),
                                 dict(xdv=1 << 14, ydv=1 << 12, zds=16)])
def test_invalid_parameters_are_rejected(pkg, bad):
    p = pkg.make_params(xdv=16, ydv=16, zdv=9, zds=6, gratio=2)
    for k, v in bad.items():
        setattr(p, k, v)
    with pytest.raises(pkg.DnsError) as e:
        pkg.geometry(p)
    assert e.value.code == pkg.DNS_EINVAL


def test_error_strings(pkg):
    lib = pkg.lib()
    for code in (0, -1, -2, -3, -4, -5, -6):
        assert lib.dns_error_string(code)


def test_python_structs_match_the_header_layout(pkg, tmp_path):
    """The ctypes mirrors have the C structs' sizes and field offsets (a
    program built with gcc against include/dns_embed.h prints them)."""
    pairs = [("dns_params", pkg.Params), ("dns_geometry", pkg.Geometry), ("dns_step_log", pkg.StepLog),
             ("dns_tile", pkg.Tile), ("dns_batch_info", pkg.BatchInfo)]
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "dns_embed.h"', "int main(void) {"]
    for cname, py in pairs:
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", str(HEADER.parent), str(src), "-o", str(exe)],
                   check=True)
    got = {}
    for ln in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        cname, key, val = ln.split()
        got[(cname, key)] = int(val)
    for cname, py in pairs:
        assert got[(cname, "sizeof")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


# ---- allocation-free reduction: the checks made before any device work ----
STATIC_PAIRS = 262144  # slots of the scratch array compiled into the library


def flow_sums_pairs(xdv, ydv, zdv, zds, gratio, bx=128, jb=2):
    """Reduction blocks of the direct encalc2 pass: max(fine, coarse) x/y block
    counts of the kernels' launch shape (bx threads along x, jb rows) times
    the coarse planes plus both fine blocks' planes."""
    nxf, nyf = gratio * xdv, gratio * ydv
    gx = max(-(-nxf // bx), -(-xdv // bx))
    gy = max(-(-nyf // jb), -(-ydv // jb))
    return gx * gy * (zdv + 2 * zds)


def _static_fn(pkg):
    fn = pkg.lib().dns_flow_sums_static
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(pkg.Params), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return fn


def test_static_scratch_covers_the_superhydrophobic_channel():
    # the 384 x 128 x 192 channel (xdv 384, ydv 192, zdv 115, zds 16): 6 x 192 x 147 blocks
    assert flow_sums_pairs(384, 192, 115, 16, 2) == 169344 <= STATIC_PAIRS
    # the boundary cases the GPU test and the rejection test use
    assert flow_sums_pairs(64, 4096, 48, 8, 2) == STATIC_PAIRS
    assert flow_sums_pairs(2368, 109, 33, 16, 2) == STATIC_PAIRS + 1


def test_static_reduction_refusals_touch_no_device(pkg):
    fn = _static_fn(pkg)
    dummy = C.c_double()
    ptr = C.addressof(dummy)
    # one slot beyond the array
    p = pkg.make_params(xdv=2368, ydv=109, zdv=33, zds=16, gratio=2)
    assert fn(C.byref(p), ptr, ptr, ptr, None) == pkg.DNS_EINVAL
    assert b"262145 reduction slots" in pkg.lib().dns_last_error()
    # the FP32 layout is not read
    p = pkg.make_params(xdv=16, ydv=16, zdv=9, zds=4, gratio=2, precision=pkg.FP32)
    assert fn(C.byref(p), ptr, ptr, ptr, None) == pkg.DNS_EINVAL
    assert b"DNS_FP64" in pkg.lib().dns_last_error()
    # invalid geometry: dns_geometry_of's own message is kept
    p = pkg.make_params(xdv=16, ydv=16, zdv=9, zds=4, gratio=1)
    assert fn(C.byref(p), ptr, ptr, ptr, None) == pkg.DNS_EINVAL
    msg = pkg.lib().dns_last_error()
    assert b"gratio" in msg and b"invalid parameters" not in msg
