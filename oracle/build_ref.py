"""Build recipe for the compiled reference — TEST INFRASTRUCTURE ONLY (oracle).

Compiles the reference solver's own C sources, where they lie under the mounted
reference tree, into ``oracle/_ref/<config>/``:

* ``ref_harness`` — every ``DNS-solver-with-grid-embedding/src/*.c`` except the
  main program, plus ``oracle/ref_harness.c`` (drives the routines in the main
  loop's order) and the single-rank MPI shim;
* ``ref_main`` (configurations that ask for it) — the unmodified main program
  ``dns-q-mgrd-all-patterns-xyc.c`` with the same routines and the shim;
* ``tke_budget`` (configurations with ``tke``) — the unmodified turbulence
  statistics / kinetic-energy budget program of ``TKE-budget/computations/``
  (``budget-no-slip-mgrd.c`` with ``reading.c``, ``budget2D.c``, ``uv_fluc.c``
  ...), configured through its own ``definitions.h`` with the same grid and
  ``TSTR = TEND`` = the configuration's ``TSTR``; it reads ``../vel-*.TTTT`` /
  ``../den-*.TTTT`` relative to its working directory.

The reference has no build system beyond a two-line Makefile (``mpicc -O3``).
It configures itself only through compile-time macros in ``src/definitions.h``
(no ``#ifndef`` guards), and every source includes it with a quoted include, so
it cannot be overridden with ``-I``.  This recipe therefore writes a copy of
that header with the configuration's macro values into the build folder and
places symbolic links to the unmodified ``.c`` files beside it; the links and
the header copy are deleted after linking, so only the two binaries stay in
``oracle/_ref/`` (which is git-ignored).

Flags: ``-O3`` (the reference's own) plus ``-ffp-contract=off`` so no fused
multiply-add is formed (x86-64 baseline code has none anyway) and ``-fcommon``
because ``definitions.h`` defines ``DP PI;`` in every translation unit.

Run ``python oracle/build_ref.py [config ...]``; with no argument every
configuration in ``REF_CONFIGS`` is built.  Needs the reference tree, found at
``$DNS_REFERENCE_ROOT`` (default: the tree's mount point, ``REFERENCE_ROOT`` below).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
# root of the reference project's tree (read-only); DNS_REFERENCE_ROOT overrides it
REFERENCE_ROOT = Path(os.environ.get("DNS_REFERENCE_ROOT", "/root/reference"))
REF_SRC = REFERENCE_ROOT / "DNS-solver-with-grid-embedding" / "src"
TKE_SRC = REFERENCE_ROOT / "TKE-budget" / "computations"
# macros of TKE-budget/computations/definitions.h:21-47 taken from the configuration
TKE_MACROS = ("zdv", "ydv", "xdv", "CFL", "Rebs", "ub", "gratio", "zds", "TSTR", "TEND", "DT")
OUT = HERE / "_ref"
SHIM = HERE / "mpi_shim"
MAIN_FILE = "dns-q-mgrd-all-patterns-xyc.c"

sys.path.insert(0, str(HERE))
from ref_configs import REF_CONFIGS  # noqa: E402

# macros the configurations may set (reference src/definitions.h:34-119)
VALUE_MACROS = ("Rebs", "ub", "zdv", "ydv", "xdv", "TSTR", "TEND", "CFL", "gratio", "zds",
                "gyplussize", "wyplussize", "gxplussize", "wxplussize", "XDIM", "YDIM", "xdu", "ydu", "zdu")
PATTERNS = ("PSLIP", "RSLIP", "SSLIP")
# "fltr": True selects the filtered fine-to-coarse transfer (FLTR instead of NOFLTR)


def render_definitions(cfg: dict) -> str:
    text = (REF_SRC / "definitions.h").read_text()
    out = []
    seen = set()
    for line in text.splitlines():
        m = re.match(r"^\s*(//)?\s*#define\s+(\w+)\b(.*)$", line)
        if m:
            name = m.group(2)
            if name in VALUE_MACROS and name in cfg:
                out.append(f"#define {name} {cfg[name]}")
                seen.add(name)
                continue
            if name in PATTERNS:
                out.append(f"#define {name}" if cfg.get("pattern") == name else f"//#define {name}")
                seen.add(name)
                continue
            if name in ("NOFLTR", "FLTR"):
                on = bool(cfg.get("fltr")) == (name == "FLTR")
                out.append(f"#define {name}" if on else f"//#define {name}")
                seen.add(name)
                continue
            if name == "ITER":
                out.append(f"#define ITER {cfg['ITER']}" if "ITER" in cfg else "//#define ITER 1")
                seen.add(name)
                continue
        out.append(line)
    missing = [k for k in cfg if k in VALUE_MACROS and k not in seen]
    if missing:
        raise RuntimeError(f"macros not found in the reference definitions.h: {missing}")
    return "\n".join(out) + "\n"


def render_tke_definitions(cfg: dict) -> str:
    vals = {k: cfg[k] for k in TKE_MACROS if k in cfg}
    vals["TEND"] = vals["TSTR"] = cfg["TSTR"]
    vals["DT"] = 1
    out, seen = [], set()
    for line in (TKE_SRC / "definitions.h").read_text().splitlines():
        m = re.match(r"^\s*#define\s+(\w+)\b(.*)$", line)
        if m and m.group(1) in vals:
            out.append(f"#define {m.group(1)} {vals[m.group(1)]}")
            seen.add(m.group(1))
            continue
        out.append(line)
    missing = [k for k in vals if k not in seen]
    if missing:
        raise RuntimeError(f"macros not found in the TKE-budget definitions.h: {missing}")
    return "\n".join(out) + "\n"


def _cc(args, cwd):
    r = subprocess.run(args, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(map(str, args))}\n{r.stderr}")


def build_config(name: str) -> Path:
    cfg = REF_CONFIGS[name]
    d = OUT / name
    if d.exists():
        shutil.rmtree(d)
    d.mkdir(parents=True)
    (d / "definitions.h").write_text(render_definitions(cfg))
    sources = sorted(p.name for p in REF_SRC.glob("*.c"))
    for s in sources + ["fun_defs.h"]:
        os.symlink(REF_SRC / s, d / s)
    cflags = ["gcc", "-O3", "-ffp-contract=off", "-fcommon", "-w", f"-I{d}", f"-I{SHIM}"]
    objs = []
    for s in sources:
        o = d / (s[:-2] + ".o")
        _cc(cflags + ["-c", str(d / s), "-o", str(o)], d)
        objs.append(o)
    _cc(cflags + ["-c", str(SHIM / "mpi_shim.c"), "-o", str(d / "mpi_shim.o")], d)
    _cc(cflags[:-2] + ["-Wall", f"-I{d}", f"-I{SHIM}", "-c", str(HERE / "ref_harness.c"),
                       "-o", str(d / "ref_harness.o")], d)
    lib_objs = [str(o) for o in objs if o.name != MAIN_FILE[:-2] + ".o"]
    _cc(["gcc", "-o", str(d / "ref_harness"), str(d / "ref_harness.o"), str(d / "mpi_shim.o")]
        + lib_objs + ["-lm"], d)
    if cfg.get("main"):
        _cc(["gcc", "-o", str(d / "ref_main"), str(d / "mpi_shim.o")] + [str(o) for o in objs]
            + ["-lm"], d)
    # keep only the binaries: no reference source (or header copy) stays here
    for p in d.iterdir():
        if p.name not in ("ref_harness", "ref_main"):
            p.unlink()
    if cfg.get("tke"):
        build_tke(cfg, d)
    return d


def build_tke(cfg: dict, d: Path) -> Path:
    """TKE-budget/computations compiled unmodified into d/tke_budget."""
    t = d / "tke_src"
    t.mkdir()
    (t / "definitions.h").write_text(render_tke_definitions(cfg))
    sources = sorted(p.name for p in TKE_SRC.glob("*.c"))
    for s in sources + ["fun_defs.h"]:
        os.symlink(TKE_SRC / s, t / s)
    cflags = ["gcc", "-O3", "-ffp-contract=off", "-w", f"-I{t}", f"-I{SHIM}"]
    objs = []
    for s in sources + [str(SHIM / "mpi_shim.c")]:
        o = t / (Path(s).name[:-2] + ".o")
        _cc(cflags + ["-c", str(t / s) if "/" not in s else s, "-o", str(o)], t)
        objs.append(str(o))
    _cc(["gcc", "-o", str(d / "tke_budget")] + objs + ["-lm"], t)
    shutil.rmtree(t)
    return d / "tke_budget"


def main(names):
    if not REF_SRC.is_dir():
        print("reference tree not mounted; nothing to build")
        return 0
    names = names or list(REF_CONFIGS)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for n, d in zip(names, ex.map(build_config, names)):
            print(f"built {n} -> {d.relative_to(HERE.parent)}")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
