"""Build the CUDA library ``libdnsembed.so`` in-tree for sm_100a, and the host
programs ``dns_run`` (the solver) and ``dns_budget`` (the budget analysis),
plain C over the library's C ABI.

``kernels_f64.cu`` is compiled with ``-fmad=false``: the FP64 plain form must
not fuse multiply-adds, so that its per-node arithmetic rounds exactly like the
reference.  ``tke.cu`` (the statistics / budget analysis) likewise.  Everything else uses the default flags.  Run
``python build.py`` (or call ``build()``); nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "libdnsembed.so"
PROGRAMS = (HERE / "dns_run", HERE / "dns_budget")
INCLUDE = HERE.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", str(INCLUDE), "-I", str(CSRC)]
UNITS = {  # source -> extra flags
    "kernels_f64.cu": ["-fmad=false"],
    "kernels_f32.cu": [],
    "batch_f32.cu": [],
    "dns_api.cu": [],
    "batch_api.cu": [],
    "noalloc.cu": [],
    "tke.cu": ["-fmad=false"],
}


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (Path(c).exists() or c == "nvcc"):
            return c
    return "nvcc"


def _stale(obj: Path, deps) -> bool:
    return not obj.exists() or any(d.stat().st_mtime > obj.stat().st_mtime for d in deps)


def build(verbose: bool = False) -> Path:
    """Compile stale units and link.  Extra nvcc flags (e.g. a tuning macro
    such as -DDNS_ITY=16) can be given in DNS_NVCC_FLAGS; touch the sources to
    rebuild with them."""
    nvcc = _nvcc()
    extra_env = os.environ.get("DNS_NVCC_FLAGS", "").split()
    gen = CSRC / "bicubic_gen.cuh"
    if _stale(gen, [CSRC / "gen_bicubic.py"]):
        subprocess.run([sys.executable, str(CSRC / "gen_bicubic.py")], check=True)
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [INCLUDE / "dns_embed.h"]
    objs = []
    build_dir = HERE / "_build"
    build_dir.mkdir(exist_ok=True)
    for src, extra in UNITS.items():
        obj = build_dir / (Path(src).stem + ".o")
        if _stale(obj, [CSRC / src] + headers):
            cmd = [nvcc] + ARCH + COMMON + extra + extra_env + ["-c", str(CSRC / src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
        objs.append(obj)
    if _stale(OUT, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", str(OUT)] + [str(o) for o in objs] + ["-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    # the host programs (C, against the C ABI only), found next to the library
    for exe in PROGRAMS:
        src = CSRC / (exe.name + ".c")
        if _stale(exe, [src, INCLUDE / "dns_embed.h", OUT]):
            cmd = ["gcc", "-O2", "-std=c11", "-Wall", "-Werror", "-I", str(INCLUDE), str(src), "-o", str(exe),
                   "-L", str(HERE), "-ldnsembed", "-Wl,-rpath,$ORIGIN", "-lm"]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(verbose=True))
