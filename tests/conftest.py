"""Shared fixtures: the product package (CUDA library via ctypes) and the oracle.

The oracle (``oracle/``) is only the checker here.  The compiled reference
binaries (``oracle/_ref/<config>/``) are built from the mounted reference tree
when it is present; on a machine without it (the GPU box) the prebuilt binaries
are used if they travelled, and the oracle's CPU restatement is pinned by the
golden fixtures in ``tests/golden/`` instead.
"""
from __future__ import annotations

import importlib
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG_NAME = "dns-solvers-with-grid-embedding_b200"

if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
if str(ROOT / "oracle") not in sys.path:
    sys.path.insert(0, str(ROOT / "oracle"))

from build_ref import REF_SRC as REF_TREE  # noqa: E402  (the reference's solver sources, where mounted)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def load_pkg():
    return importlib.import_module(PKG_NAME)


@pytest.fixture(scope="session")
def pkg():
    return load_pkg()


@pytest.fixture(scope="session")
def port():
    import port as _port

    _port.build_port()
    return _port


@pytest.fixture(scope="session")
def ref_configs():
    from ref_configs import REF_CONFIGS

    return REF_CONFIGS


def ref_binary(name: str, kind: str = "ref_harness") -> Path | None:
    """Path of a compiled reference binary, building it when the tree is mounted."""
    p = ROOT / "oracle" / "_ref" / name / kind
    if p.exists():
        return p
    if REF_TREE.is_dir():
        subprocess.run([sys.executable, str(ROOT / "oracle" / "build_ref.py"), name], check=True,
                       capture_output=True)
        if p.exists():
            return p
    return None


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def write_definitions(m: dict, path: Path, **over) -> Path:
    """A reference-style definitions.h (#define NAME value lines) with the
    macros of an oracle configuration, as the host driver reads it."""
    m = dict(m, **over)
    lines = []
    for k in ("Rebs", "ub", "zdv", "ydv", "xdv", "TSTR", "TEND", "CFL", "gratio", "zds", "gyplussize",
              "wyplussize", "gxplussize", "wxplussize", "XDIM", "YDIM", "xdu", "ydu", "zdu"):
        if k in m:
            lines.append(f"#define {k} {m[k]}")
    if m.get("ITER") is not None:
        lines.append(f"#define ITER {int(m['ITER'])}")
    if m.get("pattern"):
        lines.append(f"#define {m['pattern']}")
    lines.append("#define FLTR" if m.get("fltr") else "#define NOFLTR")
    path.write_text("\n".join(lines) + "\n")
    return path
