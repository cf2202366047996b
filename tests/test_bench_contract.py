"""bench.py's reference arm on the host (no GPU): one JSON line with the
contract's keys, timing the compiled reference on the host cores; under N
ranks only rank 0 runs and prints, the others exit 0 without work."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT, ref_binary


def _run(env_extra, config="c1"):
    env = dict(os.environ, **env_extra)
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--config", config,
                        "--steps", "1", "--warmup", "0"], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return [ln for ln in r.stdout.splitlines() if ln.startswith("{")]


def test_reference_arm_prints_the_contract_line():
    if ref_binary("c1") is None:
        pytest.skip("compiled reference not available")
    lines = _run({"RANK": "0", "WORLD_SIZE": "1"})
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "MLUPS" and d["higher_is_better"] is True
    assert d["metric"].startswith("MLUPS") and d["config"]["workload"] == "c1"
    assert d["value"] > 0 and d["ms_per_step"] > 0 and d["n_gpus"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # the same workload description as the main line, and the step counts it ran
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    args = type("A", (), {"config": "c1"})()
    assert d["config"] == bench.arm_config(args, 1)
    assert d["steps"] == 1 and d["warmup"] == 3  # W is raised to the contract's minimum of 3
    assert "after 3 untimed" in cb["sample"]


def test_reference_arm_runs_on_rank_zero_only():
    if ref_binary("c1") is None:
        pytest.skip("compiled reference not available")
    assert _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}) == []
    d = json.loads(_run({"RANK": "0", "WORLD_SIZE": "2", "LOCAL_RANK": "0"})[0])
    assert d["n_gpus"] == 2 and d["value"] > 0
