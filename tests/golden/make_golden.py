"""Generate the golden fixtures of the oracle from the compiled reference.

For each case: write the seeded initial state (oracle restatement) as restart
files, run the reference's own routines (``oracle/_ref/<config>/ref_harness``,
compiled from the mounted reference sources) for N coarse steps, and record
SHA-256 digests of the post-stream lattices and interface histories it writes,
plus a few sampled values and the logged flow rate.  The tests check the CPU
restatement against these digests on machines where the reference tree is not
mounted.  A second file, ``uniform_golden.json``, holds the same digests for
mode -i starts of the unmodified reference main from a uniform-grid file, and
``tke_golden.json`` the output profiles of the reference's offline budget
program (TKE-budget/computations) on the fields of a seeded state.

``c1_1000_golden.json`` (``--c1-long``, about four minutes of CPU) holds the
plain FP64 channel c1 after its stated 1000 coarse steps, run by the
reference's own routines.

Run from the repository root: ``python tests/golden/make_golden.py`` and
``python tests/golden/make_golden.py --c1-long``.
"""
from __future__ import annotations

import hashlib
import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))

import port  # noqa: E402
from ref_configs import REF_CONFIGS  # noqa: E402

CASES = [
    ("t_noslip", "const", 20), ("t_noslip", "cfr", 20), ("t_ridges", "cfr", 20), ("t_posts", "const", 20),
    ("t_span", "cfr", 20), ("t_gr4", "cfr", 10), ("t_odd", "const", 20), ("t_gr4f", "cfr", 10),
]
SEED, UC, AMP, GCONST = 42, 0.05, 0.005, 1.0e-5


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def run_case(name, mode, n):
    m = REF_CONFIGS[name]
    p = port.Port(m)
    g = GCONST if mode == "const" else 0.0
    p.init_seeded(SEED, UC, AMP, g)
    p.set_forcing(mode == "cfr", g)
    with tempfile.TemporaryDirectory() as d:
        din, dout = Path(d, "in"), Path(d, "out")
        din.mkdir()
        dout.mkdir()
        p.save(din, 100)
        exe = ROOT / "oracle" / "_ref" / name / "ref_harness"
        subprocess.run([str(exe), str(din), "100", str(dout), "101", str(n), mode, g.hex()], check=True,
                       capture_output=True)
        nx, ny, zdc, nxf, nyf, zdf = p.nx, p.ny, p.zdc, p.nxf, p.nyf, p.zdf
        out = {"config": name, "mode": mode, "steps": n, "seed": SEED, "uc": UC, "amp": AMP, "g": g}
        shapes = {"lbf-c": (nx, ny, zdc, 19), "lbf-slf": (nxf, nyf, zdf, 19), "lbf-suf": (nxf, nyf, zdf, 19)}
        for fn, sh in shapes.items():
            a = np.fromfile(dout / f"{fn}.0101")
            s = a[: a.size // 2].reshape(sh)
            out[fn] = {"sha256": digest(s), "sum": float(s.sum()), "sample": [float(x) for x in s.reshape(-1)[::997][:16]]}
        for w in ("lin", "uin"):
            h = np.fromfile(dout / f"lbf-{w}.0101").reshape(3, nx, ny, 23)
            out[f"lbf-{w}"] = {"sha256": digest(h)}
        out["force_next"] = float(np.fromfile(dout / "force.0101")[0])
        fl = np.loadtxt(dout / "flowrate.txt")
        out["flowrate_log"] = [float(x) for x in np.atleast_2d(fl)[:, 1]]
    return out


# mode -i starts: the unmodified reference main (``ref_main -i``) reads a
# uniform-grid lbf.TSTR built by port.uniform_state and writes its restart at
# the first iteration, before any step
UNIFORM_CASES = [("t_noslip", 1, 2), ("t_ridges", 3, 4)]


def run_uniform_case(name, seed_first, seed_second):
    m = REF_CONFIGS[name]
    xu, yu, zu, tstr = int(m["xdu"]), int(m["ydu"]), int(m["zdu"]), int(m["TSTR"])
    p = port.Port(m)
    out = {"config": name, "uniform": [xu, yu, zu], "seeds": [seed_first, seed_second], "cntr": tstr}
    with tempfile.TemporaryDirectory() as d:
        port.write_uniform_file(Path(d, f"lbf.{tstr:04d}"), port.uniform_state(xu, yu, zu, seed_first),
                                port.uniform_state(xu, yu, zu, seed_second))
        exe = ROOT / "oracle" / "_ref" / name / "ref_main"
        subprocess.run([str(exe), "-i"], cwd=d, check=True, capture_output=True)
        nx, ny, zdc, nxf, nyf, zdf = p.nx, p.ny, p.zdc, p.nxf, p.nyf, p.zdf
        shapes = {"lbf-c": (nx, ny, zdc, 19), "lbf-slf": (nxf, nyf, zdf, 19), "lbf-suf": (nxf, nyf, zdf, 19)}
        for fn, sh in shapes.items():
            a = np.fromfile(Path(d, f"{fn}.{tstr:04d}"))
            s = a[: a.size // 2].reshape(sh)
            out[fn] = {"sha256": digest(s), "sum": float(s.sum())}
        lin = np.fromfile(Path(d, f"lbf-lin.{tstr:04d}")).reshape(3, nx, ny, 23)
        uin = np.fromfile(Path(d, f"lbf-uin.{tstr:04d}")).reshape(3, nx, ny, 23)
        # level n: f^neq of the lower and upper planes; the density and velocity
        # the reference writes into the lower history are the upper plane's
        out["lin_fneq_n"] = digest(lin[0, ..., 4:])
        out["uin_fneq_n"] = digest(uin[0, ..., 4:])
        out["upper_moments_n"] = digest(lin[0, ..., :4])
        out["force"] = float(np.fromfile(Path(d, f"force.{tstr:04d}"))[0])
    return out


# the reference's offline budget program (oracle/_ref/<config>/tke_budget) on
# the fields of a seeded state after a few constant-force coarse steps, written
# by the reference's own vel_print through the harness
TKE_CASES = [("t_odd", 6), ("t_gr4", 4)]


def run_tke_case(name, steps):
    m = REF_CONFIGS[name]
    cntr = int(m["TSTR"])
    p = port.Port(m)
    p.init_seeded(42, UC, AMP, GCONST)
    p.set_forcing(False, GCONST)
    with tempfile.TemporaryDirectory() as d:
        din, dout = Path(d, "in"), Path(d, "out")
        din.mkdir()
        (dout / "tke").mkdir(parents=True)
        p.save(din, cntr - 1)
        exe = ROOT / "oracle" / "_ref" / name / "ref_harness"
        subprocess.run([str(exe), str(din), str(cntr - 1), str(dout), str(cntr), str(steps), "const",
                        GCONST.hex(), "0", "1"], check=True, capture_output=True)
        subprocess.run([str(ROOT / "oracle" / "_ref" / name / "tke_budget")], cwd=dout / "tke", check=True,
                       capture_output=True)
        nz = 2 * (int(m["zds"]) + 1) + int(m["zdv"]) - 4
        prof = []
        for fn in ("turb-fld-2d", "vort-fluc-2d", "KE-Budget-2d"):
            prof.extend(np.fromfile(dout / "tke" / f"{fn}.000.{cntr:04d}").reshape(-1, nz).tolist())
    return {"config": name, "seed": SEED, "uc": UC, "amp": AMP, "g": GCONST, "steps": steps, "profiles": prof}


# the plain FP64 channel of the parity configuration (c1: reference macros xdv
# 64, ydv 64, zdv 27, zds 8, GR 2) run for its stated 1000 coarse steps by the
# reference's own routines: with the constant body force of Re_tau = 180
# (g_c = GR u_tau^2 / h_f) the digests of the lattices, which the FP64 form
# reproduces bit for bit; at constant flow rate, whose whole-domain flow-rate
# sum is associated differently, per-population plane sums of each lattice
# and the logged flow rate, compared at 1e-12
C1_LONG_STEPS = 1000


def c1_force(m):
    nzs = 2 * (int(m["zds"]) + 1) + int(m["gratio"]) * (int(m["zdv"]) - 4) + int(m["gratio"]) - 1
    tau_f = (3.0 / float(m["Rebs"])) * float(m["ub"]) * (nzs - 2.0) + 0.5
    nu_f = (tau_f - 0.5) / 3.0
    h_f = (nzs - 2) / 2.0
    u_tau = 180.0 * nu_f / h_f
    return int(m["gratio"]) * u_tau * u_tau / h_f


def plane_sums(s: np.ndarray) -> list:
    """(nx, ny, nz, 19) lattice -> sums over x and y per (z, population), [nz][19]."""
    return s.sum(axis=(0, 1)).tolist()


def run_c1_long(mode):
    name, n = "c1", C1_LONG_STEPS
    m = REF_CONFIGS[name]
    p = port.Port(m)
    g = c1_force(m) if mode == "const" else 0.0
    p.init_seeded(SEED, UC, AMP, g)
    p.set_forcing(mode == "cfr", g)
    with tempfile.TemporaryDirectory() as d:
        din, dout = Path(d, "in"), Path(d, "out")
        din.mkdir()
        dout.mkdir()
        p.save(din, 100)
        exe = ROOT / "oracle" / "_ref" / name / "ref_harness"
        subprocess.run([str(exe), str(din), "100", str(dout), "101", str(n), mode, g.hex()], check=True,
                       capture_output=True)
        nx, ny, zdc, nxf, nyf, zdf = p.nx, p.ny, p.zdc, p.nxf, p.nyf, p.zdf
        out = {"config": name, "mode": mode, "steps": n, "seed": SEED, "uc": UC, "amp": AMP, "g": g}
        shapes = {"lbf-c": (nx, ny, zdc, 19), "lbf-slf": (nxf, nyf, zdf, 19), "lbf-suf": (nxf, nyf, zdf, 19)}
        for fn, sh in shapes.items():
            a = np.fromfile(dout / f"{fn}.0101")
            s = a[: a.size // 2].reshape(sh)
            out[fn] = {"sha256": digest(s), "plane_sums": plane_sums(s)}
        for w in ("lin", "uin"):
            h = np.fromfile(dout / f"lbf-{w}.0101").reshape(3, nx, ny, 23)
            out[f"lbf-{w}"] = {"sha256": digest(h)}
        out["force_next"] = float(np.fromfile(dout / "force.0101")[0])
        fl = np.loadtxt(dout / "flowrate.txt")
        out["flowrate_log"] = [float(x) for x in np.atleast_2d(fl)[:, 1]]
    return out


def main():
    if "--c1-long" in sys.argv:
        long_cases = [run_c1_long(mode) for mode in ("const", "cfr")]
        (Path(__file__).parent / "c1_1000_golden.json").write_text(json.dumps(long_cases))
        print("wrote the c1 1000-step cases")
        return
    cases = [run_case(*c) for c in CASES]
    (Path(__file__).parent / "oracle_golden.json").write_text(json.dumps(cases, indent=1))
    print(f"wrote {len(cases)} cases")
    uni = [run_uniform_case(*c) for c in UNIFORM_CASES]
    (Path(__file__).parent / "uniform_golden.json").write_text(json.dumps(uni, indent=1))
    print(f"wrote {len(uni)} uniform-start cases")
    tke = [run_tke_case(*c) for c in TKE_CASES]
    (Path(__file__).parent / "tke_golden.json").write_text(json.dumps(tke))
    print(f"wrote {len(tke)} budget cases")


if __name__ == "__main__":
    main()
