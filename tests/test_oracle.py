"""The oracle against the reference: known answers, golden fixtures, and the
compiled reference itself (CPU only)."""
from __future__ import annotations

import hashlib
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, ref_binary

GOLDEN = json.loads((ROOT / "tests" / "golden" / "oracle_golden.json").read_text())
UNIFORM_GOLDEN = json.loads((ROOT / "tests" / "golden" / "uniform_golden.json").read_text())


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def test_philox_known_answers(port):
    # Random123 known-answer vectors for Philox4x32-10 (Salmon et al. 2011)
    assert port.philox((0, 0, 0, 0), (0, 0)) == (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)
    assert port.philox((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2) == (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)
    assert port.philox((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0)) == (
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)


def test_bicubic_weights_reproduce_cubics():
    """The generated coefficient map must interpolate any bicubic exactly."""
    import importlib.util

    spec = importlib.util.spec_from_file_location(
        "gen_bicubic", ROOT / "dns-solvers-with-grid-embedding_b200" / "csrc" / "gen_bicubic.py")
    gb = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gb)
    W = np.array(gb.weights(), dtype=float)
    rng = np.random.default_rng(1)
    c = rng.normal(size=(4, 4))  # p(t,u) = sum c[n,m] t^n u^m
    corners = [(0, 0), (1, 0), (1, 1), (0, 1)]

    def ev(t, u, dn, dm):
        s = 0.0
        for n in range(4):
            for m in range(4):
                if n < dn or m < dm:
                    continue
                f = (n if dn else 1) * (m if dm else 1)
                s += c[n, m] * f * t ** (n - dn) * u ** (m - dm)
        return s

    x = [ev(t, u, dn, dm) for (dn, dm) in ((0, 0), (1, 0), (0, 1), (1, 1)) for (t, u) in corners]
    np.testing.assert_allclose(W @ np.array(x), c.reshape(-1), atol=1e-12)


def test_hermite_tensor_form_equals_bicubic_map():
    """The FP32 interface evaluates the patch as a tensor product of cubic
    Hermite bases; with exact rationals it equals the reference's coefficient
    map followed by the power-series evaluation at every GR-th point."""
    import importlib.util
    from fractions import Fraction as Fr

    spec = importlib.util.spec_from_file_location(
        "gen_bicubic", ROOT / "dns-solvers-with-grid-embedding_b200" / "csrc" / "gen_bicubic.py")
    gb = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gb)
    W = gb.weights()
    rng = np.random.default_rng(7)
    x = [Fr(int(v), 97) for v in rng.integers(-500, 500, size=16)]  # [V, Dx, Dy, Dxy] x corners
    coef = [sum(W[r][k] * x[k] for k in range(16)) for r in range(16)]
    h = [lambda t: 2 * t ** 3 - 3 * t ** 2 + 1, lambda t: -2 * t ** 3 + 3 * t ** 2,
         lambda t: t ** 3 - 2 * t ** 2 + t, lambda t: t ** 3 - t ** 2]
    corner = {(0, 0): 0, (1, 0): 1, (1, 1): 2, (0, 1): 3}
    for gr in (2, 3, 4):
        for ii in range(gr):
            for jj in range(gr):
                t, u = Fr(ii, gr), Fr(jj, gr)
                power = sum(coef[n * 4 + m] * t ** n * u ** m for n in range(4) for m in range(4))
                tensor = Fr(0)
                for a in (0, 1):
                    for b in (0, 1):
                        q = corner[(a, b)]
                        tensor += (h[a](t) * h[b](u) * x[q] + h[2 + a](t) * h[b](u) * x[4 + q]
                                   + h[a](t) * h[2 + b](u) * x[8 + q] + h[2 + a](t) * h[2 + b](u) * x[12 + q])
                assert tensor == power, (gr, ii, jj)


@pytest.mark.parametrize("case", GOLDEN, ids=lambda c: f"{c['config']}-{c['mode']}")
def test_port_matches_golden(port, ref_configs, case):
    """CPU restatement reproduces the reference's own output bit for bit."""
    p = port.Port(ref_configs[case["config"]])
    p.init_seeded(case["seed"], case["uc"], case["amp"], case["g"])
    p.set_forcing(case["mode"] == "cfr", case["g"])
    log = p.step(case["steps"])
    for lvl, fn in enumerate(("lbf-c", "lbf-slf", "lbf-suf")):
        assert _digest(p.export(lvl)) == case[fn]["sha256"], fn
    h = p.history()
    assert _digest(h[:, 0]) == case["lbf-lin"]["sha256"]
    assert _digest(h[:, 1]) == case["lbf-uin"]["sha256"]
    assert p.force() == case["force_next"]
    # the reference logs with %.12f
    np.testing.assert_allclose(log[:, 3], case["flowrate_log"][: case["steps"]], atol=6e-13, rtol=0)


@pytest.mark.parametrize("name,mode,steps", [("t_noslip", "cfr", 12), ("t_posts", "cfr", 12),
                                             ("t_gr4", "const", 6), ("t_gr4f", "cfr", 12), ("t_gr4f", "const", 6),
                                             ("t_odd", "cfr", 12)])
def test_port_matches_compiled_reference(port, ref_configs, tmp_path, name, mode, steps):
    exe = ref_binary(name)
    if exe is None:
        pytest.skip("compiled reference not available (reference tree not mounted)")
    p = port.Port(ref_configs[name])
    g = 2.0e-5 if mode == "const" else 0.0
    p.init_seeded(7, 0.04, 0.01, g)
    p.set_forcing(mode == "cfr", g)
    din, dout = tmp_path / "in", tmp_path / "out"
    din.mkdir()
    dout.mkdir()
    p.save(din, 3)
    subprocess.run([str(exe), str(din), "3", str(dout), "4", str(steps), mode, g.hex()], check=True,
                   capture_output=True)
    p.step(steps)
    for lvl, fn in enumerate(("lbf-c", "lbf-slf", "lbf-suf")):
        a = np.fromfile(dout / f"{fn}.0004")
        np.testing.assert_array_equal(p.export(lvl).reshape(-1), a[: a.size // 2])
    h = p.history()
    for w, fn in enumerate(("lbf-lin", "lbf-uin")):
        np.testing.assert_array_equal(h[:, w].reshape(-1), np.fromfile(dout / f"{fn}.0004"))


@pytest.mark.parametrize("name", ["t_noslip", "t_ridges", "t_gr4"])
def test_port_log_rows_match_reference_text_logs(port, ref_configs, tmp_path, name):
    """The per-step log values (force-derived p-grad included) against the text
    logs the reference's own encalc2 / wshearstr append (flowrate.txt,
    density.txt: encalc2.c:135-144; str-up, str-do, w-str, p-grad:
    wshearstr.c:145-166), which print 12 decimals."""
    exe = ref_binary(name)
    if exe is None:
        pytest.skip("compiled reference not available (reference tree not mounted)")
    p = port.Port(ref_configs[name])
    p.init_seeded(42, 0.05, 0.005, 0.0)
    p.set_forcing(True)
    din, dout = tmp_path / "in", tmp_path / "out"
    din.mkdir()
    dout.mkdir()
    p.save(din, 100)
    subprocess.run([str(exe), str(din), "100", str(dout), "-1", "10", "cfr"], check=True, capture_output=True)
    rows = p.step(10)  # force momentum denst flowrate stup stdown stress pgrad
    for fn, col in (("flowrate.txt", 3), ("density.txt", 2), ("str-up.txt", 4), ("str-do.txt", 5),
                    ("w-str.txt", 6), ("p-grad.txt", 7)):
        t = np.loadtxt(dout / fn)
        assert t.shape == (10, 2), fn
        np.testing.assert_allclose(t[:, 1], rows[:, col], rtol=0, atol=5.01e-13, err_msg=fn)
    # the time stamps TM + dt ss with dt = GR / (0.5 (NZs - 2) / CFL)
    _, _, nzs = p.params()
    m = ref_configs[name]
    dt = m["gratio"] * 1.0 / (0.5 * (nzs - 2.0) / m["CFL"])
    np.testing.assert_allclose(t[:, 0], 100 + dt * np.arange(10), rtol=0, atol=5.01e-7)


@pytest.mark.parametrize("name", ["t_noslip", "t_ridges", "t_gr4f"])
def test_port_matches_reference_main(port, ref_configs, tmp_path, name):
    """Pin against the unmodified reference main program (mode -p, ITER = 50,
    one unit time per step): its restart written at step 50, and its
    instantaneous plane statistics file at that step."""
    exe = ref_binary(name, "ref_main")
    if exe is None:
        pytest.skip("compiled reference main not available")
    p = port.Port(ref_configs[name])
    p.init_seeded(42, 0.05, 0.005, 0.0)
    p.set_forcing(True)
    p.save(tmp_path, 100)
    subprocess.run([str(exe), "-p"], cwd=tmp_path, check=True, capture_output=True)
    p.step(50)
    for lvl, fn in enumerate(("lbf-c", "lbf-slf", "lbf-suf")):
        a = np.fromfile(tmp_path / f"{fn}.0150")
        np.testing.assert_array_equal(p.export(lvl).reshape(-1), a[: a.size // 2])
    h = p.history()
    for w, fn in enumerate(("lbf-lin", "lbf-uin")):
        np.testing.assert_array_equal(h[:, w].reshape(-1), np.fromfile(tmp_path / f"{fn}.0150"))
    assert p.force() == np.fromfile(tmp_path / "force.0150")[0]
    st = np.fromfile(tmp_path / "turb-fld.000.150").reshape(9, -1)
    np.testing.assert_array_equal(p.plane_stats(), st)


def test_port_restart_roundtrip(port, ref_configs, tmp_path):
    a = port.Port(ref_configs["t_ridges"])
    a.init_seeded(3, 0.05, 0.005, 0.0)
    a.set_forcing(True)
    a.step(5)
    a.save(tmp_path, 9)
    b = port.Port(ref_configs["t_ridges"])
    b.load(tmp_path, 9)
    b.set_forcing(True)
    a.step(5)
    b.step(5)
    for lvl in range(3):
        np.testing.assert_array_equal(a.export(lvl), b.export(lvl))


def test_laminar_profile_known_answer(port, ref_configs):
    """Laminar known answer of the reference (statistics.c:331-335): a
    constant-flow-rate run from the exact parabola stays on it."""
    m = dict(ref_configs["t_noslip"])
    p = port.Port(m)
    ub = m["ub"]
    p.init_seeded(1, 1.5 * ub, 0.0, 0.0)  # centreline 1.5 ub, no perturbation
    p.set_forcing(True)
    p.step(200)
    st = p.plane_stats()
    nz = st.shape[1]
    _, _, nzs = p.params()
    H = nzs - 2.0
    zdf, zdc, gr = p.zdf, p.zdc, m["gratio"]
    z = np.zeros(nz)
    for k in range(1, zdf):
        z[k] = k - 0.5
    for k in range(2, zdc - 2):
        z[zdf - 2 + k] = gr * (k - 1) + (zdf - 1 - 0.5)
    for k in range(0, zdf - 1):
        z[zdf + zdc - 4 + k] = k + gr * (zdc - 3) + zdf - 1.0 - 0.5
    zeta = z / H
    exact = 6.0 * ub * zeta * (1.0 - zeta)
    used = slice(1, nz - 1)
    assert np.max(np.abs(st[0, used] - exact[used])) < 0.05 * ub


def _moments_seq(f):
    """vel_print's per-node sums, sequential in population order (Python floats are IEEE doubles)."""
    EX = (0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, 1, -1, -1, 0, 0, 0, 0)
    EY = (0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, 1, -1, -1)
    EZ = (0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1)
    ux = uy = uz = d = 0.0
    for a in range(19):
        v = float(f[a])
        ux += EX[a] * v
        uy += EY[a] * v
        uz += EZ[a] * v
        d += v
    if d > 0.0:
        return ux / d, uy / d, uz / d, d
    return 0.0, 0.0, 0.0, 0.0


def test_reference_field_files_layout(ref_configs, tmp_path):
    """The reference's own vel_print (through the harness) writes, per level,
    (nx, ny, nz, 3) velocities and (nx, ny, nz) densities of the post-stream
    state, each node's sums in population order: pins the layout that
    dns_write_fields reproduces."""
    name = "t_ridges"
    exe = ref_binary(name)
    if exe is None:
        pytest.skip("compiled reference not available")
    m = ref_configs[name]
    subprocess.run([str(exe), "-", "0", str(tmp_path), "5", "3", "const", (1e-5).hex(), "0", "1"], check=True,
                   capture_output=True)
    gr = m["gratio"]
    shapes = {"c": (m["xdv"], m["ydv"], m["zdv"]), "slf": (gr * m["xdv"], gr * m["ydv"], m["zds"] + 1),
              "suf": (gr * m["xdv"], gr * m["ydv"], m["zds"] + 1)}
    for lv, (nx, ny, nz) in shapes.items():
        lat = np.fromfile(tmp_path / f"lbf-{lv}.0005", dtype=np.float64)[: nx * ny * nz * 19].reshape(nx, ny, nz, 19)
        vel = np.fromfile(tmp_path / f"vel-{lv}.0005", dtype=np.float64).reshape(nx, ny, nz, 3)
        den = np.fromfile(tmp_path / f"den-{lv}.0005", dtype=np.float64).reshape(nx, ny, nz)
        for i in range(nx):
            for j in range(ny):
                for k in range(nz):
                    ux, uy, uz, d = _moments_seq(lat[i, j, k])
                    assert (vel[i, j, k, 0], vel[i, j, k, 1], vel[i, j, k, 2], den[i, j, k]) == (ux, uy, uz, d), \
                        (lv, i, j, k)


# ------------------------------------------------------------ mode -i start
def _uniform_pair(port, m, tmp_path, seeds=(1, 2)):
    xu, yu, zu, tstr = int(m["xdu"]), int(m["ydu"]), int(m["zdu"]), int(m["TSTR"])
    first = port.uniform_state(xu, yu, zu, seeds[0])
    port.write_uniform_file(tmp_path / f"lbf.{tstr:04d}", first, port.uniform_state(xu, yu, zu, seeds[1]))
    p = port.Port(m)
    p.set_forcing(True)
    p.init_uniform(first)
    return p, tstr


@pytest.mark.parametrize("name", ["t_noslip", "t_ridges"])
def test_port_uniform_start_matches_reference_main(port, ref_configs, tmp_path, name):
    """Mode -i of the unmodified reference main (initializer + inter_init), its
    restart written at the first iteration: the three post-stream lattices,
    the f^neq history and the force are bit-identical.  Two slips of
    inter_init are pinned as what they are: the reference's lower history
    carries the upper plane's density and velocity (its upper one keeps
    zeros), and its levels p and pp hold level n only where the flat index of
    the halo-padded array is below the 19-field extent it copies."""
    exe = ref_binary(name, "ref_main")
    if exe is None:
        pytest.skip("compiled reference main not available")
    m = ref_configs[name]
    p, tstr = _uniform_pair(port, m, tmp_path)
    subprocess.run([str(exe), "-i"], cwd=tmp_path, check=True, capture_output=True)
    for lvl, fn in enumerate(("lbf-c", "lbf-slf", "lbf-suf")):
        a = np.fromfile(tmp_path / f"{fn}.{tstr:04d}")
        np.testing.assert_array_equal(p.export(lvl).reshape(-1), a[: a.size // 2])
    assert p.force() == np.fromfile(tmp_path / f"force.{tstr:04d}")[0]
    h = p.history()
    nx, ny = p.nx, p.ny
    lin = np.fromfile(tmp_path / f"lbf-lin.{tstr:04d}").reshape(3, nx, ny, 23)
    uin = np.fromfile(tmp_path / f"lbf-uin.{tstr:04d}").reshape(3, nx, ny, 23)
    np.testing.assert_array_equal(h[0, 0, ..., 4:], lin[0, ..., 4:])
    np.testing.assert_array_equal(h[0, 1, ..., 4:], uin[0, ..., 4:])
    np.testing.assert_array_equal(h[0, 1, ..., :4], lin[0, ..., :4])
    assert not uin[0, ..., :4].any()
    # the restatement: p = pp = n in full
    np.testing.assert_array_equal(h[1], h[0])
    np.testing.assert_array_equal(h[2], h[0])
    # the reference: inter_init.c:237-248 copies element q < 19 (xdc+5)(ydc+5)
    # of the padded [xdc+5][ydc+5][23] array, xdc = xdv + 1, ydc = ydv + 1
    i, j, b = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(23), indexing="ij")
    q = (i + 2) * (ny + 6) * 23 + (j + 2) * 23 + b
    copied = q < 19 * (nx + 6) * (ny + 6)
    for ref in (lin, uin):
        for lvl in (1, 2):
            np.testing.assert_array_equal(ref[lvl], np.where(copied, ref[0], 0.0))


@pytest.mark.parametrize("case", UNIFORM_GOLDEN, ids=lambda c: c["config"])
def test_port_uniform_start_golden(port, ref_configs, tmp_path, case):
    """The restatement's mode -i start against digests of the reference main's."""
    m = ref_configs[case["config"]]
    assert [int(m["xdu"]), int(m["ydu"]), int(m["zdu"])] == case["uniform"]
    p, _ = _uniform_pair(port, m, tmp_path, case["seeds"])
    for lvl, fn in enumerate(("lbf-c", "lbf-slf", "lbf-suf")):
        assert _digest(p.export(lvl)) == case[fn]["sha256"], fn
    h = p.history()
    assert _digest(h[0, 0, ..., 4:]) == case["lin_fneq_n"]
    assert _digest(h[0, 1, ..., 4:]) == case["uin_fneq_n"]
    assert _digest(h[0, 1, ..., :4]) == case["upper_moments_n"]
    assert p.force() == case["force"]


def test_port_uniform_start_rejects_short_grid(port, ref_configs):
    """A uniform grid too short for the channel, whose stencils would leave
    the reference's periodic halo in x or y, is refused."""
    m = ref_configs["t_ridges"]
    p = port.Port(m)
    with pytest.raises(ValueError):
        p.init_uniform(port.uniform_state(4, 12, 11, 1))
    with pytest.raises(ValueError):
        p.init_uniform(port.uniform_state(12, 4, 11, 1))
    p.init_uniform(port.uniform_state(12, 12, 5, 1))   # a coarser wall-normal grid is fine


# ------------------------------------------------------------ budget program
TKE_GOLDEN = json.loads((ROOT / "tests" / "golden" / "tke_golden.json").read_text())


@pytest.mark.parametrize("case", TKE_GOLDEN, ids=lambda c: c["config"])
def test_reference_budget_program_reproduces_golden(case):
    """The compiled reference budget program (TKE-budget/computations under the
    single-rank shim) reproduces its stored output bit for bit."""
    if ref_binary(case["config"], "tke_budget") is None or ref_binary(case["config"]) is None:
        pytest.skip("compiled reference not available")
    import sys

    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    import make_golden

    again = make_golden.run_tke_case(case["config"], case["steps"])
    assert np.array_equal(np.array(again["profiles"]), np.array(case["profiles"]))
