"""CUDA path against the oracle (needs a B200).

Constant-force runs must be bit-identical to the oracle (the per-node FP64
arithmetic follows the reference's operation order with no fused
multiply-add).  Constant-flow-rate runs differ only through the association of
the whole-domain momentum sum, so they are held to 1e-12 relative in every
population, the tolerance the solver is specified to.
"""
from __future__ import annotations

import hashlib
import json

import numpy as np
import pytest

from conftest import ROOT, gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]

RTOL_CFR = 1e-12
GCONST = 1.0e-5


def params_for(pkg, m, mode, g=GCONST):
    return pkg.make_params(
        xdv=m["xdv"], ydv=m["ydv"], zdv=m["zdv"], zds=m["zds"], gratio=m["gratio"], Rebs=float(m["Rebs"]),
        ub=m["ub"], CFL=m["CFL"], TSTR=m["TSTR"], pattern=m.get("pattern"), gyplussize=m["gyplussize"],
        wyplussize=m["wyplussize"], gxplussize=m["gxplussize"], wxplussize=m["wxplussize"],
        forcing=pkg.FORCING_CFR if mode == "cfr" else pkg.FORCING_CONST, force_const=g if mode == "const" else 0.0,
        fltr=1 if m.get("fltr") else 0)


def pair(pkg, port, m, mode, g=GCONST, seed=42, uc=0.05, amp=0.005):
    ch = pkg.Channel(params_for(pkg, m, mode, g))
    ch.init_seeded(seed, uc, amp)
    p = port.Port(m)
    p.init_seeded(seed, uc, amp, g if mode == "const" else 0.0)
    p.set_forcing(mode == "cfr", g if mode == "const" else 0.0)
    return ch, p


def assert_state(ch, p, exact, rtol=RTOL_CFR):
    for lvl in range(3):
        a, b = ch.export_state(lvl), p.export(lvl)
        if exact:
            np.testing.assert_array_equal(a, b, err_msg=f"level {lvl}")
        else:
            np.testing.assert_allclose(a, b, rtol=rtol, atol=0, err_msg=f"level {lvl}")
    ha, hb = ch.export_history(), p.history()
    if exact:
        np.testing.assert_array_equal(ha, hb)
    else:
        # history fields are rho, u and fneq = f - feq: differences of O(0.05)
        # populations, so their error is absolute at the populations' scale
        np.testing.assert_allclose(ha, hb, rtol=rtol, atol=1e-14)


CASES = [("t_noslip", "const"), ("t_noslip", "cfr"), ("t_ridges", "cfr"), ("t_posts", "const"),
         ("t_posts", "cfr"), ("t_span", "cfr"), ("t_gr4", "const"), ("t_gr4", "cfr"), ("t_gr4f", "const"),
         ("t_gr4f", "cfr"), ("t_odd", "const"), ("t_odd", "cfr")]


@pytest.mark.parametrize("name", ["t_noslip", "t_gr4", "t_odd", "c1"])
def test_seeded_state_is_bit_identical(pkg, port, ref_configs, name):
    ch, p = pair(pkg, port, ref_configs[name], "cfr")
    assert_state(ch, p, exact=True)
    # the force is a whole-domain sum: association differs from the reference loop
    np.testing.assert_allclose(ch.force(), p.force(), rtol=1e-13, atol=0)


@pytest.mark.parametrize("name,mode", CASES, ids=lambda x: str(x))
def test_steps_match_oracle(pkg, port, ref_configs, name, mode):
    ch, p = pair(pkg, port, ref_configs[name], mode)
    n = 20
    la = ch.step(n)
    lb = p.step(n)
    assert_state(ch, p, exact=(mode == "const"))
    # log rows: force, momentum, denst, flowrate (oracle columns 0..3)
    np.testing.assert_allclose(la[:, 1:5], lb[:, 0:4], rtol=1e-11, atol=1e-15)
    np.testing.assert_allclose(la[:, 5:8], lb[:, 4:7], rtol=1e-9, atol=1e-14)  # wall shear (plane-sum order)
    np.testing.assert_allclose(ch.force(), p.force(), rtol=1e-9, atol=1e-16)


def c1_force(pkg, m):
    """Body force for Re_tau = 180 on the half height: g_c = GR u_tau^2 / h_f."""
    g = pkg.geometry(params_for(pkg, m, "cfr"))
    nu_f = (1.0 / g.omega_f - 0.5) / 3.0
    h_f = (g.nzs - 2) / 2.0
    u_tau = 180.0 * nu_f / h_f
    return g.gr * u_tau * u_tau / h_f


@pytest.mark.parametrize("mode", ["const", "cfr"])
def test_config1_100_steps(pkg, port, ref_configs, mode):
    """Plain FP64 channel 64 x 32 x 64 (coarse) with 2:1 near-wall blocks,
    100 coarse steps from the seeded state: every population within 1e-12
    (bit-identical with the constant body force)."""
    m = ref_configs["c1"]
    g = c1_force(pkg, m)
    ch, p = pair(pkg, port, m, mode, g=g)
    ch.step(100)
    p.step(100)
    assert_state(ch, p, exact=(mode == "const"))


C1_LONG_FILE = ROOT / "tests" / "golden" / "c1_1000_golden.json"
C1_LONG = json.loads(C1_LONG_FILE.read_text()) if C1_LONG_FILE.exists() else []


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


@pytest.mark.parametrize("case", C1_LONG, ids=lambda c: c["mode"])
def test_config1_1000_steps_against_reference(pkg, ref_configs, case):
    """The plain FP64 channel c1 for its stated 1000 coarse steps against the
    reference's own routines (golden data made by tests/golden/make_golden.py
    --c1-long from the compiled reference).  Constant body force (Re_tau =
    180): the lattices and interface histories bit for bit.  Constant flow
    rate: per-population plane sums of every lattice within 1e-12 and the
    logged flow rate within 1e-11 (the whole-domain flow-rate sum is
    associated differently from the reference's loop)."""
    m = ref_configs["c1"]
    ch = pkg.Channel(params_for(pkg, m, case["mode"], g=case["g"]))
    ch.init_seeded(case["seed"], case["uc"], case["amp"])
    log = ch.step(case["steps"])
    for lvl, fn in enumerate(("lbf-c", "lbf-slf", "lbf-suf")):
        s = ch.export_state(lvl)
        if case["mode"] == "const":
            assert _digest(s) == case[fn]["sha256"], fn
        np.testing.assert_allclose(s.sum(axis=(0, 1)), np.array(case[fn]["plane_sums"]), rtol=1e-12, atol=1e-12,
                                   err_msg=fn)
    if case["mode"] == "const":
        h = ch.export_history()
        assert _digest(h[:, 0]) == case["lbf-lin"]["sha256"]
        assert _digest(h[:, 1]) == case["lbf-uin"]["sha256"]
    # the harness logs one more row, the flow rate of the state it writes
    np.testing.assert_allclose(log[:, 4], case["flowrate_log"][:case["steps"]], rtol=1e-11, atol=0)
    np.testing.assert_allclose(ch.force(), case["force_next"], rtol=1e-9, atol=1e-16)


def test_restart_roundtrip(pkg, port, ref_configs, tmp_path):
    m = ref_configs["t_ridges"]
    a, p = pair(pkg, port, m, "cfr")
    a.step(5)
    a.write_restart(tmp_path, 7)
    # the files are the reference layout: the oracle reads them
    q = port.Port(m)
    q.load(tmp_path, 7)
    q.set_forcing(True)
    p.step(5)
    for lvl in range(3):
        np.testing.assert_allclose(q.export(lvl), p.export(lvl), rtol=RTOL_CFR, atol=0)
    b = pkg.Channel(params_for(pkg, m, "cfr"))
    b.load_restart(tmp_path, 7)
    a.step(4)
    b.step(4)
    for lvl in range(3):
        np.testing.assert_array_equal(a.export_state(lvl), b.export_state(lvl))


def test_plane_stats_match_reference_definition(pkg, port, ref_configs):
    ch, p = pair(pkg, port, ref_configs["t_posts"], "const")
    ch.step(7)
    p.step(7)
    np.testing.assert_array_equal(ch.plane_stats(), p.plane_stats())


def _sampled_vs_two_pass(pkg, port, m, uc, amp, steps, every, rtol_mean, rtol_var):
    """The device's sampled statistics against the time mean of the oracle's
    per-sample plane records (statistics.c: plane means, then two-pass rms and
    <u'w'> about them)."""
    ch, p = pair(pkg, port, m, "cfr", uc=uc, amp=amp)
    ch.set_sampling(every)
    snaps = []
    for s in range(steps):
        if s % every == 0:
            snaps.append(p.plane_stats())
        p.step(1)
    ch.step(steps)
    st, ns = ch.stats()
    assert ns == len(snaps)
    ref = np.mean(snaps, axis=0)  # time mean of the per-sample plane records
    used = slice(1, st.shape[1] - 1)
    for name, row, col in (("U", 1, 0), ("V", 2, 1), ("W", 3, 2), ("rho", 4, 7)):
        np.testing.assert_allclose(st[row, used], ref[col, used], rtol=rtol_mean, atol=1e-15, err_msg=name)
    # per-sample variances: per-thread Welford moments merged pairwise (Chan)
    # against the reference's two-pass definition
    sq = np.mean(np.square(snaps), axis=0)
    for name, row, col in (("uu", 5, 3), ("vv", 6, 4), ("ww", 7, 5)):
        np.testing.assert_allclose(st[row, used], sq[col, used], rtol=rtol_var, atol=0, err_msg=name)
    scale = np.max(np.abs(ref[6, used]))
    np.testing.assert_allclose(st[8, used], ref[6, used], rtol=0, atol=rtol_var * scale, err_msg="uw")


def test_sampled_statistics(pkg, port, ref_configs):
    _sampled_vs_two_pass(pkg, port, ref_configs["t_odd"], 0.05, 0.005, steps=6, every=2, rtol_mean=1e-11,
                         rtol_var=1e-10)


def test_sampled_variance_survives_cancellation(pkg, port, ref_configs):
    """Perturbations of 1e-6 on a mean flow of 0.1 that the flow-rate forcing
    accelerates by ~1e-2 a step: the plane variances are ~1e-13 against squared
    means of ~1e-2, so E[x^2] - E[x]^2 would keep only ~5 significant digits
    (and sums about any fixed reference value fare no better while the mean
    moves); Welford moments merged pairwise keep the two-pass result to 1e-9."""
    _sampled_vs_two_pass(pkg, port, ref_configs["t_odd"], 0.1, 1e-6, steps=4, every=1, rtol_mean=1e-11,
                         rtol_var=1e-9)


def test_non_finite_state_is_reported(pkg, port, ref_configs):
    """Fault injected on the host: a NaN population makes the step report
    DNS_ENAN (the reference aborts on a NaN wall shear stress)."""
    m = ref_configs["t_noslip"]
    ch, _ = pair(pkg, port, m, "cfr")
    s = ch.export_state(1)
    s[3, 3, 2, 5] = np.nan
    ch.import_state(1, s)
    with pytest.raises(pkg.DnsError) as e:
        ch.step(3)
    assert e.value.code == pkg.DNS_ENAN
