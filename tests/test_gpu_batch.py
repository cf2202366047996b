"""Batched FP32 engine (needs a B200).

Each instance of a batch is held to the FP32 form's bar against the FP64
oracle (populations within 2e-6 after tens of steps, logged flow values within
1e-5 relative), and to batching invariance: an instance's state and log are
bit-identical whether it runs alone or among other instances of different
sizes, patterns, forcing and budgets, joining and leaving at any time.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import gpu_available
from test_gpu_parity import GCONST, params_for

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]

SEED, UC, AMP = 42, 0.05, 0.005


def oracle(port, m, mode, g=GCONST):
    o = port.Port(m)
    o.init_seeded(SEED, UC, AMP, g if mode == "const" else 0.0)
    o.set_forcing(mode == "cfr", g if mode == "const" else 0.0)
    return o


def states(b, i):
    return [b.export_state(i, lvl) for lvl in range(3)]


@pytest.mark.parametrize("name,mode", [("t_noslip", "const"), ("t_ridges", "cfr"), ("t_posts", "cfr"),
                                       ("t_span", "const"), ("t_gr4", "cfr"), ("t_gr4f", "cfr"), ("t_odd", "cfr")])
def test_batch_instance_tracks_fp64_oracle(pkg, port, ref_configs, name, mode):
    m = ref_configs[name]
    with pkg.Batch() as b:
        i = b.add(params_for(pkg, m, mode), steps=30, seed=SEED, uc=UC, amp=AMP)
        assert b.run(30) == 0
        o = oracle(port, m, mode)
        lb = o.step(30)
        dev = max(np.max(np.abs(b.export_state(i, lvl) - o.export(lvl))) for lvl in range(3))
        assert dev < 2e-6, dev
        la = b.log(i)
        assert la.shape == (30, 9)
        np.testing.assert_allclose(la[:, 2:5], lb[:, 1:4], rtol=1e-5, atol=1e-8)
        inf = b.info(i)
        assert inf.steps_done == 30 and inf.remaining == 0 and inf.status == 0


def test_batch_matches_single_fp32_channel(pkg, ref_configs):
    """The batch and the single-channel FP32 form compute the same deviation
    arithmetic with different kernels (the batch moves four nodes per thread
    and sums its flow-rate partials per node group): they agree to FP32
    rounding, states within 5e-7 and the logged quantities within 1e-5 (the
    wall shear stresses, differences of near-wall velocities, within 1e-3)."""
    m = ref_configs["t_ridges"]
    p = params_for(pkg, m, "cfr")
    q = params_for(pkg, m, "cfr")
    q.precision = pkg.FP32
    ch = pkg.Channel(q)
    ch.init_seeded(SEED, UC, AMP)
    ch.set_sampling(2)
    la = ch.step(20)
    with pkg.Batch() as b:
        i = b.add(p, steps=20, seed=SEED, uc=UC, amp=AMP, sample_every=2, tile=(128, 2, 128, 2))
        b.run(20)
        for lvl in range(3):
            np.testing.assert_allclose(b.export_state(i, lvl), ch.export_state(lvl), rtol=0, atol=5e-7)
        lb = b.log(i)
        np.testing.assert_allclose(lb[:, 1:5], la[:, 1:5], rtol=1e-5, atol=1e-9)
        np.testing.assert_allclose(lb[:, 5:], la[:, 5:], rtol=1e-3, atol=1e-8)
        sa, na = b.stats(i)
        sb, nb = ch.stats()
        assert na == nb == 10
        np.testing.assert_allclose(sa, sb, rtol=1e-5, atol=1e-9)
    ch.close()


def test_batch_mix_invariance(pkg, ref_configs):
    """Instance A alone == A among others (bit for bit), whatever joins,
    leaves or runs out of budget around it."""
    pa = params_for(pkg, ref_configs["t_ridges"], "cfr")
    pb = params_for(pkg, ref_configs["t_posts"], "cfr")
    pc = params_for(pkg, ref_configs["t_noslip"], "const")
    pd = params_for(pkg, ref_configs["t_odd"], "cfr")
    with pkg.Batch() as solo:
        a = solo.add(pa, steps=12, seed=7, sample_every=3)
        solo.run(40)
        ref_state, ref_log, ref_stats = states(solo, a), solo.log(a), solo.stats(a)[0]
    with pkg.Batch() as mix:
        b = mix.add(pb, steps=5, seed=3, sample_every=1)
        c = mix.add(pc, steps=100, seed=9)
        mix.run(3)                                     # A joins two steps late
        a = mix.add(pa, steps=12, seed=7, sample_every=3)
        d = mix.add(pd, steps=4, seed=11, tile=(32, 1, 32, 4))
        assert mix.run(7) == 2                         # b and d are spent
        mix.remove(b)
        e = mix.add(pb, steps=30, seed=5)              # reuses b's slot
        mix.run(10)
        assert mix.info(a).steps_done == 12 and mix.info(a).remaining == 0
        assert mix.info(d).steps_done == 4
        assert mix.info(c).steps_done == 20
        assert mix.info(e).steps_done == 10
        for x, y in zip(states(mix, a), ref_state):
            assert np.array_equal(x, y)
        assert np.array_equal(mix.log(a), ref_log)
        assert np.array_equal(mix.stats(a)[0], ref_stats)
        # a second copy of A admitted late reproduces A again
        a2 = mix.add(pa, steps=12, seed=7, sample_every=3)
        mix.run(12)
        for x, y in zip(states(mix, a2), ref_state):
            assert np.array_equal(x, y)


def test_batch_rejects_mixed_gratio_and_bad_tiles(pkg, ref_configs):
    with pkg.Batch() as b:
        b.add(params_for(pkg, ref_configs["t_noslip"], "cfr"), steps=1)
        with pytest.raises(pkg.DnsError) as e:
            b.add(params_for(pkg, ref_configs["t_gr4"], "cfr"), steps=1)
        assert e.value.code == pkg.DNS_EINVAL
        with pytest.raises(pkg.DnsError):
            b.add(params_for(pkg, ref_configs["t_noslip"], "cfr"), steps=1, tile=(48, 2, 128, 2))


def test_batch_autotune_sets_table(pkg, ref_configs):
    p = params_for(pkg, ref_configs["c1"], "cfr")
    with pkg.Batch() as b:
        tile, ms = b.autotune(p, steps=3)
        assert ms > 0
        assert b.tile_for(p).as_tuple() == tile
        i = b.add(p, steps=2)
        assert b.info(i).tile.as_tuple() == tile
        b.run(2)
        assert b.info(i).steps_done == 2


def test_batch_config4_shapes_track_fp64_channel(pkg):
    """Shapes of the batched workload (Nx in {64..256}, span in {64..128},
    Ny in {32, 48, 64} with Ny/8 coarse cells embedded per wall, ridges or
    posts): each batched FP32 instance within 1e-5 of the FP64 channel after
    20 steps."""
    shapes = [dict(xdv=64, ydv=64, Ny=32, pattern="RSLIP", pitch=16, g=10),
              dict(xdv=192, ydv=96, Ny=48, pattern="PSLIP", pitch=24, g=12),
              dict(xdv=128, ydv=128, Ny=64, pattern="RSLIP", pitch=32, g=24)]
    with pkg.Batch() as b:
        ids, chans = [], []
        for s in shapes:
            zds = 2 * s["Ny"] // 8
            kw = dict(xdv=s["xdv"], ydv=s["ydv"], zdv=s["Ny"] - zds + 3, zds=zds, gratio=2, Rebs=3000.0,
                      ub=0.0866034, CFL=0.1, pattern=s["pattern"], forcing=pkg.FORCING_CFR)
            if s["pattern"] == "RSLIP":
                kw.update(gyplussize=s["g"], wyplussize=s["pitch"] - s["g"])
            else:
                kw.update(gxplussize=s["g"], wxplussize=s["pitch"] - s["g"], gyplussize=s["g"],
                          wyplussize=s["pitch"] - s["g"])
            p = pkg.make_params(**kw)
            ids.append(b.add(p, steps=20, seed=SEED))
            ch = pkg.Channel(p)
            ch.init_seeded(SEED, UC, AMP)
            ch.step(20)
            chans.append(ch)
        b.run(20)
        for i, ch in zip(ids, chans):
            for lvl in range(3):
                assert np.max(np.abs(b.export_state(i, lvl) - ch.export_state(lvl))) < 1e-5
            ch.close()
