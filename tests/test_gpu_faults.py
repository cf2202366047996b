"""Faults injected on the host (needs a B200; nothing here faults the GPU).

Restart files that are truncated, missing or written for a smaller grid are
refused before anything is imported, so the channel keeps its state.  A NaN
planted in one batched instance's state retires that instance with DNS_ENAN
while the instances sharing its kernels run on bit-identically to a batch
without it.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import gpu_available
from test_gpu_parity import params_for

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="no CUDA device")]

SEED, UC, AMP = 42, 0.05, 0.005


def snapshot(ch):
    return [ch.export_state(lvl) for lvl in range(3)] + [ch.export_history()]


def assert_same(a, b):
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def _channel(pkg, m, seed):
    ch = pkg.Channel(params_for(pkg, m, "cfr"))
    ch.init_seeded(seed, UC, AMP)
    return ch


@pytest.mark.parametrize("victim", ["lbf-slf", "lbf-uin", "force"])
def test_truncated_restart_is_refused_and_state_kept(pkg, ref_configs, tmp_path, victim):
    m = ref_configs["t_odd"]
    a = _channel(pkg, m, 1)
    a.step(3)
    a.write_restart(tmp_path, 9)
    b = _channel(pkg, m, 2)
    b.step(2)
    before = snapshot(b)
    fn = tmp_path / f"{victim}.0009"
    whole = fn.read_bytes()
    fn.write_bytes(whole[: len(whole) // 2 // 8 * 8])
    with pytest.raises(pkg.DnsError) as e:
        b.load_restart(tmp_path, 9)
    assert e.value.code == pkg.DNS_EIO and "truncated" in str(e.value)
    assert_same(snapshot(b), before)
    os.remove(fn)
    with pytest.raises(pkg.DnsError) as e:
        b.load_restart(tmp_path, 9)
    assert e.value.code == pkg.DNS_EIO
    assert_same(snapshot(b), before)
    # the intact files load, and the run resumes where the writer left off
    fn.write_bytes(whole)
    b.load_restart(tmp_path, 9)
    assert_same(snapshot(b), snapshot(a))
    a.step(2)
    b.step(2)
    assert_same(snapshot(b), snapshot(a))
    a.close()
    b.close()


def test_restart_of_a_smaller_grid_is_refused(pkg, ref_configs, tmp_path):
    small, big = ref_configs["t_odd"], ref_configs["c1"]
    gs = pkg.geometry(params_for(pkg, small, "cfr"))
    gb = pkg.geometry(params_for(pkg, big, "cfr"))
    assert gs.nx * gs.ny * gs.nzc < gb.nx * gb.ny * gb.nzc
    a = _channel(pkg, small, 1)
    a.write_restart(tmp_path, 4)
    b = _channel(pkg, big, 2)
    before = snapshot(b)
    with pytest.raises(pkg.DnsError) as e:
        b.load_restart(tmp_path, 4)
    assert e.value.code == pkg.DNS_EIO
    assert_same(snapshot(b), before)
    a.close()
    b.close()


def test_nan_instance_retires_while_others_run_on_bit_identically(pkg, ref_configs):
    cases = [("t_ridges", "cfr", 3), ("t_odd", "cfr", 4), ("t_noslip", "const", 5)]
    steps = 24
    with pkg.Batch() as b, pkg.Batch() as clean:
        ids, ref = [], []
        for name, mode, seed in cases:
            p = params_for(pkg, ref_configs[name], mode)
            ids.append(b.add(p, steps=steps, seed=seed, uc=UC, amp=AMP, sample_every=4))
            if name != "t_odd":
                ref.append(clean.add(p, steps=steps, seed=seed, uc=UC, amp=AMP, sample_every=4))
        bad = ids[1]
        s = b.export_state(bad, 1)
        s[2, 3, 2, 5] = np.nan  # a lower-block population next to the wall
        b.import_state(bad, 1, s)
        for _ in range(steps // 4):  # one step group per run(4): the stop lands at a group boundary
            b.run(4)
            clean.run(4)
        inf = b.info(bad)
        assert inf.status == pkg.DNS_ENAN and inf.remaining == 0 and 0 < inf.steps_done < steps
        assert not np.isfinite(b.log(bad)[-1, 7])
        for i, j in zip([ids[0], ids[2]], ref):
            assert b.info(i).status == 0 and b.info(i).steps_done == steps
            for lvl in range(3):
                np.testing.assert_array_equal(b.export_state(i, lvl), clean.export_state(j, lvl))
            np.testing.assert_array_equal(b.log(i), clean.log(j))
            np.testing.assert_array_equal(b.stats(i)[0], clean.stats(j)[0])
        # the failed instance's memory goes back; the batch keeps serving
        b.remove(bad)
        k = b.add(params_for(pkg, ref_configs["t_odd"], "cfr"), steps=4, seed=4, uc=UC, amp=AMP)
        b.run(4)
        assert b.info(k).status == 0 and b.info(k).steps_done == 4
