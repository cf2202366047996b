"""The four-node stream-collide kernels' x-direction stores, restated on the CPU.

A thread of ``quad_f32.cuh`` owns four consecutive nodes of a row and stores
each population's four post-collision values with one 16-byte store.  A push
along +x or -x shifts the group by one node, so the thread's aligned store
takes one value from its neighbour lane (a warp shuffle) and the value that
leaves the group at a warp, block or row edge is stored singly by the thread
it leaves.  These tests replay ``quad_pos`` and ``quad_store`` for every block
geometry the library launches and check that every destination node of a row
is written exactly once, with the value of the node the push came from, and
that no store falls outside the row:

* the batched engine: tiles of W threads (W = 8 .. 128) along a row, a row
  segment of 4 W nodes per tile;
* the single-channel FP32 form: blocks of 32 x jb threads, 32 along a row of
  128 nodes.
"""
from __future__ import annotations

import pytest


def quad_pos(tx, lane, W, gx0, nx, row_ok=True):
    """(x0, ok, has_left, has_right) as quad_f32.cuh computes them."""
    x0 = gx0 + 4 * tx
    ok = row_ok and x0 < nx
    has_left = tx > 0 and lane > 0
    has_right = tx < W - 1 and lane < 31 and x0 + 4 < nx
    return x0, ok, has_left, has_right


def row_stores(nx, W, segments, lane_of):
    """Every (destination, source node) store of one row for e_x = +1 and -1."""
    out = {+1: [], -1: []}
    threads = []
    for gx0 in segments:
        for tx in range(W):
            threads.append((gx0, tx) + quad_pos(tx, lane_of(tx), W, gx0, nx))
    by_x0 = {t[2]: t for t in threads if t[3]}  # valid threads by first node
    for gx0, tx, x0, ok, hl, hr in threads:
        if not ok:
            continue
        v = [x0, x0 + 1, x0 + 2, x0 + 3]  # the source node of each held value
        # +x: the aligned group x0..x0+3 takes the left lane's last value
        if hl:
            left = by_x0[x0 - 4]
            assert left[0] == gx0 and left[1] == tx - 1, "left group belongs to the neighbour lane"
            out[+1] += [(x0, x0 - 1), (x0 + 1, v[0]), (x0 + 2, v[1]), (x0 + 3, v[2])]
        else:
            out[+1] += [(x0 + 1, v[0]), (x0 + 2, v[1]), (x0 + 3, v[2])]
        if not hr:
            out[+1].append((0 if x0 + 4 == nx else x0 + 4, v[3]))
        # -x: the aligned group takes the right lane's first value
        if hr:
            right = by_x0[x0 + 4]
            assert right[0] == gx0 and right[1] == tx + 1, "right group belongs to the neighbour lane"
            out[-1] += [(x0, v[1]), (x0 + 1, v[2]), (x0 + 2, v[3]), (x0 + 3, x0 + 4)]
        else:
            out[-1] += [(x0, v[1]), (x0 + 1, v[2]), (x0 + 2, v[3])]
        if not hl:
            out[-1].append((nx - 1 if x0 == 0 else x0 - 1, v[0]))
    return out


def check_row(nx, W, segments, lane_of):
    stores = row_stores(nx, W, segments, lane_of)
    for ex, lst in stores.items():
        dests = [d for d, _ in lst]
        assert all(0 <= d < nx for d in dests), (ex, nx, W)
        assert sorted(dests) == list(range(nx)), f"e_x {ex}: each node written once (nx {nx}, W {W})"
        for d, src in lst:
            assert d == (src + ex) % nx, f"e_x {ex}: node {d} got the value of node {src}"


@pytest.mark.parametrize("W", [8, 16, 32, 64, 128])
def test_batched_tiles_write_every_node_once(W):
    """Batched engine: row segments of 4 W nodes, lane = tx mod 32 (a tile of
    W > 32 threads spans several warps), every x extent that is a multiple of
    4 up to 1024 (a tile wider than the row leaves threads idle)."""
    for nx in range(4, 1028, 4):
        check_row(nx, W, list(range(0, nx, 4 * W)), lane_of=lambda tx: tx % 32)


def test_single_channel_blocks_write_every_node_once():
    """Single-channel FP32 form: blocks of 32 threads along a row of 128 nodes,
    every x extent that is a multiple of 4 up to 1024 (the last block of a row
    may be partly idle)."""
    for nx in range(4, 1028, 4):
        check_row(nx, 32, list(range(0, nx, 128)), lane_of=lambda tx: tx)


def test_idle_threads_store_nothing():
    """A thread whose group starts at or past the row's end stores nothing and
    is not relied on by its left neighbour."""
    nx, W = 200, 32
    for gx0 in range(0, nx, 128):
        for tx in range(W):
            x0, ok, hl, hr = quad_pos(tx, tx, W, gx0, nx)
            if x0 + 4 >= nx:
                assert not hr
            if x0 >= nx:
                assert not ok
