"""The CPU oracle: pinned against the reference's own known-answer checks for the
scan / compaction / tile-list layer, and the three solvers (BK exact max-flow, the
restated reference schedule ref_tiled, a brute-force augmenting-path solver) agree."""
import collections

import numpy as np
import pytest

import synth
import strokes


def test_prefix_sum_reference_check(oracle):
    """test_PrefixSum.py:15-35: 65536 random ints in [0,20); total == sum."""
    h = np.random.default_rng(0).integers(0, 20, 65536).astype(np.int32)
    scan, total = oracle.exclusive_scan(h)
    assert total == h.sum()
    assert scan[0] == 0 and np.array_equal(scan[1:], np.cumsum(h)[:-1])


def test_stream_compact_reference_check(oracle):
    """test_StreamCompact.py:26-41: 65536 random 0/1 flags; list == np.where(flags == 1)."""
    f = np.random.default_rng(1).integers(0, 2, 65536).astype(np.int32)
    ids, n = oracle.compact(f)
    assert np.array_equal(np.where(f == 1)[0], ids[:n])


def test_tile_list_reference_check(oracle):
    """test_IncrementalTileList.py:18-40: 4096^2 / 16^2 tiles, stamps in [0,20),
    build(GTE, 10) == row-major ids of np.where(tiles >= 10)."""
    dim = (256, 256)
    h = np.random.default_rng(2).integers(0, 20, (dim[1], dim[0])).astype(np.int32)
    ids, n = oracle.compact(oracle.flag(h.reshape(-1), oracle.OPERATOR_GTE, 10))
    ys, xs = np.where(h >= 10)
    assert np.array_equal(ys * dim[0] + xs, ids[:n])


def _edmonds_karp(g):
    H, W = g.excess.shape
    N = W * H
    s, t = N, N + 1
    cap = collections.defaultdict(int)
    adj = collections.defaultdict(set)

    def add(u, v, c):
        cap[(u, v)] += c
        adj[u].add(v)
        adj[v].add(u)
    for y in range(H):
        for x in range(W):
            i = y * W + x
            e = int(g.excess[y, x])
            if e > 0:
                add(s, i, e)
            elif e < 0:
                add(i, t, -e)
            if y > 0: add(i, i - W, int(g.up[y, x]))
            if y < H - 1: add(i, i + W, int(g.down[y, x]))
            if x > 0: add(i, i - 1, int(g.left[y, x]))
            if x < W - 1: add(i, i + 1, int(g.right[y, x]))
    flow = 0
    while True:
        par = {s: None}
        q = collections.deque([s])
        while q and t not in par:
            u = q.popleft()
            for v in adj[u]:
                if v not in par and cap[(u, v)] > 0:
                    par[v] = u
                    q.append(v)
        if t not in par:
            break
        f, v = 1 << 60, t
        while par[v] is not None:
            f = min(f, cap[(par[v], v)])
            v = par[v]
        v = t
        while par[v] is not None:
            cap[(par[v], v)] -= f
            cap[(v, par[v])] += f
            v = par[v]
        flow += f
    seen = {s}
    q = collections.deque([s])
    while q:
        u = q.popleft()
        for v in adj[u]:
            if v not in seen and cap[(u, v)] > 0:
                seen.add(v)
                q.append(v)
    lab = np.zeros((H, W), np.uint8)
    for i in seen:
        if i < N:
            lab[i // W, i % W] = 1
    return flow, lab


@pytest.mark.parametrize("seed", range(40))
def test_bk_matches_brute_force(oracle, seed):
    H, W = [(4, 4), (5, 7), (8, 8), (3, 9), (6, 6)][seed % 5]
    g = synth.random_graph(W, H, seed, cap_max=9, tlink_max=20, sparsity=0.3,
                           symmetric=bool(seed % 2))
    f1, l1 = oracle.maxflow_bk(*g.planes())
    f2, l2 = _edmonds_karp(g)
    assert f1 == f2 and np.array_equal(l1, l2)


@pytest.mark.parametrize("w,h,seed", [(64, 64, 0), (96, 64, 1), (256, 256, 3), (512, 512, 0)])
def test_ref_tiled_matches_bk_synthetic(oracle, w, h, seed):
    g = synth.make_graph(w, h, seed)
    f1, l1 = oracle.maxflow_bk(*g.planes())
    f2, l2, st = oracle.ref_tiled(*g.planes())
    assert f1 == f2 and np.array_equal(l1, l2)
    assert oracle.cut_capacity(*g.planes(), l1) == f1


@pytest.mark.parametrize("seed,sym", [(0, True), (1, False), (2, True)])
def test_ref_tiled_matches_bk_random(oracle, seed, sym):
    g = synth.random_graph(256, 192, seed, cap_max=100, tlink_max=150, symmetric=sym)
    f1, l1 = oracle.maxflow_bk(*g.planes())
    f2, l2, st = oracle.ref_tiled(*g.planes())
    assert f1 == f2 and np.array_equal(l1, l2)


def test_canonical_of_bk_state(oracle):
    """The canonical cut of BK's final residual state equals BK's labels, and the flow
    formula sum(max(t,0)) - sum(max(e,0)) equals the augmented flow."""
    g = synth.random_graph(64, 48, 5, cap_max=30, tlink_max=50)
    f, lab, fe = oracle.maxflow_bk(*g.planes(), return_excess=True)
    assert lab.sum() == (lab == 1).sum()
    assert f == int(np.maximum(g.excess, 0).sum() - np.maximum(fe, 0).sum())


def test_stroke_raster_exact():
    s = strokes.Stroke(np.array([10, 40], np.int32), np.array([10, 10], np.int32), 3, 1)
    idx = strokes.rasterize(s, 64, 32)
    ys, xs = idx // 64, idx % 64
    # a horizontal capsule: x in [7, 43] at y = 10, |dy| <= 3 between the endpoints
    assert set(xs[ys == 10]) == set(range(7, 44))
    assert ys.min() == 7 and ys.max() == 13
    single = strokes.Stroke(np.array([5], np.int32), np.array([5], np.int32), 2, 1)
    d = strokes.rasterize(single, 16, 16)
    assert len(d) == 13  # lattice points with x^2 + y^2 <= 4


def test_generator_is_deterministic():
    a = synth.make_graph(128, 96, 3)
    b = synth.make_graph(128, 96, 3)
    for p, q in zip(a.planes(), b.planes()):
        assert np.array_equal(p, q)
    assert (a.up[0] == 0).all() and (a.down[-1] == 0).all()
    assert (a.left[:, 0] == 0).all() and (a.right[:, -1] == 0).all()
    assert np.array_equal(a.down[:-1], a.up[1:]) and np.array_equal(a.right[:, :-1], a.left[:, 1:])


def test_tiles_view_oracle_small_case(oracle):
    """incremental_tile_list.cl:156-175 by hand: 2x2 tiles of 4x3 pixels, image 9x7 (one
    column and one row past the tile grid stay black)."""
    tiles = np.array([[5, 2], [2, 5]], np.int32)
    v = oracle.tiles_view(tiles, 4, 3, 5, 9, 7)
    red, black = 0xFF0000FF, 0xFF000000
    want = np.full((7, 9), black, np.uint32)
    want[0:3, 0:4] = red
    want[3:6, 4:8] = red
    assert np.array_equal(v, want)
    assert np.all(oracle.tiles_view(np.zeros((0, 0), np.int32), 4, 4, 0, 5, 5) == black)
