"""Session pools (gcp_*): many graphs resident in one tile pool, subsets solved by one
launch; every result bit-exact against the exact max-flow oracle, and the slots a solve does
not list keep their results."""
import numpy as np
import pytest

import strokes
import synth
from session_pool import SessionPool

pytestmark = pytest.mark.gpu


def _labels(pool, slot, w):
    from GraphCut import unpack_labels
    return unpack_labels(pool.labels_packed(slot).cpu().numpy(), w)


@pytest.mark.parametrize("use_graph", [True, False])
def test_subsets_fresh_warm_and_untouched(cuda, oracle, use_graph):
    torch = cuda
    shapes = [(256, 192), (100, 37), (512, 384), (33, 31), (640, 480)]
    graphs = [synth.make_graph(w, h, 50 + i) for i, (w, h) in enumerate(shapes)]
    pool = SessionPool(4096, 16, use_graph=use_graph)
    slots = [3, 0, 9, 15, 7]
    t0s = {}
    try:
        for s, g in zip(slots, graphs):
            t0 = t0s[s] = pool.alloc_tiles(g.width, g.height)
            pool.open(s, g.width, g.height, t0)
            pool.upload_capacities(s, *[torch.from_numpy(p).cuda() for p in g.planes()])
        ref = [oracle.maxflow_bk(*g.planes()) for g in graphs]
        # two fresh slots first, then the rest together
        pool.solve([slots[0], slots[2]])
        for k in (0, 2):
            assert pool.flow(slots[k]) == ref[k][0]
            assert np.array_equal(_labels(pool, slots[k], graphs[k].width), ref[k][1])
        pool.solve([slots[1], slots[3], slots[4]])
        for k in range(5):
            assert pool.flow(slots[k]) == ref[k][0], k
            assert np.array_equal(_labels(pool, slots[k], graphs[k].width), ref[k][1]), k
        # strokes on two slots, warm re-solve of those two with a fresh re-upload of a third
        rng = np.random.default_rng(4)
        ts = [g.excess.copy() for g in graphs]
        for k in (0, 4):
            st = strokes.random_stroke(rng, graphs[k].width, graphs[k].height)
            pool.edit_stroke(slots[k], st.xs, st.ys, st.radius, st.value)
            ts[k] = strokes.apply(ts[k], st)
        pool.upload_capacities(slots[3], *[torch.from_numpy(p).cuda() for p in graphs[3].planes()])
        pool.solve([slots[4], slots[3], slots[0]])
        for k in range(5):
            f, l = oracle.maxflow_bk(graphs[k].up, graphs[k].down, graphs[k].left,
                                     graphs[k].right, ts[k])
            assert pool.flow(slots[k]) == f, k
            assert np.array_equal(_labels(pool, slots[k], graphs[k].width), l), k
        # a slot closes and its tiles take an image of another size
        pool.close(slots[2])
        pool.free_tiles(t0s[slots[2]], *shapes[2])
        g = synth.make_graph(300, 211, 99, keep_image=True)
        t0 = pool.alloc_tiles(g.width, g.height)
        assert t0 is not None
        pool.open(slots[2], g.width, g.height, t0)
        pool.upload_image(slots[2], g.image, g.excess)
        pool.solve([slots[2]])
        assert pool.flow(slots[2]) == oracle.maxflow_bk(*g.planes())[0]
    finally:
        pool.close_pool()


def test_rejects_overlap_and_bad_slots(cuda):
    from _gcut import GCError
    pool = SessionPool(64, 4)
    try:
        pool.open(0, 128, 128, 0)            # 16 tiles
        with pytest.raises(GCError):
            pool.open(1, 64, 64, 10)         # overlaps tiles 10..13
        with pytest.raises(GCError):
            pool.open(1, 256, 256, 0 + 16)   # 64 tiles past the pool end
        with pytest.raises(GCError):
            pool.open(4, 32, 32, 40)         # no slot 4
        with pytest.raises(GCError):
            pool.solve([0])                  # not uploaded
        pool.open(1, 64, 64, 16)
    finally:
        pool.close_pool()


@pytest.mark.parametrize("use_graph", [True, False])
def test_solve_labels_matches_solve_then_labels(cuda, oracle, use_graph):
    """gcp_solve_labels (the solve and every slot's labels with one host wait) gives the
    flows and labels of gcp_solve followed by gcp_labels / gcp_labels_packed, fresh and
    warm, packed and one byte per pixel."""
    torch = cuda
    from GraphCut import unpack_labels
    shapes = [(300, 211), (64, 97), (515, 260)]
    graphs = [synth.make_graph(w, h, 70 + i) for i, (w, h) in enumerate(shapes)]
    pool = SessionPool(4096, 8, use_graph=use_graph)
    slots = [5, 1, 2]
    try:
        for s, g in zip(slots, graphs):
            pool.open(s, g.width, g.height, pool.alloc_tiles(g.width, g.height))
            pool.upload_capacities(s, *[torch.from_numpy(p).cuda() for p in g.planes()])
        outs = pool.solve_labels(slots, packed=True)
        for k, g in enumerate(graphs):
            f, l = oracle.maxflow_bk(*g.planes())
            assert pool.flow(slots[k]) == f, k
            assert np.array_equal(unpack_labels(outs[k].cpu().numpy(), g.width), l), k
        # warm re-solve after strokes, labels one byte per pixel
        rng = np.random.default_rng(11)
        ts = [g.excess.copy() for g in graphs]
        for k in (0, 2):
            st = strokes.random_stroke(rng, graphs[k].width, graphs[k].height)
            pool.edit_stroke(slots[k], st.xs, st.ys, st.radius, st.value)
            ts[k] = strokes.apply(ts[k], st)
        outs = pool.solve_labels([slots[2], slots[0]], packed=False)
        for k, out in zip((2, 0), outs):
            g = graphs[k]
            f, l = oracle.maxflow_bk(g.up, g.down, g.left, g.right, ts[k])
            assert pool.flow(slots[k]) == f, k
            assert np.array_equal(out.cpu().numpy(), l), k
            assert np.array_equal(pool.labels(slots[k]).cpu().numpy(), l), k
    finally:
        pool.close_pool()
