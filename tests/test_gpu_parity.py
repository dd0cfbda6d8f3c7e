"""Parity of the CUDA solver with the oracle (bit-exact flow value and canonical cut).

Every case calls libgcut through the C ABI (via the GraphCut class) and compares with the
Boykov-Kolmogorov oracle on the same seeded inputs; at the benchmark size (2048^2) the
oracle still finishes in well under a second, so the comparison is direct, plus the
size-independent certificate flow == capacity(cut).
"""
import numpy as np
import pytest

import synth
import strokes
from GraphCut import GraphCut
from GraphCutBatch import GraphCutBatch

pytestmark = pytest.mark.gpu


def solve_gpu(g, **kw):
    with GraphCut(g.width, g.height, **kw) as gc:
        gc.upload_capacities(*g.planes())
        gc.cut()
        return gc.flow, gc.labels().cpu().numpy(), gc.stats()


def check(g, oracle, **kw):
    f_ref, l_ref = oracle.maxflow_bk(*g.planes())
    f, lab, st = solve_gpu(g, **kw)
    assert f == f_ref, (f, f_ref, st)
    assert np.array_equal(lab, l_ref), (int((lab != l_ref).sum()), st)
    return st


@pytest.mark.parametrize("w,h,seed", [(512, 512, 0), (512, 512, 1), (256, 384, 2), (64, 96, 3),
                                      (32, 32, 4), (1024, 512, 5)])
@pytest.mark.parametrize("graph", [True, False])
def test_synthetic_matches_oracle(cuda, oracle, w, h, seed, graph):
    check(synth.make_graph(w, h, seed), oracle, use_graph=graph)


@pytest.mark.parametrize("w,h", [(1, 1), (1, 7), (7, 1), (33, 31), (100, 37), (300, 211)])
def test_ragged_sizes(cuda, oracle, w, h):
    check(synth.random_graph(w, h, w * 1000 + h, cap_max=30, tlink_max=60), oracle)


@pytest.mark.parametrize("seed,sym,sparsity", [(0, True, 0.0), (1, False, 0.0), (2, True, 0.4),
                                               (3, False, 0.6), (4, True, 0.9)])
@pytest.mark.parametrize("graph", [True, False])
def test_random_graphs(cuda, oracle, seed, sym, sparsity, graph):
    g = synth.random_graph(256, 192, seed, cap_max=100, tlink_max=150, sparsity=sparsity,
                           symmetric=sym)
    check(g, oracle, use_graph=graph)


@pytest.mark.parametrize("w,h", [(1, 1), (7, 3), (33, 31), (100, 37), (257, 130), (1000, 3),
                                 (64, 64)])
def test_packed_labels_match_oracle(cuda, oracle, w, h):
    """Bit-packed labels (device and host forms) unpack to the oracle's canonical cut, and
    the padding bits of each row's last byte are 0."""
    from GraphCut import unpack_labels
    g = synth.random_graph(w, h, 7 * w + h, cap_max=30, tlink_max=60)
    _, l_ref = oracle.maxflow_bk(*g.planes())
    with GraphCut(w, h) as gc:
        gc.upload_capacities(*g.planes())
        gc.cut()
        dev = gc.labels_packed().cpu().numpy()
        host = gc.labels_packed_host()
    assert host.shape == (h, (w + 7) // 8)
    assert np.array_equal(dev, host)
    assert np.array_equal(host, np.packbits(l_ref, axis=1, bitorder="little"))
    assert np.array_equal(unpack_labels(host, w), l_ref)


@pytest.mark.parametrize("w,h,graph", [(1, 1, True), (33, 31, True), (257, 130, True),
                                       (257, 130, False), (1000, 3, True)])
def test_cut_labels_matches_cut_then_labels(cuda, oracle, w, h, graph):
    """gc_solve_labels (solve and labels, one host wait) gives the flow and the labels, packed
    and one byte per pixel, of gc_solve followed by gc_labels / gc_labels_packed."""
    from GraphCut import unpack_labels
    g = synth.random_graph(w, h, 3 * w + h, cap_max=30, tlink_max=60)
    f_ref, l_ref = oracle.maxflow_bk(*g.planes())
    with GraphCut(w, h, use_graph=graph) as gc:
        gc.upload_capacities(*g.planes())
        lab = gc.cut_labels().cpu().numpy()
        assert gc.flow == f_ref
        assert np.array_equal(lab, l_ref)
        gc.upload_capacities(*g.planes())
        bits = gc.cut_labels(packed=True).cpu().numpy()
        assert gc.flow == f_ref
        assert np.array_equal(unpack_labels(bits, w), l_ref)
        assert np.array_equal(gc.labels().cpu().numpy(), l_ref)


def test_cut_labels_graph_follows_buffers_fresh_and_warm(cuda, oracle):
    """The solve graph that ends with the labels: its labels nodes follow the caller's buffer
    from call to call (two buffers alternate, bytes and packed), on a synthetic image and on
    random capacities, fresh and warm (after stroke edits), each equal to the exact cut."""
    import torch
    from GraphCut import unpack_labels
    rng = np.random.default_rng(5)
    for g in (synth.make_graph(300, 200, 4), synth.random_graph(300, 200, 6, cap_max=30,
                                                                tlink_max=60)):
        w, h = g.width, g.height
        bufs = [torch.empty((h, w), dtype=torch.uint8, device="cuda") for _ in range(2)]
        pbufs = [torch.empty((h, (w + 7) // 8), dtype=torch.uint8, device="cuda")
                 for _ in range(2)]
        t = g.excess.copy()
        with GraphCut(w, h) as gc:
            gc.upload_capacities(*g.planes())
            for k in range(6):
                if k >= 2:   # warm: the graph variant that floods the previous flow first
                    s = strokes.random_stroke(rng, w, h)
                    gc.edit_stroke(s.xs, s.ys, s.radius, s.value)
                    t = strokes.apply(t, s)
                f_ref, l_ref = oracle.maxflow_bk(g.up, g.down, g.left, g.right, t)
                for b in (bufs[k % 2], bufs[(k + 1) % 2]):
                    b.fill_(7)
                    gc.cut_labels(out=b)
                    assert gc.flow == f_ref, k
                    assert np.array_equal(b.cpu().numpy(), l_ref), k
                    if k < 2:
                        gc.upload_capacities(*g.planes())
                pb = pbufs[k % 2]
                pb.fill_(0xFF)
                gc.cut_labels(out=pb, packed=True)
                assert np.array_equal(unpack_labels(pb.cpu().numpy(), w), l_ref), k
                if k < 2:
                    gc.upload_capacities(*g.planes())


def test_cut_labels_graph_strides_over_a_large_image(cuda, oracle):
    """2500^2: the labels kernels inside the solve graph cap their grid at 4 CTAs per SM and
    stride over the tile rows (2500 rows x 79 tiles need 771 CTAs of 256 threads), bytes and
    packed, equal to the exact cut."""
    from GraphCut import unpack_labels
    g = synth.make_graph(2500, 2500, 7)
    f_ref, l_ref = oracle.maxflow_bk(*g.planes())
    with GraphCut(g.width, g.height) as gc:
        gc.upload_capacities(*g.planes())
        lab = gc.cut_labels().cpu().numpy()
        assert gc.flow == f_ref
        assert np.array_equal(lab, l_ref)
        gc.upload_capacities(*g.planes())
        bits = gc.cut_labels(packed=True).cpu().numpy()
        assert gc.flow == f_ref
        assert np.array_equal(unpack_labels(bits, g.width), l_ref)


def test_handles_in_caller_memory(cuda, oracle):
    """gc_create_in: handles placed in one caller-owned buffer solve like gc_create, and
    the memory is reused for a handle of another size after gc_destroy."""
    import torch
    from _gcut import GCError
    sizes = [(300, 211), (64, 500), (513, 97)]
    need = max(GraphCut.arena_bytes(w, h) for w, h in sizes)
    buf = torch.empty(need + 4096, dtype=torch.uint8, device="cuda")
    base = buf.data_ptr()
    for k, (w, h) in enumerate(sizes):
        g = synth.random_graph(w, h, 40 + k, cap_max=40, tlink_max=80)
        f_ref, l_ref = oracle.maxflow_bk(*g.planes())
        buf.fill_(0xAB)   # garbage left by an earlier tenant must not matter
        with GraphCut(w, h, arena=(base, GraphCut.arena_bytes(w, h))) as gc:
            gc.upload_capacities(*g.planes())
            gc.cut()
            assert gc.flow == f_ref
            assert np.array_equal(gc.labels_host(), l_ref)
    with pytest.raises(GCError):   # too small
        GraphCut(300, 211, arena=(base, GraphCut.arena_bytes(300, 211) - 256))
    with pytest.raises(GCError):   # not 256-byte aligned
        GraphCut(64, 64, arena=(base + 16, need))


@pytest.mark.parametrize("w,h,seed,kind", [(1, 1, 0, "random"), (1, 9, 1, "random"),
                                            (9, 1, 2, "random"), (33, 31, 3, "random"),
                                            (300, 211, 4, "synthetic"), (512, 512, 5, "synthetic"),
                                            (70, 40, 6, "uniform")])
def test_upload_image_builds_the_generator_planes(cuda, oracle, w, h, seed, kind):
    """gc_upload_rgba(_host): capacities built on the device from the image equal the
    generator's planes bit for bit, and the solve matches the oracle."""
    import torch
    rng = np.random.default_rng(seed)
    if kind == "synthetic":
        g = synth.make_graph(w, h, seed, keep_image=True)
        img, excess = g.image, g.excess
    else:
        img = rng.integers(0, 256, (h, w, 3), dtype=np.uint8)
        if kind == "uniform":
            img[:] = img[0, 0]
        excess = rng.integers(-300, 300, (h, w)).astype(np.int32)
    wv, wh = synth.nlinks(img)
    planes = synth.planes_from_weights(wv, wh, excess) + (excess,)
    f_ref, l_ref = oracle.maxflow_bk(*planes)
    for host in (False, True):
        with GraphCut(w, h) as gc:
            if host:
                gc.upload_image(img, excess)
            else:
                gc.upload_image(torch.from_numpy(img).cuda(), torch.from_numpy(excess).cuda())
            for name, ref in zip(("dUp", "dDown", "dLeft", "dRight", "dExcess"), planes):
                assert np.array_equal(getattr(gc, name).cpu().numpy(), ref), (name, host)
            gc.cut()
            assert gc.flow == f_ref
            assert np.array_equal(gc.labels_host(), l_ref)


@pytest.mark.parametrize("w,h,lam", [(96, 64, 60), (257, 131, 60), (64, 64, 7), (300, 211, 1000)])
def test_upload_image_reference_weighting(cuda, oracle, w, h, lam):
    """gc_upload_rgba_lambda(_host): the reference's n-link rule (graphcut.cl:1018-1031),
    rounded exactly, built on the device equals the oracle's planes bit for bit, and the
    solve on them matches the exact max-flow."""
    import torch
    g = synth.make_graph(w, h, 5, keep_image=True)
    from GraphCut import _as_rgba32
    rgba = _as_rgba32(g.image)
    planes = oracle.nlinks_reference(rgba, lam) + (g.excess,)
    f_ref, l_ref = oracle.maxflow_bk(*planes)
    for host in (False, True):
        with GraphCut(w, h) as gc:
            if host:
                gc.upload_image(g.image, g.excess, lamda=lam)
            else:
                gc.upload_image(torch.from_numpy(g.image).cuda(), torch.from_numpy(g.excess).cuda(),
                                lamda=lam)
            for name, ref in zip(("dUp", "dDown", "dLeft", "dRight", "dExcess"), planes):
                assert np.array_equal(getattr(gc, name).cpu().numpy(), ref), (name, host)
            gc.cut()
            assert gc.flow == f_ref
            assert np.array_equal(gc.labels().cpu().numpy(), l_ref)


def test_upload_image_many_contrasts(cuda, oracle):
    """The device-side scale and weight table of gc_upload_rgba over images of many contrasts
    (so many values of beta): the capacities equal the generator's float64 formula."""
    import torch
    rng = np.random.default_rng(77)
    for k in range(24):
        h, w = int(rng.integers(8, 90)), int(rng.integers(8, 90))
        amp = float(rng.choice([1, 2, 5, 20, 60, 128, 255]))
        img = np.clip(rng.normal(128, amp, (h, w, 3)), 0, 255).astype(np.uint8)
        excess = rng.integers(-50, 50, (h, w)).astype(np.int32)
        wv, wh = synth.nlinks(img)
        planes = synth.planes_from_weights(wv, wh, excess) + (excess,)
        with GraphCut(w, h) as gc:
            gc.upload_image(torch.from_numpy(img).cuda(), torch.from_numpy(excess).cuda())
            for name, ref in zip(("dUp", "dDown", "dLeft", "dRight"), planes):
                assert np.array_equal(getattr(gc, name).cpu().numpy(), ref), (k, name)


@pytest.mark.parametrize("iters,pulses,init", [(1, 1, 0), (4, 1, 1), (64, 5, 0), (32, 1, 1)])
def test_schedules_agree(cuda, oracle, iters, pulses, init):
    g = synth.random_graph(160, 128, 11, cap_max=80, tlink_max=120, symmetric=False)
    check(g, oracle, discharge_iters=iters, bfs=pulses, initial_relabel=bool(init))


def test_edge_cases_zero_and_uniform(cuda, oracle):
    w, h = 96, 64
    z = np.zeros((h, w), np.int32)
    g = synth.Graph(w, h, z, z, z, z, z)
    f, lab, _ = solve_gpu(g)
    assert f == 0 and lab.sum() == 0
    # all source, no sink: no flow, everything on the source side
    g = synth.Graph(w, h, *synth.planes_from_weights(np.full((h - 1, w), 5, np.int32),
                                                     np.full((h, w - 1), 5, np.int32), z),
                    np.full((h, w), 7, np.int32))
    f, lab, _ = solve_gpu(g)
    assert f == 0 and lab.all()
    # single sink pixel in the middle: everything drains into it up to the cut
    e = np.full((h, w), 3, np.int32)
    e[h // 2, w // 2] = -10 ** 6
    g = synth.Graph(w, h, *synth.planes_from_weights(np.full((h - 1, w), 2, np.int32),
                                                     np.full((h, w - 1), 2, np.int32), e), e)
    check(g, oracle)


def test_benchmark_size_2048(cuda, oracle):
    g = synth.make_graph(2048, 2048, 1)
    st = check(g, oracle)
    assert st["cycles"] >= 1


def test_flow_equals_cut_capacity(cuda, oracle):
    g = synth.make_graph(1024, 1024, 7)
    f, lab, _ = solve_gpu(g)
    assert oracle.cut_capacity(*g.planes(), lab) == f


@pytest.mark.parametrize("w,h,seed", [(4096, 4096, 3), (3000, 4096, 21)])
def test_full_size_certificates(cuda, oracle, w, h, seed):
    """Sizes of the stroke and serving workloads, checked without an exact max-flow run:
    (1) the flow equals the capacity of the returned cut, which by weak duality proves both
    optimal; (2) the labels equal the canonical cut recomputed by the oracle from the final
    residual graph the device holds; (3) the flow the oracle derives from that residual
    state equals the reported one."""
    g = synth.make_graph(w, h, seed)
    with GraphCut(w, h) as gc:
        gc.upload_capacities(*g.planes())
        gc.cut()
        f = gc.flow
        lab = gc.labels_host()
        state = [getattr(gc, n).cpu().numpy() for n in ("dUp", "dDown", "dLeft", "dRight", "dExcess")]
    assert oracle.cut_capacity(*g.planes(), lab) == f
    f_state, l_state = oracle.canonical(*state, g.excess)
    assert f_state == f
    assert np.array_equal(l_state, lab)


def test_manual_stepping_matches(cuda, oracle):
    g = synth.random_graph(128, 96, 5, cap_max=60, tlink_max=90)
    f_ref, l_ref = oracle.maxflow_bk(*g.planes())
    with GraphCut(g.width, g.height) as gc:
        gc.upload_capacities(*g.planes())
        done = False
        for _ in range(10000):
            for _ in range(3):
                gc.push()
                gc.relabel()
            gc.startBfs()
            if gc.isCompleted():
                done = True
                break
        assert done
        assert gc.flow == f_ref
        assert np.array_equal(gc.labels().cpu().numpy(), l_ref)


def test_warm_start_strokes_match_cold(cuda, oracle):
    g = synth.make_graph(512, 512, 3)
    rng = np.random.default_rng(0)
    t = g.excess.copy()
    with GraphCut(g.width, g.height) as gc:
        gc.upload_capacities(*g.planes())
        gc.cut()
        for k in range(6):
            s = strokes.random_stroke(rng, g.width, g.height)
            gc.edit_stroke(s.xs, s.ys, s.radius, s.value)
            t = strokes.apply(t, s)
            gc.cut()
            f_ref, l_ref = oracle.maxflow_bk(g.up, g.down, g.left, g.right, t)
            assert gc.flow == f_ref, k
            assert np.array_equal(gc.labels().cpu().numpy(), l_ref), k


def test_edit_tlinks_match_cold(cuda, oracle):
    g = synth.random_graph(200, 150, 9, cap_max=50, tlink_max=80)
    rng = np.random.default_rng(1)
    t = g.excess.copy()
    with GraphCut(g.width, g.height) as gc:
        gc.upload_capacities(*g.planes())
        gc.cut()
        for k in range(4):
            idx = rng.choice(g.width * g.height, 500, replace=False)
            vals = rng.integers(-200, 201, 500).astype(np.int32)
            gc.edit_tlinks(idx, vals)
            t.reshape(-1)[idx] = vals
            gc.cut()
            f_ref, l_ref = oracle.maxflow_bk(g.up, g.down, g.left, g.right, t)
            assert gc.flow == f_ref
            assert np.array_equal(gc.labels().cpu().numpy(), l_ref)


def test_stroke_raster_matches_host(cuda):
    g = synth.random_graph(300, 200, 2, cap_max=5, tlink_max=5)
    rng = np.random.default_rng(5)
    with GraphCut(g.width, g.height) as gc:
        gc.upload_capacities(*g.planes())
        t = g.excess.copy()
        for _ in range(5):
            s = strokes.random_stroke(rng, g.width, g.height)
            gc.edit_stroke(s.xs, s.ys, s.radius, s.value)
            t = strokes.apply(t, s)
        # the excess plane before any solve is exactly the edited t-links
        assert np.array_equal(gc.dExcess.cpu().numpy(), t)


def test_brush_pixel_set_matches_oracle(cuda, oracle):
    """gc_edit_brush: the reference Brush's pixel set (brush.pyx:138-161; centred disc,
    clipped to the image) equals the oracle's restatement, for points, segments and
    polylines, radii 0..40 and strokes that leave the image."""
    g = synth.random_graph(257, 131, 3, cap_max=5, tlink_max=5)
    rng = np.random.default_rng(8)
    with GraphCut(g.width, g.height) as gc:
        gc.upload_capacities(*g.planes())
        t = g.excess.copy()
        for k in range(40):
            n = int(rng.integers(1, 6))
            xs = rng.integers(-30, g.width + 30, n).astype(np.int32)
            ys = rng.integers(-30, g.height + 30, n).astype(np.int32)
            r = int(rng.integers(0, 41))
            v = int(rng.choice([strokes.HARD, -strokes.HARD, 0, 17]))
            gc.edit_brush(xs, ys, r, v)
            t.reshape(-1)[oracle.brush_pixels(xs, ys, r, g.width, g.height)] = v
            if k % 8 == 7:
                assert np.array_equal(gc.dExcess.cpu().numpy(), t), k
        assert np.array_equal(gc.dExcess.cpu().numpy(), t)


def test_brush_warm_solves_match_cold(cuda, oracle):
    """Brush strokes on a solved graph re-solve warm to the exact cut of the edited graph."""
    g = synth.make_graph(384, 256, 12)
    rng = np.random.default_rng(9)
    with GraphCut(g.width, g.height) as gc:
        gc.upload_capacities(*g.planes())
        gc.cut()
        t = g.excess.copy()
        for _ in range(4):
            n = int(rng.integers(1, 5))
            xs = rng.integers(0, g.width, n).astype(np.int32)
            ys = rng.integers(0, g.height, n).astype(np.int32)
            r = int(rng.integers(4, 24))
            v = strokes.HARD if rng.random() < 0.5 else -strokes.HARD
            gc.edit_brush(xs, ys, r, v)
            t.reshape(-1)[oracle.brush_pixels(xs, ys, r, g.width, g.height)] = v
            gc.cut()
            f_ref, l_ref = oracle.maxflow_bk(*(list(g.planes())[:4] + [t]))
            assert gc.flow == f_ref
            assert np.array_equal(gc.labels().cpu().numpy(), l_ref)


def test_batch_matches_per_image(cuda, oracle):
    shapes = synth.batch_shapes(12, seed=3, lo=128, hi=512, step=64)
    graphs = [synth.make_graph(w, h, 100 + i) for i, (w, h) in enumerate(shapes)]
    b = GraphCutBatch(shapes)
    for i, g in enumerate(graphs):
        b.upload(i, *g.planes())
    b.cut()
    for i, g in enumerate(graphs):
        f_ref, l_ref = oracle.maxflow_bk(*g.planes())
        assert b.flow(i) == f_ref, i
        assert np.array_equal(b.labels(i).cpu().numpy(), l_ref), i
    b.close()


def test_negative_capacity_rejected(cuda):
    import _gcut
    g = synth.random_graph(64, 64, 0)
    g.up[5, 5] = -1
    with GraphCut(64, 64) as gc:
        gc.upload_capacities(*g.planes())
        with pytest.raises(_gcut.GCError) as ei:
            gc.cut()
        assert ei.value.code == _gcut.GC_ERR_INVALID


@pytest.mark.parametrize("graph", [True, False])
def test_cycle_cap_reports_not_converged(cuda, graph):
    import _gcut
    g = synth.random_graph(256, 256, 3, cap_max=100, tlink_max=100)
    with GraphCut(256, 256, max_cycles=1, bfs=1, discharge_iters=1, use_graph=graph) as gc:
        gc.upload_capacities(*g.planes())
        with pytest.raises(_gcut.GCError) as ei:
            gc.cut()
        assert ei.value.code == _gcut.GC_ERR_NOT_CONVERGED


@pytest.mark.parametrize("graph", [True, False])
def test_round_cap_reports_not_converged(cuda, graph):
    import _gcut
    g = synth.random_graph(512, 512, 4, cap_max=100, tlink_max=100)
    with GraphCut(512, 512, max_bfs_rounds=1, use_graph=graph) as gc:
        gc.upload_capacities(*g.planes())
        with pytest.raises(_gcut.GCError) as ei:
            gc.cut()
        assert ei.value.code == _gcut.GC_ERR_NOT_CONVERGED


def test_repeated_solves_reuse_graph(cuda, oracle):
    g = synth.make_graph(384, 256, 8)
    f_ref, l_ref = oracle.maxflow_bk(*g.planes())
    with GraphCut(g.width, g.height) as gc:
        for _ in range(4):
            gc.upload_capacities(*g.planes())
            gc.cut()
            assert gc.flow == f_ref
            assert np.array_equal(gc.labels().cpu().numpy(), l_ref)
        gc.cut()  # solving a solved state again is a no-op
        assert gc.flow == f_ref


def test_invalid_options_rejected(cuda):
    import _gcut
    for kw in ({"bfs": 0}, {"discharge_iters": 0}, {"max_cycles": 0}):
        with pytest.raises(_gcut.GCError) as ei:
            GraphCut(64, 64, **kw)
        assert ei.value.code == _gcut.GC_ERR_INVALID


def test_state_errors(cuda):
    import _gcut
    with GraphCut(64, 64) as gc:
        with pytest.raises(_gcut.GCError) as ei:
            gc.cut()
        assert ei.value.code == _gcut.GC_ERR_STATE
        with pytest.raises(_gcut.GCError):
            _ = gc.flow
