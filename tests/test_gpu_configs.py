"""The benchmark's multi-grid and interactive configurations at their stated sizes.

* The 64-grid batch: sides drawn from {256, 384, ..., 1536} (width and height independent),
  one synthetic grid per seed 10000 + i, all solved together in one tile pool; every grid's
  flow and canonical cut equal the exact max-flow oracle's, on the CUDA-graph path and on
  the host-driven path.
* A slice of the interactive workload: one 4096 x 4096 grid, then brush strokes (radius
  8-32, t-links +-10^6), each re-solved warm from the previous residual graph; after every
  stroke the cut equals a cold solve of the edited graph and the flow equals the capacity
  of the cut (weak duality certifies both optimal).
"""
import numpy as np
import pytest

import strokes
import synth
from GraphCut import GraphCut
from GraphCutBatch import GraphCutBatch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch64():
    shapes = synth.batch_shapes(64, seed=2)
    graphs = synth.make_graphs([(w, h, 10_000 + i) for i, (w, h) in enumerate(shapes)])
    return shapes, graphs


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_of_64_mixed_grids_matches_oracle(cuda, oracle, batch64, use_graph):
    torch = cuda
    shapes, graphs = batch64
    assert len(shapes) == 64 and {w % 128 for w, _ in shapes} == {0}
    assert min(min(s) for s in shapes) >= 256 and max(max(s) for s in shapes) <= 1536
    b = GraphCutBatch(shapes, use_graph=use_graph)
    try:
        for i, g in enumerate(graphs):
            b.upload(i, *[torch.from_numpy(p).cuda() for p in g.planes()])
        b.cut()
        for i, g in enumerate(graphs):
            f_ref, l_ref = oracle.maxflow_bk(*g.planes())
            assert b.flow(i) == f_ref, i
            assert np.array_equal(b.labels(i).cpu().numpy(), l_ref), i
    finally:
        b.close()


def test_strokes_on_4096_grid_warm_equals_cold(cuda, oracle):
    torch = cuda
    g = synth.make_graph(4096, 4096, 1001)
    dev = [torch.from_numpy(p).cuda() for p in g.planes()]
    rng = np.random.default_rng(31)
    t = g.excess.copy()
    warm = GraphCut(g.width, g.height)
    cold = GraphCut(g.width, g.height)
    try:
        warm.upload_capacities(*dev)
        warm.cut()
        for k in range(24):
            s = strokes.random_stroke(rng, g.width, g.height)
            warm.edit_stroke(s.xs, s.ys, s.radius, s.value)
            t = strokes.apply(t, s)
            warm.cut()
            cold.upload_capacities(*dev[:4], torch.from_numpy(t).cuda())
            cold.cut()
            lw, lc = warm.labels_host(), cold.labels_host()
            assert warm.flow == cold.flow, k
            assert np.array_equal(lw, lc), k
            if k % 6 == 5:   # certificate: flow == capacity of the cut
                assert oracle.cut_capacity(g.up, g.down, g.left, g.right, t, lw) == warm.flow, k
    finally:
        warm.close()
        cold.close()


def test_runtime_autotuner_on_the_device(cuda, tmp_path):
    """The tuner times every candidate schedule on a grid of the class, each candidate's cut
    must equal the others' (tune raises otherwise), and the choice is cached: asking again
    does no device work, a new tuner reads it from the file, and GraphCut picks it up."""
    import autotune
    grid = {"discharge_iters": [2, 4], "pulses_per_relabel": [1, 2], "initial_relabel": [0, 1]}
    t = autotune.Autotuner(cache_path=str(tmp_path / "sched.json"), grid=grid, repeats=1)
    best = t.ensure(0, 320, 320)          # class of grids up to 512 x 512
    assert set(best) == set(autotune.KNOBS) and t.tunings == 1
    assert t.ensure(0, 300, 333) == best and t.tunings == 1
    t2 = autotune.Autotuner(cache_path=str(tmp_path / "sched.json"), grid=grid)
    assert t2.schedule(0, 256, 256) == best
    old = autotune._default
    autotune._default = t2
    try:
        gc = GraphCut(256, 256)
        assert (gc.opts.discharge_iters, gc.opts.pulses_per_relabel, gc.opts.initial_relabel) == \
            (best["discharge_iters"], best["pulses_per_relabel"], best["initial_relabel"])
        gc.close()
    finally:
        autotune._default = old


def test_solve_pipeline_frames_match_single_solves(cuda, oracle):
    """SolvePipeline (copies of frame k+1 overlapping the solve of frame k) returns, frame by
    frame and in order, the exact flow and cut of each frame: from (image, t-links) frames and
    from (image, colour models) frames, with frames that differ from one another."""
    import torch

    from GraphCut import _as_rgba32, unpack_labels
    from gmm_tlinks import Mixture
    from pipeline import SolvePipeline
    graphs = [synth.make_graph(300, 200, 900 + k, keep_image=True) for k in range(5)]
    refs = [oracle.maxflow_bk(*g.planes()) for g in graphs]
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    frames = [(pin(_as_rgba32(g.image)), pin(g.excess)) for g in graphs]
    with SolvePipeline(300, 200) as pipe:
        out = list(pipe.run(frames + frames[::-1]))
        assert len(out) == 10
        for (f, bits), k in zip(out, list(range(5)) + list(range(4, -1, -1))):
            assert f == refs[k][0], k
            assert np.array_equal(unpack_labels(bits, 300), refs[k][1]), k
        mframes = [(pin(_as_rgba32(g.image)), tuple(Mixture.from_components(c) for c in g.models))
                   for g in graphs]
        for (f, bits), k in zip(pipe.run(mframes), range(5)):
            assert f == refs[k][0], k
            assert np.array_equal(unpack_labels(bits, 300), refs[k][1]), k


def test_device_trace_of_a_graph_solve(cuda):
    """The device-side trace sees inside a CUDA-graph solve: upload, solve start, active list,
    discharge pulses, flood rounds (whose first round rebuilds changed masks: no separate
    rebuild launch), the flood check and the solve's end, in launch order with increasing
    stamps; off, it records nothing."""
    import _gcut
    g = synth.make_graph(512, 512, 21)
    # a fixed schedule without the initial relabel: a fresh solve (a tuned schedule cached
    # by another test could start with the relabel, which makes the image warm)
    with GraphCut(g.width, g.height, discharge_iters=3, bfs=2, initial_relabel=False) as gc:
        gc.set_trace(True)
        gc.upload_capacities(*g.planes())
        gc.cut()
        gc.labels()
        tr = gc.trace()
        kinds = [k for k, _ in tr]
        assert kinds[0] == "upload" and kinds[1] == "begin" and kinds[-1] == "labels"
        assert "end" in kinds and kinds.index("end") < kinds.index("labels")
        assert kinds.count("discharge") == gc.stats()["pulses"]
        for k in ("active_list", "flood_first", "check"):
            assert k in kinds, k
        assert "masks" not in kinds
        stamps = [t for _, t in tr]
        assert all(b >= a for a, b in zip(stamps, stamps[1:]))
        summ = _gcut.trace_summary(tr)
        assert summ["discharge"][0] == kinds.count("discharge")
        # every solver kernel of the graph marks its start once; the fresh solve of a pool
        # this small begins with the one launch that also builds the first active list
        kernel_marks = sum(kinds.count(k) for k in ("begin", "active_list", "discharge",
                                                    "flood_first", "flood", "bfs_first", "bfs"))
        assert gc.stats()["launches"] == kernel_marks - 1, (" ".join(kinds), gc.stats())
        gc.set_trace(False)
        gc.upload_capacities(*g.planes())
        gc.cut()
        assert gc.trace() == []
