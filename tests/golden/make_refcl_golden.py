"""Makes golden fixtures from the reference's own graph-cut kernels.

``oracle/refcl.py`` runs graphcut.cl, compiled unchanged as C, under the reference's host
loop (GraphCut.cut, GraphCut.pyx:348-418) on 800 x 608 integer graphs (the kernels' fixed
image size, graphcut.cl:15-16), and at 512 x 512 from a copy with those two lines
rewritten (the reference's CPU-sized configuration).  This script runs it on eight graphs
and writes, for each,
``tests/golden/refcl_<name>.npz``: the flow value, the canonical minimum cut of the
kernels' final residual graph (pixels reachable from excess > 0, bit-packed rows), and the
kernels' step counts (push iterations, relabel passes, BFS rounds).  Each answer is checked
against the oracle's Boykov-Kolmogorov solver before it is written, and the restated
reference schedule (``ref_tiled``) must take the same steps.

The graphs:

* ``scores``: the reference's own test input, ``excess = scoreBg - scoreFg``
  (test_GraphCut.py:44-47) from its ``scoreFg.npy`` / ``scoreBg.npy``, in the solver's integer
  units (``make_golden.tlinks``); n-links from the synthetic image of ``make_golden``.  The
  excess plane is stored in the fixture, since the score files are not present where the
  tests run.
* ``synth1`` .. ``synth3``: the benchmark's synthetic graphs (``synth.make_graph``) at
  800 x 608.
* ``directed``: independent random capacities in all four directions and random t-links.
* ``sparse_sources``: sink pixels everywhere except six blocks of sources, so that most
  tiles start unloaded and are loaded as flow reaches them (GraphCut.pyx:394-405).
* ``config0_seed1``, ``config0_seed2``: the 512 x 512 synthetic graphs of the CPU-sized
  configuration.

Inputs other than ``scores`` are regenerated from their seeds by ``graph()``; each fixture
holds a SHA-256 of its input planes, so a test notices a generator that changed.

    python tests/golden/make_refcl_golden.py REFERENCE_DIR [NAME ...]
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "cl-util_b200"), ROOT, HERE):
    if p not in sys.path:
        sys.path.insert(0, p)

W, H = 800, 608
NAMES = ("scores", "synth1", "synth2", "synth3", "directed", "sparse_sources",
         "config0_seed1", "config0_seed2")


STEP_NAMES = ("iterations", "relabels", "bfs_rounds")


def size(name: str):
    """(width, height) of a fixture's graph."""
    return (512, 512) if name.startswith("config0") else (W, H)


def planes_sha256(planes) -> str:
    h = hashlib.sha256()
    for a in planes:
        h.update(np.ascontiguousarray(a, dtype=np.int32).tobytes())
    return h.hexdigest()


def graph(name: str, excess=None):
    """The input planes (up, down, left, right, excess) of a fixture; ``scores`` needs the
    fixture's excess plane."""
    if name == "scores":
        from make_golden import nlink_planes
        planes, _ = nlink_planes(H, W, excess)
        return (*planes, np.ascontiguousarray(excess, dtype=np.int32))
    if name.startswith("synth"):
        import synth
        return synth.make_graph(W, H, int(name[len("synth"):])).planes()
    if name.startswith("config0_seed"):
        import synth
        return synth.make_graph(512, 512, int(name[len("config0_seed"):])).planes()
    rng = np.random.default_rng({"directed": 5, "sparse_sources": 6}[name])
    up, down, left, right = (rng.integers(0, 60, (H, W)).astype(np.int32) for _ in range(4))
    up[0, :] = 0
    down[-1, :] = 0
    left[:, 0] = 0
    right[:, -1] = 0
    ex = rng.integers(-300, 300, (H, W)).astype(np.int32)
    if name == "sparse_sources":
        ex = -np.abs(ex) - 1
        for _ in range(6):
            y, x = rng.integers(0, H - 40), rng.integers(0, W - 40)
            ex[y:y + 40, x:x + 40] = rng.integers(100, 5000, (40, 40))
    return up, down, left, right, ex


def main(ref_root, names=NAMES):
    from make_golden import tlinks
    from oracle import oracle as O
    from oracle import refcl
    if not refcl.build(ref_root):
        sys.exit(f"graphcut.cl not found under {ref_root}")
    fg = np.load(os.path.join(ref_root, "scoreFg.npy")).reshape(H, W)
    bg = np.load(os.path.join(ref_root, "scoreBg.npy")).reshape(H, W)
    for name in names:
        excess = tlinks(fg, bg) if name == "scores" else None
        planes = graph(name, excess)
        r = refcl.cut(*planes)
        st = r["stats"]
        assert st["non_integral_values"] == 0 and st["barriers_without_fibers"] == 0, st
        flow, labels = O.canonical(r["up"], r["down"], r["left"], r["right"], r["excess"],
                                   planes[4])
        f_bk, l_bk = O.maxflow_bk(*planes)
        assert flow == f_bk and np.array_equal(labels, l_bk), (name, flow, f_bk)
        f_t, _, st_t = O.ref_tiled(*planes)
        steps = np.array([st[k] for k in STEP_NAMES], np.int64)
        assert f_t == flow and np.array_equal(steps, st_t), (name, steps, st_t)
        serial = refcl.cut(*planes, schedule=refcl.SCHEDULE_SERIAL)
        f_serial, _ = O.canonical(serial["up"], serial["down"], serial["left"],
                                  serial["right"], serial["excess"], planes[4])
        extra = {"excess": planes[4]} if name == "scores" else {}
        out = os.path.join(HERE, f"refcl_{name}.npz")
        np.savez_compressed(out, planes_sha256=planes_sha256(planes), flow=flow,
                            labels_packed=np.packbits(labels, axis=1, bitorder="little"),
                            steps=steps, serial_flow=f_serial, **extra)
        print(f"{out}: flow {flow}, source pixels {int(labels.sum())}, steps {steps.tolist()}, "
              f"serial-schedule flow {f_serial}, {os.path.getsize(out)} bytes")


if __name__ == "__main__":
    if len(sys.argv) < 2 or any(n not in NAMES for n in sys.argv[2:]):
        sys.exit("usage: python tests/golden/make_refcl_golden.py REFERENCE_DIR [NAME ...]  "
                 "(the checkout of rheiland/cl-util holding graphcut.cl, scoreFg.npy and "
                 f"scoreBg.npy; names from {', '.join(NAMES)}; default all)")
    main(sys.argv[1], tuple(sys.argv[2:]) or NAMES)
