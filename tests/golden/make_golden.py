"""Makes the graph-cut golden fixtures from the reference's own score fixtures.

The reference feeds its solver ``excess = scoreBg - scoreFg`` (test_GraphCut.py:44-47),
read from ``scoreFg.npy`` / ``scoreBg.npy``: float32 [608 * 800] per-pixel scores in which a
hard constraint is written as 2^31.  Those files live in the reference tree, which is not
present where the tests run, so this script turns windows of them into fixtures:

* t-links ``floor(100 * (scoreBg - scoreFg) + 0.5)`` clamped to +-10^6 (int32), the solver's
  integer units; a hard constraint becomes a t-link of +-10^6;
* n-links from the synthetic image generator at the window's size and ``IMAGE_SEED`` (the
  image the scores belong to is not part of the reference tree), with a SHA-256 of them so
  that a test notices if the generator ever changes;
* the exact max-flow value and the canonical minimum cut (pixels reachable from excess > 0
  in the final residual graph, bit-packed rows) from the oracle's Boykov-Kolmogorov solver,
  cross-checked against the restated reference schedule (same flow).

    python tests/golden/make_golden.py REFERENCE_DIR
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "cl-util_b200"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

SHAPE = (608, 800)        # graphcut.cl:15-16 (IMAGEW 800, IMAGEH 608)
IMAGE_SEED = 7
# name -> (y0, x0, height, width): "hard" holds every hard constraint of both kinds
# (400 foreground-side, 3320 background-side pixels); "ragged" has sides that are not
# multiples of the 32-pixel tile and about half of whose pixels have excess > 0
WINDOWS = {"hard": (192, 32, 256, 320), "ragged": (238, 203, 131, 257)}
TLINK_SCALE, TLINK_CLAMP = 100.0, 10 ** 6


def tlinks(score_fg, score_bg):
    d = score_bg.astype(np.float64) - score_fg.astype(np.float64)
    return np.clip(np.floor(TLINK_SCALE * d + 0.5), -TLINK_CLAMP, TLINK_CLAMP).astype(np.int32)


def nlink_planes(h, w, excess):
    """Capacity planes from the synthetic image of this size, and the n-links' SHA-256."""
    import synth
    img, _, _ = synth.make_image(w, h, IMAGE_SEED)
    wv, wh = synth.nlinks(img)
    digest = hashlib.sha256(wv.tobytes() + wh.tobytes()).hexdigest()
    return synth.planes_from_weights(wv, wh, excess), digest


def main(ref_root):
    from oracle import oracle as O
    fg = np.load(os.path.join(ref_root, "scoreFg.npy")).reshape(SHAPE)
    bg = np.load(os.path.join(ref_root, "scoreBg.npy")).reshape(SHAPE)
    for name, (y0, x0, h, w) in WINDOWS.items():
        ex = tlinks(fg[y0:y0 + h, x0:x0 + w], bg[y0:y0 + h, x0:x0 + w])
        (up, down, left, right), digest = nlink_planes(h, w, ex)
        flow, labels = O.maxflow_bk(up, down, left, right, ex)
        # the restated reference schedule wants whole tiles: pad with isolated pixels
        # (no capacity, no excess), which leave the flow unchanged
        ph, pw = -(-h // 32) * 32, -(-w // 32) * 32
        pad = [np.pad(a, ((0, ph - h), (0, pw - w))) for a in (up, down, left, right, ex)]
        flow_ref, _, _ = O.ref_tiled(*pad)
        assert flow == flow_ref, (name, flow, flow_ref)
        out = os.path.join(HERE, f"scores_{name}.npz")
        np.savez_compressed(out, excess=ex, window=np.array([y0, x0, h, w]),
                            image_seed=IMAGE_SEED, nlinks_sha256=digest, flow=flow,
                            labels_packed=np.packbits(labels, axis=1, bitorder="little"))
        print(f"{out}: {w}x{h}, flow {flow}, source pixels {int(labels.sum())}, "
              f"{os.path.getsize(out)} bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py REFERENCE_DIR  (the checkout of "
                 "rheiland/cl-util holding scoreFg.npy and scoreBg.npy)")
    main(sys.argv[1])
