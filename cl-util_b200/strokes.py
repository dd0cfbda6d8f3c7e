"""Brush strokes: random polylines and their exact integer rasterisation.

The reference turns a stroke segment into a pixel set on the host with skimage's line and
disc rasterisers (brush.pyx:138-161) and paints label 7 on the device (brush.cl:1-13).
Here a stroke is a polyline with a radius; a pixel (x, y) is covered when its centre lies
within `radius` of some segment, decided with the exact int64 test used by the device
kernel (``gc_edit_stroke``): with a = p - A, b = B - A, L = b.b, s = a.b, the pixel is
inside iff |a|^2 <= r^2 (s <= 0), |p - B|^2 <= r^2 (s >= L), else |a|^2 L - s^2 <= r^2 L.
Covered pixels get the t-link +10**6 (hard foreground) or -10**6 (hard background).
"""
from __future__ import annotations

import dataclasses

import numpy as np

HARD = 10 ** 6


@dataclasses.dataclass
class Stroke:
    xs: np.ndarray   # int32 polyline x
    ys: np.ndarray   # int32 polyline y
    radius: int
    value: int       # +HARD or -HARD


def random_stroke(rng: np.random.Generator, width: int, height: int, rmin=8, rmax=32,
                  npts=(2, 5)) -> Stroke:
    n = int(rng.integers(npts[0], npts[1] + 1))
    x0, y0 = rng.integers(0, width), rng.integers(0, height)
    step = max(8, min(width, height) // 8)
    xs = np.clip(x0 + np.cumsum(np.r_[0, rng.integers(-step, step + 1, n - 1)]), 0, width - 1)
    ys = np.clip(y0 + np.cumsum(np.r_[0, rng.integers(-step, step + 1, n - 1)]), 0, height - 1)
    return Stroke(xs.astype(np.int32), ys.astype(np.int32), int(rng.integers(rmin, rmax + 1)),
                  HARD if rng.random() < 0.5 else -HARD)


def rasterize(s: Stroke, width: int, height: int) -> np.ndarray:
    """Flat indices (y * width + x) of the covered pixels, increasing."""
    r = int(s.radius)
    x0 = max(0, int(s.xs.min()) - r); x1 = min(width - 1, int(s.xs.max()) + r)
    y0 = max(0, int(s.ys.min()) - r); y1 = min(height - 1, int(s.ys.max()) + r)
    if x1 < x0 or y1 < y0:
        return np.zeros(0, np.int64)
    py, px = np.mgrid[y0:y1 + 1, x0:x1 + 1].astype(np.int64)
    hit = np.zeros(px.shape, bool)
    r2 = r * r
    pts = list(zip(s.xs.astype(np.int64), s.ys.astype(np.int64)))
    segs = list(zip(pts[:-1], pts[1:])) if len(pts) > 1 else [(pts[0], pts[0])]
    for (ax, ay), (bx, by) in segs:
        dx, dy = px - ax, py - ay
        ux, uy = bx - ax, by - ay
        L = ux * ux + uy * uy
        sdot = dx * ux + dy * uy
        if L == 0:
            hit |= dx * dx + dy * dy <= r2
            continue
        ex, ey = px - bx, py - by
        before = sdot <= 0
        after = sdot >= L
        mid = ~before & ~after
        hit |= before & (dx * dx + dy * dy <= r2)
        hit |= after & (ex * ex + ey * ey <= r2)
        hit |= mid & ((dx * dx + dy * dy) * L - sdot * sdot <= r2 * L)
    yy, xx = np.nonzero(hit)
    return np.sort((yy + y0) * width + (xx + x0))


def apply(excess_tlinks: np.ndarray, s: Stroke) -> np.ndarray:
    """The t-link plane after the stroke (cold-solve input)."""
    h, w = excess_tlinks.shape
    out = excess_tlinks.copy()
    out.reshape(-1)[rasterize(s, w, h)] = s.value
    return out
