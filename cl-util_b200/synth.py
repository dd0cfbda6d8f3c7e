"""Seeded synthetic segmentation graphs on a 4-connected pixel grid.

The reference solver (``GraphCut.pyx`` + ``graphcut.cl``) is fed an RGBA image and a float
excess plane ``scoreBg - scoreFg`` (``test_GraphCut.py:44-47``) and derives its n-link
capacities on the device (``graphcut.cl:1018-1132``).  Its image fixture is not part of the
reference tree, so the workloads here are built from a seed:

* an RGB ``uint8`` image of 12 random filled ellipses, Gaussian-blurred (sigma 3) with
  N(0, 8) noise added, rounded and clipped to [0, 255];
* foreground / background scores ``-log p(x)`` under 2-component full-covariance RGB
  Gaussian mixtures fitted (20 EM steps) to the pixels of two of the ellipses;
* t-link (signed excess) ``round(100 * (score_bg - score_fg))`` clamped to +-10**6:
  positive values are source capacities, negative values sink capacities;
* n-link capacity ``round(50 * exp(-beta * |I_i - I_j|^2))`` with
  ``beta = 1 / (2 * mean |dI|^2)`` over every 4-neighbour pair, symmetric in the two
  directions; capacities that would leave the image are 0 (``graphcut.cl:1107-1108``).

All arithmetic after the scores is integer, so the planes are exactly reproducible from
``(width, height, seed)``.  ``round`` is round-half-up (``floor(x + 0.5)``).

Planes are int32 ``[height, width]`` arrays, C-contiguous:
``up[y, x]`` is the capacity of edge (x, y) -> (x, y-1), ``down`` -> (x, y+1),
``left`` -> (x-1, y), ``right`` -> (x+1, y).
"""
from __future__ import annotations

import dataclasses

import numpy as np
from scipy import ndimage

from gmm_tlinks import components

N_ELLIPSES = 12
BLUR_SIGMA = 3.0
NOISE_SIGMA = 8.0
NLINK_SCALE = 50.0
TLINK_SCALE = 100.0
TLINK_CLAMP = 10 ** 6
EM_STEPS = 20
MAX_FIT_SAMPLES = 20000


@dataclasses.dataclass
class Graph:
    """Capacity planes of one grid graph (int32, ``[height, width]``)."""
    width: int
    height: int
    up: np.ndarray
    down: np.ndarray
    left: np.ndarray
    right: np.ndarray
    excess: np.ndarray
    image: np.ndarray | None = None
    models: tuple | None = None   # (fg, bg) components (gmm_tlinks.components), with image

    def planes(self):
        return self.up, self.down, self.left, self.right, self.excess

    def copy(self) -> "Graph":
        return Graph(self.width, self.height, self.up.copy(), self.down.copy(),
                     self.left.copy(), self.right.copy(), self.excess.copy(), self.image,
                     self.models)


def _ellipse_masks(width, height, rng, n):
    """Draws ``n`` ellipses: returns a list of (y0, y1, x0, x1, bbox-mask, colour)."""
    out = []
    short = min(width, height)
    for _ in range(n):
        cx = rng.uniform(0, width)
        cy = rng.uniform(0, height)
        a = rng.uniform(0.05, 0.30) * short
        b = rng.uniform(0.05, 0.30) * short
        theta = rng.uniform(0.0, np.pi)
        colour = rng.integers(0, 256, 3)
        r = max(a, b)
        x0, x1 = max(0, int(cx - r)), min(width, int(cx + r) + 1)
        y0, y1 = max(0, int(cy - r)), min(height, int(cy + r) + 1)
        if x0 >= x1 or y0 >= y1:
            out.append((0, 0, 0, 0, np.zeros((0, 0), bool), colour))
            continue
        ys = np.arange(y0, y1, dtype=np.float64)[:, None] - cy
        xs = np.arange(x0, x1, dtype=np.float64)[None, :] - cx
        c, s = np.cos(theta), np.sin(theta)
        u = (xs * c + ys * s) / a
        v = (-xs * s + ys * c) / b
        out.append((y0, y1, x0, x1, (u * u + v * v) <= 1.0, colour))
    return out


def make_image(width: int, height: int, seed: int):
    """RGB uint8 image of blurred ellipses + noise, and the list of ellipse masks."""
    rng = np.random.default_rng(seed)
    img = np.empty((height, width, 3), np.float64)
    img[:] = rng.integers(0, 256, 3)
    ellipses = _ellipse_masks(width, height, rng, N_ELLIPSES)
    for (y0, y1, x0, x1, m, colour) in ellipses:
        if m.size:
            img[y0:y1, x0:x1][m] = colour
    for ch in range(3):
        img[:, :, ch] = ndimage.gaussian_filter(img[:, :, ch], BLUR_SIGMA, mode="nearest",
                                                truncate=4.0)
    img += rng.normal(0.0, NOISE_SIGMA, img.shape)
    img = np.clip(np.floor(img + 0.5), 0, 255).astype(np.uint8)
    return img, ellipses, rng


def _fit_gmm2(x: np.ndarray):
    """Two-component full-covariance Gaussian mixture, ``EM_STEPS`` EM iterations.

    Initialisation splits the samples at the median of their projection on the principal
    axis, so the fit is deterministic.  1.0 is added to each covariance diagonal.
    """
    x = x.astype(np.float64)
    mu = x.mean(0)
    cov = np.cov((x - mu).T) + np.eye(3)
    w_, v_ = np.linalg.eigh(cov)
    proj = (x - mu) @ v_[:, -1]
    resp = np.zeros((x.shape[0], 2))
    resp[proj <= np.median(proj), 0] = 1.0
    resp[:, 1] = 1.0 - resp[:, 0]
    if resp[:, 1].sum() == 0:
        resp[: x.shape[0] // 2] = [0.0, 1.0]
    params = None
    for _ in range(EM_STEPS):
        nk = resp.sum(0) + 1e-9
        weights = nk / nk.sum()
        means = (resp.T @ x) / nk[:, None]
        covs = []
        for k in range(2):
            d = x - means[k]
            covs.append((resp[:, k, None] * d).T @ d / nk[k] + np.eye(3))
        params = (weights, means, np.array(covs))
        logp = _component_logpdf(x, params)
        m = logp.max(1, keepdims=True)
        resp = np.exp(logp - m)
        resp /= resp.sum(1, keepdims=True)
    return params


def _component_logpdf(x: np.ndarray, params):
    """log(w_k N(x | mu_k, S_k)) for k = 0, 1, elementwise (no BLAS reductions), in the
    evaluation form and operation order of gc_tlinks_gmm."""
    comps = components(*params)
    out = np.empty((x.shape[0], 2))
    for k in range(2):
        c, mu, li = comps[k, 0], comps[k, 1:4], comps[k, 4:10]
        d0 = x[:, 0] - mu[0]
        d1 = x[:, 1] - mu[1]
        d2 = x[:, 2] - mu[2]
        y0 = li[0] * d0
        y1 = li[1] * d0 + li[2] * d1
        y2 = li[3] * d0 + li[4] * d1 + li[5] * d2
        out[:, k] = c - 0.5 * (y0 * y0 + y1 * y1 + y2 * y2)
    return out


def _neg_log_likelihood(img: np.ndarray, params, chunk=1 << 20):
    flat = img.reshape(-1, 3)
    out = np.empty(flat.shape[0], np.float64)
    for i in range(0, flat.shape[0], chunk):
        lp = _component_logpdf(flat[i:i + chunk].astype(np.float64), params)
        m = lp.max(1)
        out[i:i + chunk] = -(m + np.log(np.exp(lp[:, 0] - m) + np.exp(lp[:, 1] - m)))
    return out.reshape(img.shape[:2])


def _samples(img, ellipse, rng):
    y0, y1, x0, x1, m, _ = ellipse
    if m.size == 0 or not m.any():
        return img.reshape(-1, 3)[:: max(1, img.shape[0] * img.shape[1] // 1000)]
    s = img[y0:y1, x0:x1][m]
    if s.shape[0] > MAX_FIT_SAMPLES:
        s = s[np.sort(rng.choice(s.shape[0], MAX_FIT_SAMPLES, replace=False))]
    return s


def nlinks(img: np.ndarray):
    """Symmetric n-link weights: (vertical [H-1, W], horizontal [H, W-1]) int32."""
    f = img.astype(np.int64)
    dv = ((f[1:] - f[:-1]) ** 2).sum(-1)
    dh = ((f[:, 1:] - f[:, :-1]) ** 2).sum(-1)
    npairs = dv.size + dh.size
    mean = (dv.sum() + dh.sum()) / max(1, npairs)
    beta = 1.0 / (2.0 * mean) if mean > 0 else 0.0
    wv = np.floor(NLINK_SCALE * np.exp(-beta * dv) + 0.5).astype(np.int32)
    wh = np.floor(NLINK_SCALE * np.exp(-beta * dh) + 0.5).astype(np.int32)
    return wv, wh


def planes_from_weights(wv: np.ndarray, wh: np.ndarray, excess: np.ndarray):
    """Directed capacity planes from symmetric vertical/horizontal edge weights."""
    h, w = excess.shape
    up = np.zeros((h, w), np.int32)
    down = np.zeros((h, w), np.int32)
    left = np.zeros((h, w), np.int32)
    right = np.zeros((h, w), np.int32)
    up[1:] = wv
    down[:-1] = wv
    left[:, 1:] = wh
    right[:, :-1] = wh
    return up, down, left, right


def make_graph(width: int, height: int, seed: int, keep_image=False) -> Graph:
    """Builds the seeded segmentation graph described in the module docstring."""
    img, ellipses, rng = make_image(width, height, seed)
    i_fg, i_bg = rng.choice(len(ellipses), 2, replace=False)
    gmm_fg = _fit_gmm2(_samples(img, ellipses[i_fg], rng))
    gmm_bg = _fit_gmm2(_samples(img, ellipses[i_bg], rng))
    s_fg = _neg_log_likelihood(img, gmm_fg)
    s_bg = _neg_log_likelihood(img, gmm_bg)
    t = np.floor(TLINK_SCALE * (s_bg - s_fg) + 0.5)
    excess = np.clip(t, -TLINK_CLAMP, TLINK_CLAMP).astype(np.int32)
    wv, wh = nlinks(img)
    up, down, left, right = planes_from_weights(wv, wh, excess)
    models = (components(*gmm_fg), components(*gmm_bg)) if keep_image else None
    return Graph(width, height, up, down, left, right, np.ascontiguousarray(excess),
                 img if keep_image else None, models)


def batch_shapes(n: int, seed: int, lo: int = 256, hi: int = 1536, step: int = 128):
    """Independent (width, height) pairs drawn uniformly from {lo, lo+step, ..., hi}."""
    rng = np.random.default_rng(seed)
    sides = np.arange(lo, hi + 1, step)
    return [(int(rng.choice(sides)), int(rng.choice(sides))) for _ in range(n)]


def random_graph(width: int, height: int, seed: int, cap_max=100, tlink_max=2000,
                 sparsity=0.0, symmetric=True) -> Graph:
    """Unstructured random graph (uniform capacities), used by the property tests.

    With ``symmetric=False`` the two directions of every n-link get independent
    capacities (a directed grid), which exercises the reverse-residual bookkeeping.
    """
    rng = np.random.default_rng(seed)
    excess = rng.integers(-tlink_max, tlink_max + 1, (height, width)).astype(np.int32)

    def draw(shape):
        w = rng.integers(0, cap_max + 1, shape).astype(np.int32)
        if sparsity > 0:
            w[rng.random(shape) < sparsity] = 0
        return w

    wv, wh = draw((height - 1, width)), draw((height, width - 1))
    up, down, left, right = planes_from_weights(wv, wh, excess)
    if not symmetric:
        down[:-1] = draw((height - 1, width))
        right[:, :-1] = draw((height, width - 1))
    return Graph(width, height, up, down, left, right, excess)


def _make_one(args):
    w, h, seed, keep = args
    return make_graph(w, h, seed, keep_image=keep)


def make_graphs(specs, processes=None, keep_image=False):
    """make_graph for each (width, height, seed), in a 'spawn' process pool (safe to call
    after CUDA has been initialised in the parent)."""
    import multiprocessing as mp
    import os
    specs = [(w, h, seed, keep_image) for w, h, seed in specs]
    n = processes or min(len(specs), os.cpu_count() or 1)
    if n <= 1 or len(specs) <= 1:
        return [_make_one(s) for s in specs]
    with mp.get_context("spawn").Pool(n) as pool:
        return pool.map(_make_one, specs, chunksize=1)
