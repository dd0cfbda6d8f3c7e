"""CPU oracle wrapper.  TEST INFRASTRUCTURE ONLY.

The parity tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use
this module to check results; the product never imports it.

* ``maxflow_bk``      exact max-flow (Boykov-Kolmogorov, TPAMI 2004), canonical labels.
* ``ref_tiled``       int32 restatement of the reference schedule (GraphCut.pyx:348-418 +
                      graphcut.cl), OpenMP over tiles; the CPU baseline.
* ``canonical``       canonical cut + flow of a residual state.
* ``cut_capacity``    capacity of a labelled cut from the original capacities.
* ``exclusive_scan``, ``compact``, ``flag``, ``flag_logical``, ``increment_logical``:
  restatements of prefixsum.cl (exclusive Blelloch scan, total in a separate word),
  streamcompact.cl:1-14 (``out[scan[i]] = i`` for flagged i) and
  incremental_tile_list.cl:40-154 (stamp predicates).  Pinned by the reference's own
  known-answer checks (test_PrefixSum.py:35, test_StreamCompact.py:40-41,
  test_IncrementalTileList.py:38-40) in tests/test_oracle.py.
* ``gmm_fit``         EM fit of a colour model (GMM.fit, GMM.pyx:165-372; gmm.cl:33-372).
* ``tlinks_gmm``      t-links from a foreground and a background colour model (GMM.score,
                      gmm.cl:373-491, and scoreBg - scoreFg, test_GraphCut.py:44-47).
* ``nlinks_reference`` the reference's n-link rule (weight(), graphcut.cl:1018-1031, with
                      LAMBDA / EPSILON of GraphCut.pyx:25-26) rounded to integers, in exact
                      integer arithmetic; ``weight_reference_float32`` is the reference's own
                      float evaluation it is pinned against.
* ``brush_pixels``    the pixel set of a brush stroke (brush.pyx:138-161).
* ``view_colorize``   the display filters' colour ramp and blend (graphcut_filter.cl:5-155).

``oracle/refcl.py`` runs the reference's own kernels, compiled for the host, under its host
code: graphcut.cl (``tests/test_refcl_golden.py`` pins ``maxflow_bk`` and ``ref_tiled`` to
it) and prefixsum.cl / streamcompact.cl (``tests/test_refcl_scan.py`` pins
``exclusive_scan`` and ``compact``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

OPERATOR_EQUAL, OPERATOR_GT, OPERATOR_LT, OPERATOR_GTE, OPERATOR_LTE = range(5)
LOGICAL_AND, LOGICAL_OR = 0, 1


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = ctypes.CDLL(path)
        P = ctypes.c_void_p
        _LIB.orc_maxflow_bk.argtypes = [ctypes.c_int, ctypes.c_int] + [P] * 5 + [P, P, P]
        _LIB.orc_canonical.argtypes = [ctypes.c_int, ctypes.c_int] + [P] * 6 + [P, P]
        _LIB.orc_cut_capacity.argtypes = [ctypes.c_int, ctypes.c_int] + [P] * 6
        _LIB.orc_cut_capacity.restype = ctypes.c_int64
        _LIB.orc_ref_tiled.argtypes = ([ctypes.c_int, ctypes.c_int] + [P] * 5 +
                                       [ctypes.c_int, ctypes.c_longlong, ctypes.c_int, P, P, P])
    return _LIB


_NATIVE = None


def native_lib():
    """The oracle built with -O3 -march=native for the host that runs it (compiled into a
    temporary directory on first use, so a build never travels to another CPU), for timing
    the CPU baseline; None when the compiler is unavailable."""
    global _NATIVE
    if _NATIVE is None:
        import tempfile
        out = os.path.join(tempfile.mkdtemp(prefix="gcut_oracle_"), "liboracle_native.so")
        cmd = ["g++", "-O3", "-march=native", "-fopenmp", "-fPIC", "-std=c++17", "-shared",
               "-o", out, os.path.join(_HERE, "gc_oracle.cpp")]
        try:
            subprocess.run(cmd, check=True, capture_output=True, timeout=300)
        except (OSError, subprocess.SubprocessError):
            _NATIVE = False
            return None
        L = ctypes.CDLL(out)
        P = ctypes.c_void_p
        L.orc_ref_tiled.argtypes = ([ctypes.c_int, ctypes.c_int] + [P] * 5 +
                                    [ctypes.c_int, ctypes.c_longlong, ctypes.c_int, P, P, P])
        _NATIVE = L
    return _NATIVE or None


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def maxflow_bk(up, down, left, right, excess, return_excess=False):
    """Exact max-flow of the grid graph: (flow:int, labels:uint8[H,W][, final excess])."""
    up, down, left, right, excess = map(_i32, (up, down, left, right, excess))
    h, w = excess.shape
    flow = np.zeros(1, np.int64)
    labels = np.zeros((h, w), np.uint8)
    fe = np.zeros((h, w), np.int64) if return_excess else None
    rc = lib().orc_maxflow_bk(w, h, _p(up), _p(down), _p(left), _p(right), _p(excess),
                              _p(flow), _p(labels), _p(fe) if fe is not None else None)
    if rc != 0:
        raise RuntimeError(f"orc_maxflow_bk failed ({rc})")
    return (int(flow[0]), labels, fe) if return_excess else (int(flow[0]), labels)


def ref_tiled(up, down, left, right, excess, bfs=5, max_iters=10 ** 7, threads=0,
              native=False):
    """The reference schedule restated: (flow, labels, stats[iterations, relabels, bfs]).
    native=True runs the -march=native build (native_lib) when it is available."""
    up, down, left, right, excess = map(_i32, (up, down, left, right, excess))
    h, w = excess.shape
    flow = np.zeros(1, np.int64)
    labels = np.zeros((h, w), np.uint8)
    stats = np.zeros(3, np.int64)
    L = (native_lib() if native else None) or lib()
    rc = L.orc_ref_tiled(w, h, _p(up), _p(down), _p(left), _p(right), _p(excess), bfs,
                         max_iters, threads, _p(flow), _p(labels), _p(stats))
    if rc != 0:
        raise RuntimeError(f"orc_ref_tiled failed ({rc})")
    return int(flow[0]), labels, stats


def canonical(rup, rdown, rleft, rright, exc, t0):
    rup, rdown, rleft, rright, exc, t0 = map(_i32, (rup, rdown, rleft, rright, exc, t0))
    h, w = exc.shape
    flow = np.zeros(1, np.int64)
    labels = np.zeros((h, w), np.uint8)
    lib().orc_canonical(w, h, _p(rup), _p(rdown), _p(rleft), _p(rright), _p(exc), _p(t0),
                        _p(flow), _p(labels))
    return int(flow[0]), labels


def cut_capacity(up, down, left, right, excess, labels):
    up, down, left, right, excess = map(_i32, (up, down, left, right, excess))
    labels = np.ascontiguousarray(labels, dtype=np.uint8)
    h, w = excess.shape
    return int(lib().orc_cut_capacity(w, h, _p(up), _p(down), _p(left), _p(right), _p(excess),
                                      _p(labels)))


# --- data-parallel primitives beneath IncrementalTileList --------------------------------

def exclusive_scan(a):
    """prefixsum.cl: exclusive scan of int32 values and the total (int32 wrap-around)."""
    a = np.asarray(a, dtype=np.int64)
    out = np.zeros(a.shape[0], np.int64)
    if a.shape[0]:
        np.cumsum(a[:-1], out=out[1:])
    total = int(a.sum())
    wrap = lambda v: ((v + 2 ** 31) % 2 ** 32) - 2 ** 31
    return wrap(out).astype(np.int32), int(wrap(np.int64(total)))


def compact(flags):
    """StreamCompact.compact: ids of the non-zero flags in increasing order, and count."""
    ids = np.flatnonzero(np.asarray(flags) != 0).astype(np.int32)
    return ids, int(ids.shape[0])


def _pred(op, v, operand):
    v = np.asarray(v, dtype=np.int64)
    return {OPERATOR_EQUAL: v == operand, OPERATOR_GT: v > operand, OPERATOR_LT: v < operand,
            OPERATOR_GTE: v >= operand, OPERATOR_LTE: v <= operand}[op]


def flag(tiles, op, operand):
    """incremental_tile_list.cl:40-64."""
    return _pred(op, tiles, operand).astype(np.int32)


def flag_logical(t1, t2, op1, op2, a1, a2, logical):
    """incremental_tile_list.cl:66-108."""
    f1, f2 = _pred(op1, t1, a1), _pred(op2, t2, a2)
    return ((f1 & f2) if logical == LOGICAL_AND else (f1 | f2)).astype(np.int32)


def increment_logical(t1, t2, op1, op2, a1, a2, logical, iteration):
    """incremental_tile_list.cl:110-154: stamp ``iteration`` where the predicate holds."""
    out = np.array(t1, dtype=np.int32, copy=True)
    out[flag_logical(t1, t2, op1, op2, a1, a2, logical) != 0] = iteration
    return out


# --- t-links from colour models (GMM.score + scoreBg - scoreFg) --------------------------

def mixture_score(x, comps):
    """-log sum_k w_k N(x | mean_k, S_k) per row of x (float64 [n, 3] colours), restating
    score_buf / score_img2d (gmm.cl:373-491: e_k per component, eMax, -(eMax + log(sum
    exp(e_k - eMax)))) with full covariances.  ``comps`` [K, 10] rows (c, mean[3], li[6]):
    e_k = c - 0.5 * ((y0 y0 + y1 y1) + y2 y2), y = Li (x - mean), evaluated left to right
    with one rounding per operation (numpy applies no fused multiply-add)."""
    comps = np.asarray(comps, np.float64).reshape(-1, 10)
    e = np.empty((x.shape[0], comps.shape[0]))
    for k, row in enumerate(comps):
        c, mu, li = row[0], row[1:4], row[4:10]
        d0, d1, d2 = x[:, 0] - mu[0], x[:, 1] - mu[1], x[:, 2] - mu[2]
        y0 = li[0] * d0
        y1 = li[1] * d0 + li[2] * d1
        y2 = (li[3] * d0 + li[4] * d1) + li[5] * d2
        e[:, k] = c - 0.5 * ((y0 * y0 + y1 * y1) + y2 * y2)
    m = e.max(1)
    s = np.exp(e[:, 0] - m)
    for k in range(1, e.shape[1]):
        s = s + np.exp(e[:, k] - m)
    return -(m + np.log(s))


def tlinks_gmm(rgba, fg, bg, scale=100.0, clamp=10 ** 6):
    """int32 excess = clamp(floor(scale * (s_bg - s_fg) + 0.5), -clamp, clamp), the
    reference's ``hSink - hSrc`` (test_GraphCut.py:44-47) in the solver's integer units, for
    a uint32 [H, W] image (R in bits 0-7, G 8-15, B 16-23).  Also returns the unrounded
    ``scale * (s_bg - s_fg) + 0.5`` (float64 [H, W]) so that a test can tell rounding ties."""
    img = np.asarray(rgba).view(np.uint32)
    h, w = img.shape
    p = img.reshape(-1)
    x = np.stack([(p & 0xFF), (p >> 8) & 0xFF, (p >> 16) & 0xFF], 1).astype(np.float64)
    v = scale * (mixture_score(x, bg) - mixture_score(x, fg)) + 0.5
    t = np.clip(np.floor(v), -clamp, clamp).astype(np.int32)
    return t.reshape(h, w), v.reshape(h, w)


def tiles_view(tiles, tile_w, tile_h, iteration, width, height):
    """incremental_tile_list.cl:156-175 (filter): uint32 [height, width], 0xFF0000FF where the
    pixel's tile stamp equals ``iteration``, else 0xFF000000; pixels outside the tile grid are
    black."""
    tiles = np.asarray(tiles, np.int32)
    th, tw = tiles.shape
    ty = np.arange(height)[:, None] // tile_h
    tx = np.arange(width)[None, :] // tile_w
    inside = (ty < th) & (tx < tw)
    on = np.zeros((height, width), bool)
    if th and tw:
        stamp = tiles[np.minimum(ty, th - 1), np.minimum(tx, tw - 1)]
        on = inside & (stamp == iteration)
    return np.where(on, np.uint32(0xFF0000FF), np.uint32(0xFF000000)).astype(np.uint32)


# --- colour-model fit (GMM.fit) ----------------------------------------------------------

def _colours(samples):
    p = np.asarray(samples).view(np.uint32).reshape(-1)
    return np.stack([p & 0xFF, (p >> 8) & 0xFF, (p >> 16) & 0xFF], 1).astype(np.float64)


def _log_joint(x, w, mu, S):
    """log(w_k N(x | mu_k, S_k)) for every sample and component (float64 [n, K])."""
    e = np.empty((x.shape[0], len(w)))
    for k in range(len(w)):
        L = np.linalg.cholesky(S[k])
        y = np.linalg.solve(L, (x - mu[k]).T)
        logdet = 2.0 * np.log(np.diag(L)).sum()
        with np.errstate(divide="ignore"):
            e[:, k] = np.log(w[k]) - 0.5 * (3 * np.log(2 * np.pi) + logdet) - 0.5 * (y * y).sum(0)
    return e


def gmm_fit(samples, n_components, max_iterations, tolerance=0.01, min_covar=1e-3,
            init_covar=30.0, full=False):
    """EM restating GMM.fit (GMM.pyx:165-372) with initA / em1 / em2 / eval /
    check_converge (gmm.cl:33-372) in float64: means start at the colours of samples
    k (n - 1) / (K - 1), covariances at init_covar I, weights 1/K; each iteration takes the
    responsibilities under the current model, then N_k = sum r, w = N / sum N,
    mean = sum r x / N, S = sum r x x^T / N - mean mean^T + min_covar I (diagonal unless
    ``full``); L_i, the log-likelihood under the model of iteration i, stops the loop when
    i > 1 and |L_i - L_{i-1}| < tolerance.  (initA reads green through the mask 0xFF0,
    gmm.cl:54; the green byte is used here.)  Returns a dict: weights [K], means [K, 3],
    covars [K, 3, 3], iterations, converged, log_likelihood."""
    x = _colours(samples)
    n, K = x.shape[0], n_components
    idx = [k * (n - 1) // (K - 1) for k in range(K)] if K > 1 else [0]
    w = np.full(K, 1.0 / K)
    mu = x[idx].copy()
    S = np.stack([np.eye(3) * init_covar for _ in range(K)])
    lprev, t, converged = 0.0, 0, False
    while True:
        e = _log_joint(x, w, mu, S)
        m = e.max(1)
        lpr = m + np.log(np.exp(e - m[:, None]).sum(1))
        L = float(lpr.sum())
        stop = False
        if t >= 1:
            if t - 1 > 1 and abs(L - lprev) < tolerance:
                stop = converged = True
            lprev = L
        if not stop and t == max_iterations:
            stop = True
        if stop:
            return {"weights": w, "means": mu, "covars": S, "iterations": t,
                    "converged": converged, "log_likelihood": L}
        r = np.exp(e - lpr[:, None])
        nk = r.sum(0)
        for k in range(K):
            if not nk[k] > 0:
                w[k] = 0.0
                continue
            w[k] = nk[k] / nk.sum()
            mu[k] = (r[:, k] @ x) / nk[k]
            c = (r[:, k, None] * x).T @ x / nk[k] - np.outer(mu[k], mu[k])
            S[k] = (c if full else np.diag(np.diag(c))) + min_covar * np.eye(3)
        t += 1


# ---- n-links of the reference (graphcut.cl:1018-1031) ------------------------------------
REF_BETA = np.float32(1.0) / np.float32(10.0)   # #define BETA 1.0f/10 (graphcut.cl:13)
REF_EPSILON = 0.05                             # DEF EPSILON = 0.05 (GraphCut.pyx:26)
REF_LAMBDA = 60                                # DEF LAMDA_DEFAULT = 60 (GraphCut.pyx:25)


def weight_reference_float32(d, lam=REF_LAMBDA):
    """The reference's capacity LAMBDA * weight(c1, c2) for |dRGB|^2 = d, evaluated as its
    OpenCL C does: sqrt of the float distance, times BETA (float), plus EPSILON (a double
    literal, so the sum and the reciprocal are double), the reciprocal rounded to float, then
    times LAMBDA in float (graphcut.cl:1030, :1089)."""
    d = np.asarray(d)
    s = np.sqrt(d.astype(np.float32))                       # float sqrt
    den = (REF_BETA * s).astype(np.float64) + REF_EPSILON   # float * float + double
    w = (1.0 / den).astype(np.float32)                      # returned as float
    return (np.float32(lam) * w).astype(np.float32)


def weight_reference(d, lam=REF_LAMBDA):
    """That weight rounded to the nearest integer, halves up, computed exactly:
    x = lam / (0.1 sqrt(d) + 0.05) = 20 lam / (2 sqrt(d) + 1), and for k >= 1
    floor(x + 0.5) >= k  <=>  b = 40 lam - 2k + 1 >= 0 and 4 (2k - 1)^2 d <= b^2.
    Python integers, one distinct distance at a time."""
    d = np.asarray(d, dtype=np.int64)
    out = np.empty(d.shape, np.int64)
    cache = {}
    a40 = 40 * int(lam)

    def ok(k, dd):
        if k < 1:
            return True
        b, a = a40 - 2 * k + 1, 2 * k - 1
        return b >= 0 and 4 * a * a * dd <= b * b

    flat = out.reshape(-1)
    for i, dd in enumerate(d.reshape(-1).tolist()):
        w = cache.get(dd)
        if w is None:
            # the largest k with ok(k): ok is monotone in k, bisect over [0, 20 lam]
            lo, hi = 0, 20 * int(lam)
            while lo < hi:
                mid = (lo + hi + 1) // 2
                if ok(mid, dd):
                    lo = mid
                else:
                    hi = mid - 1
            w = cache[dd] = lo
        flat[i] = w
    return out


def _dist2(a, b):
    a = a.astype(np.int64)
    b = b.astype(np.int64)
    return sum(((a >> s & 255) - (b >> s & 255)) ** 2 for s in (0, 8, 16))


def nlinks_reference(rgba, lam=REF_LAMBDA):
    """Capacity planes (up, down, left, right) of an RGBA image (uint32 [H, W], R in the low
    byte) under the reference's weighting rounded as ``weight_reference``: every 4-neighbour
    pair gets its weight in both directions and capacities pointing out of the image are 0
    (load_tiles, graphcut.cl:1033-1132, without its last-row/column and right-border bugs)."""
    img = np.asarray(rgba).astype(np.uint32)
    H, W = img.shape
    wv = weight_reference(_dist2(img[1:], img[:-1]), lam).astype(np.int32)    # (y, y-1) pairs
    wh = weight_reference(_dist2(img[:, 1:], img[:, :-1]), lam).astype(np.int32)
    up = np.zeros((H, W), np.int32)
    down = np.zeros((H, W), np.int32)
    left = np.zeros((H, W), np.int32)
    right = np.zeros((H, W), np.int32)
    up[1:] = wv
    down[:-1] = wv
    left[:, 1:] = wh
    right[:, :-1] = wh
    return up, down, left, right


# ---- the reference brush (brush.pyx:138-161) ---------------------------------------------
def bresenham_line(r0, c0, r1, c1):
    """Pixels (rows, cols) of the segment from (r0, c0) to (r1, c1) as skimage.draw.line
    produces them (Bresenham with the error term d = 2 dr - dc, a step of the minor axis
    while d >= 0, and the end point appended), the rasteriser brush.pyx:150 calls."""
    r, c = int(r0), int(c0)
    dr, dc = abs(int(r1) - r), abs(int(c1) - c)
    sc = 1 if int(c1) - c > 0 else -1
    sr = 1 if int(r1) - r > 0 else -1
    steep = dr > dc
    if steep:
        r, c = c, r
        dr, dc = dc, dr
        sr, sc = sc, sr
    d = 2 * dr - dc
    rr, cc = [], []
    for _ in range(dc):
        if steep:
            rr.append(c)
            cc.append(r)
        else:
            rr.append(r)
            cc.append(c)
        while d >= 0:
            r += sr
            d -= 2 * dc
        c += sc
        d += 2 * dr
    rr.append(int(r1))
    cc.append(int(c1))
    return np.array(rr, np.int64), np.array(cc, np.int64)


def disk_offsets(radius):
    """Offsets (dr, dc) of skimage.draw.circle(0, 0, radius): the integer points with
    (dr / radius)^2 + (dc / radius)^2 < 1, evaluated in float64 as skimage's ellipse test
    does (brush.pyx:147, :151)."""
    R = int(radius)
    o = np.arange(-R, R + 1, dtype=np.float64)
    a = (o / float(R)) ** 2
    inside = (a[:, None] + a[None, :]) < 1.0
    dr, dc = np.nonzero(inside)
    return dr - R, dc - R


def brush_pixels(xs, ys, radius, width, height):
    """Flat indices (y * width + x, increasing) of the pixels the reference Brush covers for
    the polyline (xs[i], ys[i]) (Brush.points, brush.pyx:138-161): one point gives the disc
    circle(y, x, radius) around it; each segment gives its line pixels, each widened by the
    disc offsets.  radius <= 0 counts as 1 (Brush.setRadius).  Two reference bugs are fixed:
    the segment disc is centred on each line pixel (the reference adds the pixels of
    circle(radius, radius, radius), i.e. offsets shifted by +radius in x and y), and pixels
    outside the image are dropped (the reference's y * width + x wraps them into other rows or
    out of the buffer)."""
    R = max(1, int(radius))
    odr, odc = disk_offsets(R)
    xs = [int(v) for v in xs]
    ys = [int(v) for v in ys]
    pts_r, pts_c = [], []
    if len(xs) == 1:
        pts_r.append(np.array([ys[0]]))
        pts_c.append(np.array([xs[0]]))
    for k in range(len(xs) - 1):
        lr, lc = bresenham_line(ys[k], xs[k], ys[k + 1], xs[k + 1])
        pts_r.append(lr)
        pts_c.append(lc)
    lr = np.concatenate(pts_r)
    lc = np.concatenate(pts_c)
    yy = (lr[:, None] + odr[None, :]).reshape(-1)
    xx = (lc[:, None] + odc[None, :]).reshape(-1)
    keep = (yy >= 0) & (yy < height) & (xx >= 0) & (xx < width)
    return np.unique(yy[keep] * width + xx[keep])


def view_colorize(values, cell_w, cell_h, width, height, ramp, base=None):
    """The display layer of graphcut_filter.cl:5-155 (colorizef, HSVtoRGB, and the blend of the
    tranpose / tilelist kernels) in float32, each operation rounded as the device does it (no
    fused multiply-add).  Sector 4 of the hue circle repeats sector 5's (v, p, q) as
    HSVtoRGB (graphcut_filter.cl:17-22) does; below the range is tested before above it
    (colorizef, :32-35); a range of one value maps it to the ramp's start (the reference
    divides 0 by 0 there).  values: int32 [rows, cols] cells; ramp: range lo, hi, hue lo,
    hi, saturation lo, hi, value lo, hi, opacity; base: uint32 RGBA words [height, width] or
    None.  Returns uint32 RGBA words [height, width], R in the low byte."""
    f32 = np.float32
    values = np.asarray(values, dtype=np.int32)
    rows, cols = values.shape
    lo, hi, h0, h1, s0, s1, v0, v1, op = [f32(x) for x in ramp]
    base = np.zeros((height, width), np.uint32) if base is None else \
        np.asarray(base).view(np.uint32).reshape(height, width)
    ys, xs = np.mgrid[0:height, 0:width]
    cx, cy = xs // cell_w, ys // cell_h
    inside = (cx < cols) & (cy < rows)
    v = np.zeros((height, width), f32)
    v[inside] = values[cy[inside], cx[inside]].astype(f32)
    H = np.zeros_like(v)
    S = np.zeros_like(v)
    V = np.zeros_like(v)
    below = v < lo
    above = ~below & (v > hi)
    mid = ~below & ~above
    V[above] = f32(1)
    with np.errstate(all="ignore"):
        t = (v - lo) / (hi - lo) if hi > lo else np.zeros_like(v)
    t = t.astype(f32)
    for arr, a, b in ((H, h0, h1), (S, s0, s1), (V, v0, v1)):
        arr[mid] = (a + t * (b - a)).astype(f32)[mid]
    h6 = (H * f32(6)).astype(f32)
    sector = np.trunc((h6 - f32(1e-6)).astype(f32)).astype(np.int64)
    f = (h6 - sector.astype(f32)).astype(f32)
    p = (V * (f32(1) - S)).astype(f32)
    q = (V * (f32(1) - S * f)).astype(f32)
    u = (V * (f32(1) - S * (f32(1) - f))).astype(f32)
    rgb = np.zeros((3, height, width), f32)
    table = {0: (V, u, p), 1: (q, V, p), 2: (p, V, u), 3: (p, q, V)}
    lit = V != 0
    for sec, chans in table.items():
        m = (sector == sec) & lit
        for k in range(3):
            rgb[k][m] = chans[k][m]
    m = ((sector < 0) | (sector > 3)) & lit     # every other sector: (v, p, q)
    for k, chan in enumerate((V, p, q)):
        rgb[k][m] = chan[m]
    out = np.zeros((height, width), np.uint32)
    for k in range(4):
        cb = ((base >> np.uint32(8 * k)) & np.uint32(0xFF)).astype(f32) / f32(255)
        co = rgb[k] if k < 3 else np.zeros_like(cb)
        c = (cb + (co - cb) * op).astype(f32)
        c = np.clip(c, f32(0), f32(1))
        out |= np.rint(c * f32(255)).astype(np.uint32) << np.uint32(8 * k)
    out[~inside] = base[~inside]
    return out
