"""The n-link table of gc_upload_rgba, restated on the CPU: weight(d) = floor(50 * exp(-beta * d)
+ 0.5) stored as 50 thresholds (the largest d with weight >= k), settled by evaluating the
formula at the integers around the real root.  Looking the weights up in the table must
reproduce the synthetic generator's n-links exactly."""
import math

import numpy as np
import pytest

import synth

DMAX = 3 * 255 * 255


def table(dsum, npairs):
    mean = dsum / max(1, npairs)
    beta = 1.0 / (2.0 * mean) if mean > 0 else 0.0

    def w(d):
        return math.floor(50.0 * math.exp(-beta * float(d)) + 0.5)

    t = []
    for k in range(1, 51):
        if beta <= 0:
            t.append(DMAX)
            continue
        root = math.log(50.0 / (k - 0.5)) / beta
        d = DMAX if root >= DMAX else max(0, math.floor(root))
        while d < DMAX and w(d + 1) >= k:
            d += 1
        while d >= 0 and w(d) < k:
            d -= 1
        t.append(d)
    return np.array(t, np.int64)


def lookup(t, d):
    # number of entries >= d (the entries do not increase with k)
    return (t[None, :] >= d.reshape(-1, 1)).sum(1).reshape(d.shape)


@pytest.mark.parametrize("w,h,seed", [(96, 80, 0), (200, 64, 1), (64, 64, 2), (150, 151, 3)])
def test_table_reproduces_generator(w, h, seed):
    g = synth.make_graph(w, h, seed, keep_image=True)
    f = g.image.astype(np.int64)
    dv = ((f[1:] - f[:-1]) ** 2).sum(-1)
    dh = ((f[:, 1:] - f[:, :-1]) ** 2).sum(-1)
    t = table(int(dv.sum() + dh.sum()), dv.size + dh.size)
    assert np.all(np.diff(t) <= 0)
    wv, wh = synth.nlinks(g.image)
    assert np.array_equal(lookup(t, dv), wv)
    assert np.array_equal(lookup(t, dh), wh)


def test_uniform_image_gives_full_weights():
    t = table(0, 100)
    assert np.all(t == DMAX)
    assert np.all(lookup(t, np.array([0, 5, DMAX])) == 50)


def test_every_distance_against_the_formula():
    """All d in [0, 3 * 255^2] for a few beta values: table lookup == direct formula."""
    d = np.arange(DMAX + 1, dtype=np.int64)
    for dsum, npairs in [(123456789, 1000000), (5, 3), (10**12, 10**7)]:
        t = table(dsum, npairs)
        mean = dsum / npairs
        beta = 1.0 / (2.0 * mean)
        direct = np.floor(50.0 * np.exp(-beta * d) + 0.5).astype(np.int64)
        assert np.array_equal(lookup(t, d), direct)
