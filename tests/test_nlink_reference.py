"""The reference's n-link rule, LAMBDA / (BETA * sqrt(|dRGB|^2) + EPSILON) (weight(),
graphcut.cl:1018-1031; BETA 1.0f/10 graphcut.cl:13; EPSILON 0.05 and LAMBDA 60,
GraphCut.pyx:25-26), rounded to integers for gc_upload_rgba_lambda.  The oracle computes the
rounding exactly with integers; these tests pin it to the reference's own float evaluation
and check the capacity planes it builds."""
import numpy as np
import pytest

from oracle import oracle as O

DMAX = 3 * 255 * 255


def test_every_distance_equals_the_rounded_reference_float_at_lambda_60():
    """At the reference's default LAMBDA every possible |dRGB|^2 gives exactly the rounded
    float32 value the reference's kernel computes."""
    d = np.arange(DMAX + 1)
    w = O.weight_reference(d, 60)
    f = O.weight_reference_float32(d, 60).astype(np.float64)
    assert np.array_equal(w, np.floor(f + 0.5).astype(np.int64))
    assert w[0] == 1200 and w[1] == 400 and w[-1] == 1
    assert np.all(np.diff(w) <= 0)


@pytest.mark.parametrize("lam", [1, 7, 100, 1000])
def test_other_lambdas_differ_from_float_only_at_rounding_ties(lam):
    """For other LAMBDA the exact rounding and the rounded float value agree except where the
    float value lies within float rounding of a half-integer."""
    d = np.unique(np.r_[np.arange(0, 2000), np.linspace(0, DMAX, 4000).astype(np.int64)])
    w = O.weight_reference(d, lam)
    f = O.weight_reference_float32(d, lam).astype(np.float64)
    r = np.floor(f + 0.5).astype(np.int64)
    bad = np.flatnonzero(w != r)
    assert np.all(np.abs(f[bad] - np.floor(f[bad]) - 0.5) < 1e-4 * np.maximum(1, f[bad]))
    assert np.all(np.abs(w - r) <= 1)


def test_exact_rule_matches_its_definition():
    """floor(x + 0.5) with x = 20 lam / (2 sqrt(d) + 1), checked in long double precision away
    from ties, over many (d, lam)."""
    rng = np.random.default_rng(0)
    d = rng.integers(0, DMAX + 1, 3000)
    for lam in (3, 60, 555):
        x = 20.0 * lam / (2.0 * np.sqrt(d.astype(np.longdouble)) + 1.0)
        ref = np.floor(x + 0.5).astype(np.int64)
        w = O.weight_reference(d, lam)
        far = np.abs(x - np.floor(x) - 0.5) > 1e-12
        assert np.array_equal(w[far], ref[far])


def test_planes_of_an_image():
    rng = np.random.default_rng(1)
    img = rng.integers(0, 1 << 24, (9, 13)).astype(np.uint32)
    up, down, left, right = O.nlinks_reference(img, 60)
    assert (up[0] == 0).all() and (down[-1] == 0).all()
    assert (left[:, 0] == 0).all() and (right[:, -1] == 0).all()
    assert np.array_equal(up[1:], down[:-1]) and np.array_equal(left[:, 1:], right[:, :-1])
    def dist(a, b):
        return sum(((int(a) >> s & 255) - (int(b) >> s & 255)) ** 2 for s in (0, 8, 16))
    for y, x in [(3, 4), (8, 12), (1, 0)]:
        assert up[y, x] == O.weight_reference([dist(img[y, x], img[y - 1, x])], 60)[0]
        if x > 0:
            assert left[y, x] == O.weight_reference([dist(img[y, x], img[y, x - 1])], 60)[0]
