"""T-links from colour models, on the CPU: the oracle restatement against the reference's own
score algebra and against the synthetic generator, the evaluation form of a mixture, and the
argument checks of gc_tlinks_gmm (which return before any CUDA call)."""
import ctypes

import numpy as np
import pytest

import synth
from gmm_tlinks import Mixture, components


def _reference_A(weights, means, covars):
    """The reference's diagonal-model coefficients (GMM.calcA_cpu, GMM.pyx:375-395), restated
    here to pin the oracle's score: e = A[0] + A[1:4] . x + A[5:8] . x^2."""
    A = np.empty((len(weights), 8))
    for i in range(len(weights)):
        w = np.log(weights[i])
        h = -0.5 * (3 * np.log(2 * np.pi) + np.sum(np.log(covars[i]))
                    + np.sum(means[i] ** 2 / covars[i]))
        A[i, 0] = w + h
        A[i, 1:4] = means[i] / covars[i]
        A[i, 4] = 0
        A[i, 5:8] = -1 / (2 * covars[i])
    return A


def _reference_score(x, A):
    """score_buf (gmm.cl:434-491) in float64: -(eMax + log(sum exp(e_i - eMax)))."""
    e = A[:, 0][None] + x @ A[:, 1:4].T + (x * x) @ A[:, 5:8].T
    m = e.max(1)
    return -(m + np.log(np.exp(e - m[:, None]).sum(1)))


def _random_model(rng, k, full):
    w = rng.uniform(0.1, 1.0, k)
    w /= w.sum()
    mu = rng.uniform(0, 255, (k, 3))
    if full:
        cov = []
        for _ in range(k):
            a = rng.normal(0, 20, (3, 3))
            cov.append(a @ a.T + np.eye(3) * rng.uniform(5, 50))
        return w, mu, np.array(cov)
    return w, mu, rng.uniform(5, 2000, (k, 3))


@pytest.mark.parametrize("k", [1, 2, 3, 5, 8])
def test_oracle_score_matches_reference_algebra(oracle, k):
    """For diagonal models (the reference's), the oracle's Cholesky-form score equals the
    reference's expanded form up to float64 rounding."""
    from oracle import oracle as O
    rng = np.random.default_rng(k)
    w, mu, cv = _random_model(rng, k, full=False)
    x = rng.integers(0, 256, (5000, 3)).astype(np.float64)
    got = O.mixture_score(x, components(w, mu, cv))
    want = _reference_score(x, _reference_A(w, mu, cv))
    np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("w,h,seed", [(160, 96, 1), (257, 131, 2), (512, 512, 0)])
def test_oracle_equals_generator_excess(oracle, w, h, seed):
    """The generator's t-links are the oracle's on its image and fitted models, bit for bit."""
    from GraphCut import _as_rgba32
    from oracle import oracle as O
    g = synth.make_graph(w, h, seed, keep_image=True)
    fg, bg = g.models
    t, _ = O.tlinks_gmm(_as_rgba32(g.image), fg, bg)
    assert np.array_equal(t, g.excess)


def test_components_diagonal_equals_full():
    rng = np.random.default_rng(4)
    w, mu, cv = _random_model(rng, 3, full=False)
    a = components(w, mu, cv)
    b = components(w, mu, np.stack([np.diag(v) for v in cv]))
    assert np.array_equal(a, b)
    assert a.shape == (3, 10)
    # Li of a diagonal model is diag(1 / sqrt(S_ii)) (up to rounding of the inverse)
    np.testing.assert_allclose(a[:, [4, 6, 9]], 1 / np.sqrt(cv), rtol=1e-15)
    assert np.all(a[:, [5, 7, 8]] == 0)


def test_components_rejects_bad_shapes():
    with pytest.raises(ValueError):
        components([1.0], [[0, 0, 0]], [[1, 1]])
    with pytest.raises(ValueError):
        components(np.ones(9) / 9, np.zeros((9, 3)), np.ones((9, 3)))


def _call(L, rgba, w, h, pitch, fg, nfg, bg, nbg, scale, clamp, out):
    return L.gc_tlinks_gmm(rgba, w, h, pitch, fg, nfg, bg, nbg, scale, clamp, out, None)


@pytest.fixture(scope="module")
def L():
    import os

    import _gcut
    if not os.path.exists(_gcut.LIB_PATH):
        import gcut_build
        gcut_build.build()
    return _gcut.lib()


def test_abi_argument_checks(L):
    import _gcut
    m = Mixture([0.5, 0.5], [[10, 20, 30], [200, 100, 50]], [[100, 100, 100], [50, 60, 70]])
    c = m.as_c()
    dummy = ctypes.c_void_p(16)   # never dereferenced: every call below fails its checks first
    bad = []
    # component counts
    bad.append(_call(L, dummy, 4, 4, 4, c, 0, c, 2, 100.0, 10, dummy))
    bad.append(_call(L, dummy, 4, 4, 4, c, 2, c, 9, 100.0, 10, dummy))
    # pitch, size, scale, clamp
    bad.append(_call(L, dummy, 4, 4, 3, c, 2, c, 2, 100.0, 10, dummy))
    bad.append(_call(L, dummy, -1, 4, 4, c, 2, c, 2, 100.0, 10, dummy))
    bad.append(_call(L, dummy, 4, 4, 4, c, 2, c, 2, float("nan"), 10, dummy))
    bad.append(_call(L, dummy, 4, 4, 4, c, 2, c, 2, 2.0 ** 33, 10, dummy))
    bad.append(_call(L, dummy, 4, 4, 4, c, 2, c, 2, 100.0, -1, dummy))
    bad.append(_call(L, dummy, 4, 4, 4, c, 2, c, 2, 100.0, (1 << 30) + 1, dummy))
    # null model / image / output
    bad.append(_call(L, dummy, 4, 4, 4, None, 2, c, 2, 100.0, 10, dummy))
    bad.append(_call(L, None, 4, 4, 4, c, 2, c, 2, 100.0, 10, dummy))
    bad.append(_call(L, dummy, 4, 4, 4, c, 2, c, 2, 100.0, 10, None))
    # non-finite and out-of-range parameters
    for field, value in (("c", float("inf")), ("c", 2.0 ** 65)):
        cc = m.as_c()
        setattr(cc[1], field, value)
        bad.append(_call(L, dummy, 4, 4, 4, c, 2, cc, 2, 100.0, 10, dummy))
    cc = m.as_c()
    cc[0].li[3] = float("nan")
    bad.append(_call(L, dummy, 4, 4, 4, cc, 2, c, 2, 100.0, 10, dummy))
    cc = m.as_c()
    cc[0].mean[2] = 2.0 ** 33
    bad.append(_call(L, dummy, 4, 4, 4, cc, 2, c, 2, 100.0, 10, dummy))
    assert bad == [_gcut.GC_ERR_INVALID] * len(bad)
    assert b"gc_tlinks_gmm" in L.gc_last_error()


def test_abi_empty_image_is_a_noop(L):
    import _gcut
    c = Mixture([1.0], [[1, 2, 3]], [[4, 5, 6]]).as_c()
    assert _call(L, None, 0, 5, 0, c, 1, c, 1, 100.0, 10, None) == _gcut.GC_OK
    assert _call(L, None, 7, 0, 7, c, 1, c, 1, 100.0, 10, None) == _gcut.GC_OK
