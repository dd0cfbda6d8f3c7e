"""Colour-model fit on the CPU: the oracle's EM restatement against scikit-learn's
GaussianMixture (the implementation the reference compares its fit with, test_GMM.py:4)
from the same start, and the argument checks of gc_gmm_fit (which return before any
CUDA call)."""
import ctypes
import warnings

import numpy as np
import pytest

import synth


def stroke_samples(seed, n, w=320, h=240):
    """RGBA words of ``n`` pixels of one ellipse of a synthetic image (a stroke's samples)."""
    from GraphCut import _as_rgba32
    img, ellipses, rng = synth.make_image(w, h, seed)
    rgba = _as_rgba32(img)
    y0, y1, x0, x1, m, _ = max(ellipses, key=lambda e: e[4].sum())
    pix = rgba[y0:y1, x0:x1][m]
    return pix[np.random.default_rng(seed).integers(0, pix.size, n)]


def _sklearn_fit(x, w0, mu0, cov0, iters, min_covar, full):
    from sklearn.mixture import GaussianMixture
    K = len(w0)
    prec = (np.stack([np.linalg.inv(c) for c in cov0]) if full
            else np.stack([1.0 / np.diag(c) for c in cov0]))
    gm = GaussianMixture(K, covariance_type="full" if full else "diag", tol=0.0,
                         reg_covar=min_covar, max_iter=iters, n_init=1, weights_init=w0,
                         means_init=mu0, precisions_init=prec, random_state=0)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        gm.fit(x)
    cov = gm.covariances_ if full else np.stack([np.diag(c) for c in gm.covariances_])
    return gm.weights_, gm.means_, cov


@pytest.mark.parametrize("K,full,iters", [(1, False, 5), (2, False, 30), (4, False, 65),
                                           (2, True, 30), (3, True, 20)])
def test_oracle_matches_sklearn_from_the_same_start(oracle, K, full, iters):
    """With the likelihood test off (tolerance 0), the oracle's model after N iterations is
    scikit-learn's after N iterations from the same start (its reg_covar is min_covar)."""
    from oracle import oracle as O
    s = stroke_samples(K * 10 + iters, 4000)
    x = O._colours(s)
    n = x.shape[0]
    idx = [k * (n - 1) // (K - 1) for k in range(K)] if K > 1 else [0]
    cov0 = np.stack([np.eye(3) * 30.0] * K)
    want = _sklearn_fit(x, np.full(K, 1.0 / K), x[idx], cov0, iters, 1e-3, full)
    got = O.gmm_fit(s, K, iters, tolerance=0.0, full=full)
    assert got["iterations"] == iters and not got["converged"]
    np.testing.assert_allclose(got["weights"], want[0], rtol=1e-7, atol=1e-10)
    np.testing.assert_allclose(got["means"], want[1], rtol=1e-7, atol=1e-7)
    np.testing.assert_allclose(got["covars"], want[2], rtol=1e-6, atol=1e-6)


def test_oracle_likelihood_test_stops_early(oracle):
    from oracle import oracle as O
    s = stroke_samples(7, 10000)
    r = O.gmm_fit(s, 2, 65, tolerance=0.01)
    assert r["converged"] and 3 <= r["iterations"] < 65
    # the same model as running exactly that many iterations without the test
    r2 = O.gmm_fit(s, 2, r["iterations"], tolerance=0.0)
    assert np.array_equal(r["means"], r2["means"]) and r["log_likelihood"] == r2["log_likelihood"]


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
    d = ctypes.c_void_p(16)   # never dereferenced: every call below fails its checks first
    calls = [
        (d, 10, 0, 5, 0.01, 1e-3, 30.0, 0, d),      # no components
        (d, 10, 9, 5, 0.01, 1e-3, 30.0, 0, d),      # too many components
        (d, 3, 4, 5, 0.01, 1e-3, 30.0, 0, d),       # fewer samples than components
        (d, 10, 2, 0, 0.01, 1e-3, 30.0, 0, d),      # no iterations
        (d, 10, 2, 100001, 0.01, 1e-3, 30.0, 0, d),
        (d, 10, 2, 5, -1.0, 1e-3, 30.0, 0, d),      # tolerance
        (d, 10, 2, 5, float("nan"), 1e-3, 30.0, 0, d),
        (d, 10, 2, 5, 0.01, -1e-3, 30.0, 0, d),     # min_covar
        (d, 10, 2, 5, 0.01, 1e-3, 0.0, 0, d),       # init_covar
        (None, 10, 2, 5, 0.01, 1e-3, 30.0, 0, d),   # null samples
        (d, 10, 2, 5, 0.01, 1e-3, 30.0, 0, None),   # null result
    ]
    for c in calls:
        assert L.gc_gmm_fit(*c, None) == _gcut.GC_ERR_INVALID, c
    assert b"gc_gmm_fit" in L.gc_last_error()


def test_result_layout_matches_header():
    import _gcut
    assert ctypes.sizeof(_gcut.GcGmmFitResult) == 8 * (8 + 24 + 48 + 1) + 4 * 4 + 8 * 80


def test_gmm_class_checks():
    from GMM import GMM
    with pytest.raises(ValueError):
        GMM(10, 0)
    with pytest.raises(ValueError):
        GMM(10, 9)
