"""gc_gmm_fit on the GPU: the colour-model fit equals the oracle's float64 EM (same iteration
count and stop, parameters to a relative 1e-7 that allows for the different summation order),
is deterministic, and feeds the device t-links and the solver end to end.

Tolerance: the device sums the samples in a fixed tree (threads, warps, blocks of the cluster)
and numpy in pairwise order, so sums differ in the last bits; EM contracts such differences,
and 65 iterations keep them below 1e-7 relative on these inputs."""
import numpy as np
import pytest

import synth
from GMM import GMM
from test_gmm_fit import stroke_samples

pytestmark = pytest.mark.gpu


def _compare(g, want, full):
    assert g.iterations == want["iterations"]
    assert g.has_converged == want["converged"]
    np.testing.assert_allclose(g.weights, want["weights"], rtol=1e-7, atol=1e-10)
    np.testing.assert_allclose(g.means, want["means"], rtol=1e-7, atol=1e-7)
    cov = want["covars"] if full else np.stack([np.diag(c) for c in want["covars"]])
    np.testing.assert_allclose(g.covars, cov, rtol=1e-7, atol=1e-6)
    np.testing.assert_allclose(g.log_likelihood, want["log_likelihood"], rtol=1e-10)


@pytest.mark.parametrize("K,full,n,iters,tol", [
    (4, False, 10000, 65, 0.01),    # the reference test_GMM.py:58-67: 20x500 samples, 4 comps, 65
    (2, False, 10000, 65, 0.01),    # stops on the likelihood test
    (1, False, 777, 10, 0.01),
    (2, True, 20000, 40, 0.0),
    (3, True, 5000, 30, 0.0),
    (6, False, 3000, 20, 0.0),      # two-pass path (5..8 components)
    (8, True, 4096, 15, 0.0),
    (3, False, 3, 5, 0.0),          # as many samples as components
    (2, False, 300000, 8, 0.0),     # many samples per thread
])
def test_fit_matches_oracle(cuda, oracle, K, full, n, iters, tol):
    s = stroke_samples(K * 100 + n % 97, n)
    g = GMM(iters, K, tolerance=tol, full_covariance=full)
    g.fit(s)
    _compare(g, oracle.gmm_fit(s, K, iters, tolerance=tol, full=full), full)
    # the evaluation form the device returns is that of the returned model
    from gmm_tlinks import components
    keep = g.weights > 0
    np.testing.assert_allclose(g.device_components[keep],
                               components(g.weights[keep], g.means[keep], g.covars[keep]),
                               rtol=1e-9, atol=1e-9)


def test_fit_is_deterministic_and_takes_device_samples(cuda):
    torch = cuda
    s = stroke_samples(5, 50000)
    d = torch.from_numpy(s.view(np.int32)).cuda()
    a = GMM(30, 4, tolerance=0.0, full_covariance=True)
    b = GMM(30, 4, tolerance=0.0, full_covariance=True)
    wa, ma, ca = a.fit(d, retParams=True)
    wb, mb, cb = b.fit(s, retParams=True)
    assert np.array_equal(wa, wb) and np.array_equal(ma, mb) and np.array_equal(ca, cb)
    assert a.log_likelihood == b.log_likelihood
    # nSamples: a prefix of the buffer
    c = GMM(30, 4, tolerance=0.0, full_covariance=True)
    c.fit(d, nSamples=1000)
    e = GMM(30, 4, tolerance=0.0, full_covariance=True)
    e.fit(s[:1000])
    assert np.array_equal(c.means, e.means)


def test_degenerate_covariance_is_reported(cuda):
    """All samples one colour and no covariance floor: the covariance becomes 0, the fit stops
    with status 1 and the class raises."""
    import _gcut
    s = np.full(500, 0xFF102030, np.uint32)
    g = GMM(10, 1, min_covar=0.0)
    with pytest.raises(_gcut.GCError) as ei:
        g.fit(s)
    assert ei.value.code == _gcut.GC_ERR_NOT_CONVERGED
    np.testing.assert_array_equal(g.means[0], [0x30, 0x20, 0x10])


def test_fit_then_tlinks_then_cut(cuda, oracle):
    """The interactive pipeline on the device: fit a foreground and a background model to
    the pixels of two ellipses, score the image, solve; checked against the oracle's t-links
    of the same models and the exact max-flow."""
    from GraphCut import GraphCut, _as_rgba32
    from gmm_tlinks import tlinks
    torch = cuda
    w, h = 400, 300
    img, ellipses, _ = synth.make_image(w, h, 11)
    rgba = _as_rgba32(img)
    big = sorted(ellipses, key=lambda e: -e[4].sum())[:2]
    models = []
    for (y0, y1, x0, x1, m, _) in big:
        g = GMM(65, 2, full_covariance=True)
        g.fit(rgba[y0:y1, x0:x1][m])
        models.append(g.mixture())
    d_img = torch.from_numpy(rgba.view(np.int32)).cuda()
    ex = tlinks(d_img, models[0], models[1]).cpu().numpy()
    want, v = oracle.tlinks_gmm(rgba, models[0].comps, models[1].comps)
    bad = ex != want
    if bad.any():
        tie = np.abs(v - np.round(v)) <= 1e-9 * np.maximum(1.0, np.abs(v))
        assert np.all(np.abs(ex[bad].astype(np.int64) - want[bad]) == 1) and np.all(tie[bad])
    with GraphCut(w, h) as gc:
        gc.upload_image(d_img, (models[0], models[1]))
        gc.cut()
        wv, wh = synth.nlinks(img)
        planes = synth.planes_from_weights(wv, wh, ex)
        f, lab = oracle.maxflow_bk(*planes, ex)
        assert gc.flow == f
        assert np.array_equal(gc.labels_host(), lab)
