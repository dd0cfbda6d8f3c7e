"""gc_tlinks_gmm on the GPU: t-links from an image and two colour models equal the oracle's
float64 evaluation, and a graph built entirely on the device (n-links from the image, t-links
from the models) cuts exactly like the generator's planes.

Tolerance: a pixel may differ from the oracle by 1 only where the oracle's unrounded value
scale * (s_bg - s_fg) + 0.5 lies within 1e-9 (relative) of an integer, i.e. where a last-bit
difference between the host's and the device's exp / log can move the floor."""
import numpy as np
import pytest

import synth
from GraphCut import GraphCut, _as_rgba32
from gmm_tlinks import Mixture, components, tlinks

pytestmark = pytest.mark.gpu


def _random_model(rng, k, full):
    w = rng.uniform(0.1, 1.0, k)
    w /= w.sum()
    mu = rng.uniform(0, 255, (k, 3))
    if full:
        cov = []
        for _ in range(k):
            a = rng.normal(0, 20, (3, 3))
            cov.append(a @ a.T + np.eye(3) * rng.uniform(5, 50))
        return components(w, mu, np.array(cov))
    return components(w, mu, rng.uniform(5, 2000, (k, 3)))


def _assert_parity(got, want, v):
    diff = got.astype(np.int64) - want
    bad = diff != 0
    if bad.any():
        tie = np.abs(v - np.round(v)) <= 1e-9 * np.maximum(1.0, np.abs(v))
        assert np.all(np.abs(diff[bad]) == 1) and np.all(tie[bad]), int(bad.sum())
    return int(bad.sum())


@pytest.mark.parametrize("kf,kb,full", [(1, 1, False), (2, 2, True), (3, 2, False),
                                        (4, 4, True), (5, 8, True), (8, 8, False)])
def test_random_models_match_oracle(cuda, oracle, kf, kb, full):
    torch = cuda
    rng = np.random.default_rng(kf * 10 + kb)
    for (w, h) in [(1, 1), (33, 7), (256, 190), (1000, 300)]:
        img = rng.integers(0, 2 ** 32, (h, w), dtype=np.uint64).astype(np.uint32)
        fg, bg = _random_model(rng, kf, full), _random_model(rng, kb, full)
        got = tlinks(torch.from_numpy(img.view(np.int32)).cuda(), fg, bg).cpu().numpy()
        want, v = oracle.tlinks_gmm(img, fg, bg)
        _assert_parity(got, want, v)


def test_pitched_image_clamp_and_scale(cuda, oracle):
    torch = cuda
    rng = np.random.default_rng(9)
    base = rng.integers(0, 2 ** 32, (300, 520), dtype=np.uint64).astype(np.uint32)
    view = torch.from_numpy(base.view(np.int32)).cuda()[:, 7:7 + 411]   # row pitch 520
    assert view.stride(0) == 520 and not view.is_contiguous()
    fg, bg = _random_model(rng, 2, True), _random_model(rng, 3, False)
    for scale, clamp in [(100.0, 10 ** 6), (1e6, 1000), (-3.5, 50), (100.0, 0)]:
        got = tlinks(view, fg, bg, scale=scale, clamp=clamp).cpu().numpy()
        want, v = oracle.tlinks_gmm(base[:, 7:7 + 411], fg, bg, scale=scale, clamp=clamp)
        _assert_parity(got, want, v)
        if clamp == 1000:
            assert (np.abs(want) == 1000).mean() > 0.5   # saturation is exercised


def test_empty_image(cuda):
    torch = cuda
    m = Mixture([1.0], [[0, 0, 0]], [[1, 1, 1]])
    out = tlinks(torch.zeros((0, 16), dtype=torch.int32, device="cuda"), m, m)
    assert out.shape == (0, 16)


@pytest.mark.parametrize("w,h,seed", [(160, 96, 1), (257, 131, 2), (512, 512, 0), (1024, 768, 3)])
def test_generator_graphs_built_on_device(cuda, oracle, w, h, seed):
    """The device t-links equal the generator's, and the graph built from the image and the
    models alone gives the generator's flow and canonical cut."""
    torch = cuda
    g = synth.make_graph(w, h, seed, keep_image=True)
    fg, bg = g.models
    rgba = torch.from_numpy(_as_rgba32(g.image).view(np.int32)).cuda()
    got = tlinks(rgba, fg, bg).cpu().numpy()
    _, v = oracle.tlinks_gmm(_as_rgba32(g.image), fg, bg)
    _assert_parity(got, g.excess, v)
    with GraphCut(w, h) as a, GraphCut(w, h) as b:
        a.upload_image(rgba, (Mixture.from_components(fg), Mixture.from_components(bg)))
        a.cut()
        b.upload_capacities(*g.planes())
        b.cut()
        assert a.flow == b.flow
        assert np.array_equal(a.labels_host(), b.labels_host())
        # from host arrays too
        a.upload_image(g.image, (fg, bg))
        a.cut()
        assert a.flow == b.flow
