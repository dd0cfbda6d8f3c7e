"""Golden fixtures made from the reference's own score fixtures (scoreFg.npy / scoreBg.npy,
test_GraphCut.py:44-47), see tests/golden/make_golden.py: the oracle still reproduces them
(CPU), and the CUDA solver reproduces them bit for bit through the C ABI (GPU)."""
import os

import numpy as np
import pytest

from golden.make_golden import IMAGE_SEED, TLINK_CLAMP, nlink_planes

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = ["hard", "ragged"]


def load(name):
    z = np.load(os.path.join(HERE, f"scores_{name}.npz"))
    ex = z["excess"]
    h, w = ex.shape
    planes, digest = nlink_planes(h, w, ex)
    assert int(z["image_seed"]) == IMAGE_SEED
    assert digest == str(z["nlinks_sha256"]), "the synthetic image generator changed"
    labels = np.unpackbits(z["labels_packed"], axis=1, bitorder="little", count=w)
    return planes, ex, int(z["flow"]), labels


def test_fixtures_hold_the_hard_constraints():
    _, ex, _, _ = load("hard")
    assert (ex == TLINK_CLAMP).sum() > 0 and (ex == -TLINK_CLAMP).sum() > 0
    _, ex, _, lab = load("ragged")
    assert ex.shape == (131, 257) and 0 < lab.mean() < 1


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_golden(oracle, name):
    (up, down, left, right), ex, flow, labels = load(name)
    f, lab = oracle.maxflow_bk(up, down, left, right, ex)
    assert f == flow and np.array_equal(lab, labels)
    assert oracle.cut_capacity(up, down, left, right, ex, labels) == flow


@pytest.mark.parametrize("name", NAMES)
def test_restated_reference_schedule_gives_the_golden_flow(oracle, name):
    """ref_tiled (GraphCut.cut + graphcut.cl restated) on the fixture padded to whole tiles
    with isolated pixels, which carry no flow."""
    planes, ex, flow, _ = load(name)
    h, w = ex.shape
    ph, pw = -(-h // 32) * 32, -(-w // 32) * 32
    pad = [np.pad(a, ((0, ph - h), (0, pw - w))) for a in (*planes, ex)]
    f, _, _ = oracle.ref_tiled(*pad)
    assert f == flow


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_cuda_reproduces_golden(cuda, name):
    import synth
    from GraphCut import GraphCut
    (up, down, left, right), ex, flow, labels = load(name)
    h, w = ex.shape
    with GraphCut(w, h) as gc:
        gc.upload_capacities(up, down, left, right, ex)
        gc.cut()
        assert gc.flow == flow
        assert np.array_equal(gc.labels_host(), labels)
        # n-links built on the device from the synthetic image the fixture names
        img, _, _ = synth.make_image(w, h, IMAGE_SEED)
        gc.upload_image(img, ex)
        gc.cut()
        assert gc.flow == flow
        assert np.array_equal(gc.labels_host(), labels)
