"""The headless display layer (gc_view_colorize): the oracle's restatement of the reference's
colour ramp and blend (graphcut_filter.cl:5-155) checked against hand-worked values on the
CPU, and the CUDA kernel checked against the restatement word for word on the GPU."""
import numpy as np
import pytest


def test_ramp_hand_worked(oracle):
    v = np.array([[0, 5, 10, 20, -1]], np.int32)
    out = oracle.view_colorize(v, 1, 1, 5, 1, [0, 10, 0.0, 0.5, 1, 1, 1, 1, 1.0])
    # hue 0 -> red; hue 0.25 -> sector 1 (0.5, 1, 0), 127.5 rounds to even 128; hue 0.5 ->
    # cyan; above the range -> white; below it -> black; alpha 0 at full opacity
    assert [int(x) for x in out.ravel()] == [0x0000FF, 0x00FF80, 0xFFFF00, 0xFFFFFF, 0x000000]


def test_blend_and_sector_four(oracle):
    v = np.array([[7]], np.int32)
    base = np.array([[0xFF204060]], np.uint32)
    # hue 0.7 is sector 4, which the reference's HSVtoRGB gives sector 5's (v, p, q):
    # (1, 0, 1 - 0.2) at full saturation and value
    solid = oracle.view_colorize(v, 1, 1, 1, 1, [0, 10, 0.0, 1.0, 1, 1, 1, 1, 1.0])
    assert int(solid[0, 0]) == (255 | (0 << 8) | (204 << 16))
    # an inverted range: below is tested first, so a value both below lo and above hi is black
    inv = oracle.view_colorize(v, 1, 1, 1, 1, [9, 3, 0.0, 1.0, 1, 1, 1, 1, 1.0])
    assert int(inv[0, 0]) == 0
    # opacity 0 keeps the base; 0.5 goes half way in every channel (alpha towards 0)
    assert int(oracle.view_colorize(v, 1, 1, 1, 1, [0, 10, 0, 1, 1, 1, 1, 1, 0.0], base)[0, 0]) \
        == 0xFF204060
    half = int(oracle.view_colorize(v, 1, 1, 1, 1, [0, 10, 0, 1, 1, 1, 1, 1, 0.5], base)[0, 0])
    assert (half >> 24) & 0xFF == 128   # 255 * 0.5 = 127.5, ties to even -> 128


def test_cells_and_outside(oracle):
    tiles = np.array([[1, 2], [3, 4]], np.int32)
    base = np.full((5, 7), 0x11223344, np.uint32)
    out = oracle.view_colorize(tiles, 3, 2, 7, 5, [0, 4, 0, 0.5, 1, 1, 1, 1, 1.0], base)
    assert out.shape == (5, 7)
    assert len({int(x) for x in out[0:2, 0:3].ravel()}) == 1   # one cell, one colour
    assert (out[:, 6] == 0x11223344).all() and (out[4, :] == 0x11223344).all()   # outside


@pytest.mark.gpu
@pytest.mark.parametrize("cell,width,height", [((1, 1), 257, 130), ((32, 32), 200, 96),
                                               ((16, 16), 64, 64)])
def test_device_matches_restatement(cuda, oracle, cell, width, height):
    torch = cuda
    from views import colorize
    rng = np.random.default_rng(width + height)
    rows, cols = -(-height // cell[1]), -(-width // cell[0])
    values = rng.integers(-50, 350, (rows, cols)).astype(np.int32)
    base = rng.integers(0, 2 ** 32, (height, width), dtype=np.uint64).astype(np.uint32)
    for ramp in ([0, 300, 0.0, 0.7, 1, 1, 1, 1, 0.6], [10, 10, 0.2, 0.9, 0.3, 1, 0.5, 1, 1.0],
                 [-40, 200, 0.95, 0.05, 1, 0.2, 0.1, 1, 0.25]):
        ref = oracle.view_colorize(values, cell[0], cell[1], width, height, ramp, base)
        got = colorize(torch.from_numpy(values).cuda(), width=width, height=height, cell=cell,
                       value_range=ramp[0:2], hues=ramp[2:4], sats=ramp[4:6], vals=ramp[6:8],
                       opacity=ramp[8], base=torch.from_numpy(base.view(np.int32)).cuda())
        assert np.array_equal(got.cpu().numpy().view(np.uint32), ref), ramp


@pytest.mark.gpu
def test_execute_returns_planes_in_image_layout(cuda, oracle):
    torch = cuda
    import synth
    from GraphCut import GraphCut
    g = synth.make_graph(100, 37, 5)
    with GraphCut(100, 37) as gc:
        gc.upload_capacities(*g.planes())
        gc.cut()
        for name, plane in (("height", gc.dHeight), ("left", gc.dLeft), ("excess", gc.dExcess)):
            out = gc.execute(name)
            assert out.dtype == torch.float32 and tuple(out.shape) == (37, 100)
            assert torch.equal(out, plane.to(torch.float32))
            assert torch.equal(gc.execute(plane), out)
        with pytest.raises(ValueError):
            gc.execute("labels")
        # a colour layer of the heights over nothing: the usual display path end to end
        h = gc.dHeight
        rgba = __import__("views").colorize(h, value_range=(0, 40), hues=(0.0, 0.7))
        ref = oracle.view_colorize(h.cpu().numpy(), 1, 1, 100, 37,
                                   [0, 40, 0.0, 0.7, 1, 1, 1, 1, 1.0])
        assert np.array_equal(rgba.cpu().numpy().view(np.uint32), ref)


def test_colorize_rejects_host_values():
    import torch
    from views import colorize
    with pytest.raises(TypeError):
        colorize(torch.zeros((2, 2), dtype=torch.int32))
