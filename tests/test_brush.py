"""The reference brush's pixel set (Brush.points, brush.pyx:138-161: skimage's line and circle
rasterisers) restated in the oracle, checked on hand-worked cases."""
import numpy as np

from oracle import oracle as O


def test_line_hand_worked():
    # (0,0) -> (2,5): dr 2, dc 5, d starts at -1; the minor axis steps before columns 2 and 4
    rr, cc = O.bresenham_line(0, 0, 2, 5)
    assert list(zip(rr.tolist(), cc.tolist())) == [(0, 0), (0, 1), (1, 2), (1, 3), (2, 4), (2, 5)]
    # steep and backwards: (5,1) -> (0,0): rows step -1, the column steps once, at d >= 0
    rr, cc = O.bresenham_line(5, 1, 0, 0)
    assert list(zip(rr.tolist(), cc.tolist())) == [(5, 1), (4, 1), (3, 1), (2, 0), (1, 0), (0, 0)]
    # a tie (dr/dc = 1/2 exactly at the midpoint) moves the minor axis: d == 0 steps
    rr, cc = O.bresenham_line(0, 0, 1, 2)
    assert list(zip(rr.tolist(), cc.tolist())) == [(0, 0), (1, 1), (1, 2)]
    # a single point
    rr, cc = O.bresenham_line(3, 4, 3, 4)
    assert rr.tolist() == [3] and cc.tolist() == [4]


def test_disk_hand_worked():
    def pts(R):
        dr, dc = O.disk_offsets(R)
        return set(zip(dr.tolist(), dc.tolist()))
    assert pts(1) == {(0, 0)}
    assert pts(2) == {(a, b) for a in (-1, 0, 1) for b in (-1, 0, 1)}        # (0, 2): 1.0
    assert pts(3) == {(a, b) for a in range(-2, 3) for b in range(-2, 3)}    # 8 < 9
    assert len(pts(4)) == 49 - 4                                             # (3, 3): 18
    p5 = pts(5)
    assert (3, 4) not in p5 and (4, 3) not in p5 and (4, 2) in p5           # 3-4-5 sums to 1.0
    assert (0, 4) in p5 and (0, 5) not in p5


def test_brush_single_point_and_segment():
    W, H = 20, 12
    # one point: the disc around it
    got = O.brush_pixels([5], [6], 2, W, H)
    want = sorted((6 + a) * W + 5 + b for a in (-1, 0, 1) for b in (-1, 0, 1))
    assert got.tolist() == want
    # a segment with radius 1: exactly its line pixels
    got = O.brush_pixels([0, 5], [0, 2], 1, W, H)
    assert got.tolist() == sorted(r * W + c for r, c in
                                  [(0, 0), (0, 1), (1, 2), (1, 3), (2, 4), (2, 5)])
    # the disc is centred on the line (the reference's +radius shift is not reproduced)
    got = set(O.brush_pixels([4, 4], [4, 4], 2, W, H).tolist())
    assert 3 * W + 3 in got and 5 * W + 5 in got and 6 * W + 6 not in got


def test_brush_clips_to_the_image():
    W, H = 10, 8
    got = O.brush_pixels([0, 9], [0, 0], 3, W, H)
    ys, xs = np.divmod(got, W)
    assert ys.min() == 0 and ys.max() == 2 and xs.min() == 0 and xs.max() == 9
    assert got.size == 3 * 10     # rows 0..2 over the whole width, nothing wrapped
    assert O.brush_pixels([50], [50], 4, W, H).size == 0
    # radius <= 0 counts as 1
    assert O.brush_pixels([3], [3], 0, W, H).tolist() == [33]
