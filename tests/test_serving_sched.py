"""Serving scheduler on the CPU: a fake solver stands in for the device, so admission,
eviction, per-session ordering, slot reservation and misses are checked without a GPU.

The fake session state is the running sum of the t-link plane plus every stroke value
applied to it, so a result proves which requests its handle has seen, in which order."""
import threading
import time

import numpy as np
import pytest

from serving import ALIGN, GraphCutServer, NewImage, Slab, Stroke, session_bytes


class FakeHandle:
    def __init__(self, w, h, off, nbytes, live):
        self.w, self.h = w, h
        self.state = None
        self.running = False
        self.closed = False
        self.range = (off, off + nbytes)
        self.live = live
        for o in live:   # no two live handles share slab bytes
            assert o.range[1] <= self.range[0] or self.range[1] <= o.range[0]
        live.add(self)

    def close(self):
        self.closed = True
        self.live.discard(self)


class FakeContext:
    def __init__(self, srv):
        self.srv = srv
        self.rng = np.random.default_rng(threading.get_ident() % 1000)

    def _enter(self, gc):
        assert not gc.running, "two requests on one handle at once"
        assert not gc.closed, "a closed handle was used"
        gc.running = True
        time.sleep(float(self.rng.uniform(0, 0.002)))

    def run_image(self, gc, planes, w, h):
        with self.srv.lock:
            self.srv.images_running += 1
            self.srv.max_images_running = max(self.srv.max_images_running,
                                              self.srv.images_running)
        self._enter(gc)
        gc.state = int(planes[4].sum())
        gc.running = False
        with self.srv.lock:
            self.srv.images_running -= 1
        return gc.state, np.zeros((h, (w + 7) // 8), np.uint8), (0.0, 0.0, 0.0)

    def run_stroke(self, gc, req, w, h):
        self._enter(gc)
        gc.state += int(req.value)
        gc.running = False
        return gc.state, np.zeros((h, (w + 7) // 8), np.uint8), (0.0, 0.0, 0.0)


class FakeServer(GraphCutServer):
    MAX_SLOTS = 8   # the scheduler's own limit; the device server accepts 1

    def __init__(self, *a, **k):
        self.images_running = 0
        self.max_images_running = 0
        self.created = 0
        self.live = set()
        super().__init__(*a, **k)

    def _context(self):
        return FakeContext(self)

    def _device_slab(self, nbytes):
        return None, 0

    def _new_handle(self, w, h, off, nbytes):
        with self.lock:
            self.created += 1
            assert nbytes >= session_bytes(w, h) and off + nbytes <= self.slab.size
            return FakeHandle(w, h, off, nbytes, self.live)


@pytest.mark.parametrize("slots,budget_images,seed", [(1, 100, 0), (3, 2, 1), (4, 5, 2),
                                                       (8, 3, 3), (8, 100, 4)])
def test_schedule_order_budget_and_misses(slots, budget_images, seed):
    rng = np.random.default_rng(seed)
    shapes = [(int(rng.integers(8, 40)), int(rng.integers(8, 40))) for _ in range(5)]
    planes = [tuple(rng.integers(-50, 50, size=(h, w)).astype(np.int32) for _ in range(5))
              for w, h in shapes]
    budget = budget_images * max(session_bytes(w, h) for w, h in shapes)
    srv = FakeServer(slots=slots, hbm_budget=budget)
    history, sid, n = {}, 0, 400
    for step in range(n):
        if step % 3 == 0 or not history:
            img = int(rng.integers(len(shapes)))
            history[sid] = (img, [])
            srv.submit(NewImage(sid, planes[img]))
            sid += 1
        else:
            recent = list(history)[-6:]
            target = recent[int(rng.integers(len(recent)))]
            v = int(rng.integers(-1000, 1000))
            history[target][1].append(v)
            srv.submit(Stroke(target, np.zeros(1, np.int32), np.zeros(1, np.int32), 1, v))
        if step % 7 == 0:
            time.sleep(0.001)
    srv.drain(timeout=60)
    results = sorted(srv.results, key=lambda r: r.arrival)
    srv.close()
    assert not srv.errors
    assert len(results) + srv.misses == n
    seen = {}
    for r in results:
        k = seen.get(r.session, 0)
        seen[r.session] = k + 1
        img, vals = history[r.session]
        assert r.flow == int(planes[img][4].sum()) + sum(vals[:k]), (r.session, k)
    assert srv.used <= budget
    assert srv.max_images_running <= max(1, slots - 1)
    if budget_images < 10:
        assert srv.evictions > 0
    if budget_images >= 100:
        assert srv.misses == 0


def test_stroke_for_unknown_session_is_a_miss():
    srv = FakeServer(slots=2, hbm_budget=1 << 30)
    srv.submit(Stroke(42, np.zeros(1, np.int32), np.zeros(1, np.int32), 1, 5))
    srv.drain(timeout=10)
    srv.close()
    assert srv.misses == 1 and not srv.results


def test_strokes_wait_for_their_queued_image():
    srv = FakeServer(slots=4, hbm_budget=1 << 30)
    pl = tuple(np.ones((16, 16), np.int32) for _ in range(5))
    srv.submit(NewImage(0, pl))
    for v in (1, 2, 3):
        srv.submit(Stroke(0, np.zeros(1, np.int32), np.zeros(1, np.int32), 1, v))
    srv.drain(timeout=10)
    srv.close()
    assert [r.flow for r in sorted(srv.results, key=lambda r: r.arrival)] == [256, 257, 259, 262]
    assert srv.misses == 0


def test_same_size_idle_session_hands_over_its_handle():
    """When the budget is full, a new image of a resident size reuses that session's handle
    (no new allocation), and later strokes on the evicted session are misses."""
    pl = tuple(np.ones((32, 32), np.int32) for _ in range(5))
    srv = FakeServer(slots=1, hbm_budget=2 * session_bytes(32, 32))
    for s in range(6):
        srv.submit(NewImage(s, pl))
        srv.drain(timeout=10)
    srv.submit(Stroke(0, np.zeros(1, np.int32), np.zeros(1, np.int32), 1, 1))
    srv.drain(timeout=10)
    srv.close()
    assert srv.created == 2
    assert srv.evictions == 4
    assert srv.misses == 1


def test_slab_best_fit_and_coalescing():
    rng = np.random.default_rng(5)
    slab = Slab(1000 * ALIGN)
    live = {}
    for step in range(3000):
        if live and (rng.random() < 0.45 or len(live) > 40):
            off = list(live)[int(rng.integers(len(live)))]
            slab.release(off, live.pop(off))
        else:
            n = int(rng.integers(1, 60)) * ALIGN - int(rng.integers(0, ALIGN))
            off = slab.alloc(n)
            if off is None:
                continue
            end = off + -(-n // ALIGN) * ALIGN
            assert off % ALIGN == 0 and end <= slab.size
            for o, ln in live.items():
                assert o + ln <= off or end <= o
            live[off] = n
        assert slab.used == sum(-(-n // ALIGN) * ALIGN for n in live.values())
    for off, n in list(live.items()):
        slab.release(off, n)
    assert slab.free == {0: slab.size} and slab.used == 0


def test_mixed_sizes_evict_to_fit():
    """Sizes that differ: evicted handles are destroyed and their ranges reused; live
    handles never overlap (checked by FakeHandle) and the budget is never exceeded."""
    rng = np.random.default_rng(11)
    shapes = [(64, 64), (200, 100), (33, 500), (400, 400), (90, 90)]
    planes = [tuple(np.ones((h, w), np.int32) for _ in range(5)) for w, h in shapes]
    srv = FakeServer(slots=4, hbm_budget=3 * session_bytes(400, 400))
    for sid in range(120):
        srv.submit(NewImage(sid, planes[int(rng.integers(len(shapes)))]))
        if sid % 3 == 0:
            srv.submit(Stroke(sid, np.zeros(1, np.int32), np.zeros(1, np.int32), 1, 1))
    srv.drain(timeout=60)
    srv.close()
    assert not srv.errors
    assert srv.evictions > 0
    assert srv.slab.used == 0 and not srv.live


def test_image_larger_than_budget_is_refused():
    srv = FakeServer(slots=2, hbm_budget=session_bytes(64, 64))
    srv.submit(NewImage(0, tuple(np.ones((512, 512), np.int32) for _ in range(5))))
    srv.submit(NewImage(1, tuple(np.ones((64, 64), np.int32) for _ in range(5))))
    with pytest.raises(MemoryError):
        srv.drain(timeout=10)
    srv.close()
    assert [r.session for r in srv.results] == [1]


def test_new_image_shape_for_every_request_form():
    """A new session may carry the five capacity planes, (image, t-links) or (image, models);
    its size comes from the t-link plane or, with models, from the image."""
    h, w = 30, 50
    planes = tuple(np.zeros((h, w), np.int32) for _ in range(5))
    rgba32 = np.zeros((h, w), np.uint32)
    rgb8 = np.zeros((h, w, 3), np.uint8)
    fg = bg = np.zeros((1, 10))
    assert NewImage(0, planes).shape == (h, w)
    assert NewImage(0, (rgba32, planes[4])).shape == (h, w)
    assert NewImage(0, (rgba32, (fg, bg))).shape == (h, w)
    assert NewImage(0, (rgb8, (fg, bg))).shape == (h, w)
