"""Serving loop: image sessions and brush-stroke edits arriving over time.

The reference is an interactive tool: one image, strokes from the GUI, ``GraphCut.cut`` run
on a button press (test_GraphCut.py:78-99).  Here many sessions share one GPU, served by
one of two servers with the same request / result interface:

* ``BatchingServer``: continuous batching.  Every session lives in one session pool
  (session_pool.SessionPool, gcp_* in include/gcut.h); each tick of its worker takes every
  request ready at that moment and solves them all in one launch of the pool's CUDA graph,
  so requests of different sizes overlap on the device and none waits for a graph build;
* ``GraphCutServer``: the plain one-at-a-time solver, one GraphCut handle per session,
  described below.

GraphCutServer:

* a request is either a NEW image (capacity planes in host memory) or a STROKE on a
  resident session; every request returns the flow value and the canonical labels of its
  session after the solve, read back bit-packed (one bit per pixel; ``Result.labels``
  unpacks them);
* each session keeps its residual graph, heights and t-links resident on the device
  (one ``GraphCut`` handle), so a stroke re-solves warm from the previous flow;
* admission is gated by HBM: the server owns one device region of ``hbm_budget`` bytes
  (the slab) and places every session's state in a range of it (best fit, freed ranges
  coalesce; ``GraphCut(arena=...)``).  A new image takes a free range, else the handle
  of the least-recently-used idle session of its size, else evicts least-recently-used
  idle sessions until a range fits.  Creating and evicting sessions therefore never calls
  cudaMalloc / cudaFree, which synchronise the device, on the request path;
* slots: each slot is a worker thread with its own stream; a request starts as soon as a
  slot is free and its session is idle (a stroke waits only for its own session).  The
  device server accepts one slot (``MAX_SLOTS``): several requests in flight on separate
  streams raised an intermittent device fault whose cause is not established.  The
  solver calls release the Python GIL;
* scheduling is earliest-arrival-first over the head new image and the sessions with a
  queued stroke, with one slot kept for strokes (at most ``slots - 1`` new images in
  flight), so an edit never waits behind a wall of image uploads.  Strokes of one session
  run in submission order.  A stroke for a session that was evicted is a miss.

Host planes in pinned memory are copied to the device asynchronously (into per-worker
staging); pageable planes work too, with synchronous copies.

Results do not depend on the mix: the flow value and the canonical cut of a session are
unique for its graph, which the tests check request by request.
"""
from __future__ import annotations

import collections
import dataclasses
import heapq
import itertools
import threading
import time

import numpy as np

import _gcut
from GraphCut import GraphCut, unpack_labels

ALIGN = 256   # arena alignment the solver requires


def session_bytes(width: int, height: int) -> int:
    """Device bytes of one resident session of this size: its solver arena (tile planes,
    masks, flags, label staging), rounded to the slab's alignment."""
    n = GraphCut.arena_bytes(width, height)
    return -(-n // ALIGN) * ALIGN


class Slab:
    """Best-fit range allocator over [0, size): offsets and lengths in ALIGN units; a
    released range merges with free neighbours.  Host bookkeeping only."""

    def __init__(self, size: int):
        self.size = size - size % ALIGN
        self.free = {0: self.size} if self.size else {}   # offset -> length
        self.used = 0

    def alloc(self, n: int):
        """Offset of a free range of n bytes (rounded up), or None."""
        n = -(-n // ALIGN) * ALIGN
        best = None
        for off, ln in self.free.items():
            if ln >= n and (best is None or ln < self.free[best]):
                best = off
        if best is None:
            return None
        ln = self.free.pop(best)
        if ln > n:
            self.free[best + n] = ln - n
        self.used += n
        return best

    def release(self, off: int, n: int):
        n = -(-n // ALIGN) * ALIGN
        self.used -= n
        end = off + n
        if end in self.free:
            n += self.free.pop(end)
        prev = next((o for o, ln in self.free.items() if o + ln == off), None)
        if prev is not None:
            self.free[prev] += n
        else:
            self.free[off] = n


@dataclasses.dataclass
class NewImage:
    """A new session.  `planes` is one of
    - (up, down, left, right, excess): host int32 [H, W] capacity planes (20 B/px);
    - (rgba, excess): the image (uint32 [H, W], RGBA bytes viewed as uint32) and the t-links,
      the reference's own inputs; the n-links are built on the device (8 B/px);
    - (rgba, (fg, bg)): the image and two colour models (gmm_tlinks.Mixture or components
      arrays); n-links and t-links are both built on the device (4 B/px)."""
    session: int
    planes: tuple

    @property
    def shape(self):
        if isinstance(self.planes[-1], tuple):
            return tuple(self.planes[0].shape[:2])
        return self.planes[-1].shape   # (H, W) of the excess plane


@dataclasses.dataclass
class Stroke:
    session: int
    xs: np.ndarray
    ys: np.ndarray
    radius: int
    value: int


@dataclasses.dataclass
class Result:
    session: int
    kind: str
    flow: int
    bits: np.ndarray         # canonical labels, bit-packed rows (GraphCut.labels_packed)
    width: int
    arrival: float
    start: float
    done: float
    pixels: int
    phases_ms: tuple = ()    # (input, solve, labels) host-side durations

    @property
    def labels(self) -> np.ndarray:
        """uint8 [H, W] canonical labels (1 = source side), unpacked on access."""
        return unpack_labels(self.bits, self.width)

    @property
    def latency_ms(self) -> float:
        return 1000.0 * (self.done - self.arrival)


class _Session:
    def __init__(self, sid, gc, width, height, off, nbytes):
        self.sid, self.gc, self.width, self.height = sid, gc, width, height
        self.off, self.nbytes = off, nbytes      # its range of the slab
        self.busy = False
        self.last_use = time.perf_counter()


class GraphCutServer:
    """Serves NewImage / Stroke requests on one GPU (see the module docstring)."""

    # Requests in flight at once.  Several requests on separate streams raised an
    # intermittent "unspecified launch failure" on the B200 whose cause is not established,
    # so the device server runs one at a time; the scheduler itself handles any number
    # (its host-side tests run it with several slots against a fake solver).
    MAX_SLOTS = 1

    def __init__(self, slots: int = 1, hbm_budget: int = 16 << 30, device: int = 0,
                 solver_kw=None, max_pixels: int = 4096 * 4096):
        if not 1 <= slots <= self.MAX_SLOTS:
            raise ValueError(f"GraphCutServer: slots must be between 1 and {self.MAX_SLOTS} "
                             "(concurrent slots raised an intermittent device fault whose "
                             "cause is not found)")
        import torch
        self.torch = torch
        self.device = device
        self.slots = slots
        self.budget = hbm_budget
        self.solver_kw = dict(solver_kw or {})
        self.max_pixels = max_pixels   # staging of each worker is sized for this at start
        self.lock = threading.Condition()
        self.images = collections.deque()              # (NewImage, arrival) in arrival order
        self.strokes = collections.defaultdict(collections.deque)  # session -> (Stroke, arrival)
        self.ready = []          # heap of (head stroke arrival, seq, session): idle + queued
        self._seq = itertools.count()
        self.sessions: dict[int, _Session] = {}
        self.lru = collections.OrderedDict()           # idle resident sessions, oldest first
        self.slab = Slab(hbm_budget)
        self._slab_mem, self._base = self._device_slab(self.slab.size)
        self.queued_images = set()    # sessions whose NewImage is queued or being solved
        self.results: list[Result] = []
        self.misses = 0
        self.evictions = 0
        self.errors = []
        self.stop = False
        self.inflight = 0
        self.images_inflight = 0
        self._ready = 0
        self.workers = [threading.Thread(target=self._worker, args=(k,), daemon=True)
                        for k in range(slots)]
        for w in self.workers:
            w.start()
        # start-up (streams, staging) is not request latency: wait until every worker is set
        with self.lock:
            while self._ready < slots:
                self.lock.wait(0.05)
        if self.errors:
            raise self.errors[0]

    # ---- client side ------------------------------------------------------------
    def submit(self, request, arrival=None):
        arrival = time.perf_counter() if arrival is None else arrival
        with self.lock:
            sid = request.session
            if isinstance(request, Stroke):
                s = self.sessions.get(sid)
                if s is None and sid not in self.queued_images:
                    self.misses += 1      # the session was evicted (or never existed)
                    return
                q = self.strokes[sid]
                q.append((request, arrival))
                if s is not None and not s.busy and len(q) == 1:
                    self._make_ready(s)
            else:
                self.queued_images.add(sid)
                self.images.append((request, arrival))
            self.lock.notify()

    def drain(self, timeout=600.0):
        t0 = time.perf_counter()
        with self.lock:
            while (self.images or self.ready or self.inflight) and time.perf_counter() - t0 < timeout:
                self.lock.wait(0.05)
        if self.errors:
            raise self.errors[0]

    def close(self):
        with self.lock:
            self.stop = True
            self.lock.notify_all()
        for w in self.workers:
            w.join()
        for s in list(self.sessions.values()):
            self._destroy(s.gc)
            self.slab.release(s.off, s.nbytes)
        self.sessions.clear()
        self.lru.clear()
        self._slab_mem = None

    @property
    def used(self) -> int:
        """Bytes of the slab held by resident and in-flight sessions."""
        return self.slab.used

    # ---- scheduling (all under self.lock) ------------------------------------------
    def _make_ready(self, s):
        """s is resident, idle and has a queued stroke: it may be picked."""
        self.lru.pop(s.sid, None)
        heapq.heappush(self.ready, (self.strokes[s.sid][0][1], next(self._seq), s.sid))

    def _release(self, s):
        """s finished a request: it is ready again, or idle (evictable)."""
        s.busy = False
        s.last_use = time.perf_counter()
        if self.strokes.get(s.sid):
            self._make_ready(s)
        else:
            self.strokes.pop(s.sid, None)
            self.lru[s.sid] = s

    def _pick(self):
        """Next request that can start now, or None."""
        stroke_arr = self.ready[0][0] if self.ready else float("inf")
        image_ok = self.images and self.images_inflight < max(1, self.slots - 1)
        if image_ok and self.images[0][1] <= stroke_arr:
            job = self._pick_image()
            if job is not None:
                return job
        if self.ready:
            _, _, sid = heapq.heappop(self.ready)
            s = self.sessions[sid]
            req, arr = self.strokes[sid].popleft()
            s.busy = True
            return req, arr, s
        return self._pick_image() if image_ok else None

    def _pick_image(self):
        if not self.images:
            return None
        req, arr = self.images[0]
        h, w = req.shape
        if session_bytes(w, h) > self.slab.size:   # can never fit: refuse it
            self.images.popleft()
            self.queued_images.discard(req.session)
            self.strokes.pop(req.session, None)
            self.errors.append(MemoryError(f"session {req.session}: {w}x{h} needs more than "
                                           f"the HBM budget of {self.slab.size} bytes"))
            return None
        place = self._admit(w, h)
        if place is None:
            return None
        self.images.popleft()
        self.images_inflight += 1
        return req, arr, place

    def _evict(self, s):
        del self.sessions[s.sid]
        self.lru.pop(s.sid, None)
        self.evictions += 1

    def _admit(self, w, h):
        """Room for a (w, h) session: (handle to reuse or None, offset, bytes), or None when
        nothing fits until a session goes idle."""
        need = session_bytes(w, h)
        off = self.slab.alloc(need)
        if off is not None:
            return None, off, need
        # full: the least-recently-used idle session of this size hands over its handle
        for s in self.lru.values():
            if (s.width, s.height) == (w, h):
                self._evict(s)
                return s.gc, s.off, s.nbytes
        # else evict least-recently-used idle sessions until a range fits
        while self.lru:
            victim = next(iter(self.lru.values()))
            self._evict(victim)
            self._destroy(victim.gc)
            self.slab.release(victim.off, victim.nbytes)
            off = self.slab.alloc(need)
            if off is not None:
                return None, off, need
        return None

    # ---- workers ----------------------------------------------------------------------
    def _context(self):
        """Per-worker device context (a stream and staging buffers); called on the worker."""
        return _DeviceContext(self.torch, self.device, self.max_pixels)

    def _device_slab(self, nbytes):
        """(owner, device address) of the slab's memory: one allocation for the server's
        lifetime."""
        t = self.torch.empty(max(nbytes, 1), dtype=self.torch.uint8,
                             device=self.torch.device("cuda", self.device))
        assert t.data_ptr() % ALIGN == 0
        return t, t.data_ptr()

    def _new_handle(self, w, h, off, nbytes):
        return GraphCut(w, h, device=self.device, arena=(self._base + off, nbytes),
                        **self.solver_kw)

    def _destroy(self, gc):
        gc.close()   # idle: returns at once; the range may be reused afterwards

    def _worker(self, k):
        try:
            ctx = self._context()
        except Exception as exc:   # surfaced by the constructor
            with self.lock:
                self.errors.append(exc)
                self._ready += 1
                self.lock.notify_all()
            return
        with self.lock:
            self._ready += 1
            self.lock.notify_all()
        while True:
            with self.lock:
                job = None
                while not self.stop:
                    job = self._pick()
                    if job is not None:
                        break
                    self.lock.wait(0.05)
                if job is None:
                    return
                req, arrival, sess = job
                self.inflight += 1
                gc = None
                if isinstance(req, NewImage):
                    (gc, off, nbytes), sess = sess, None
            try:
                start = time.perf_counter()
                if sess is None:
                    h, w = req.shape
                    if gc is None:
                        gc = self._new_handle(w, h, off, nbytes)
                    flow, bits, phases = ctx.run_image(gc, req.planes, w, h)
                    res = Result(req.session, "image", flow, bits, w, arrival, start,
                                 time.perf_counter(), w * h, phases)
                else:
                    flow, bits, phases = ctx.run_stroke(sess.gc, req, sess.width, sess.height)
                    res = Result(req.session, "stroke", flow, bits, sess.width, arrival, start,
                                 time.perf_counter(), sess.width * sess.height, phases)
                with self.lock:
                    self.results.append(res)
                    if sess is None:
                        sess = _Session(req.session, gc, w, h, off, nbytes)
                        self.sessions[req.session] = sess
                        self.queued_images.discard(req.session)
                        self.images_inflight -= 1
                    self._release(sess)
            except Exception as exc:  # surfaced by drain()
                with self.lock:
                    self.errors.append(exc)
                    if sess is not None:
                        self._release(sess)
                    else:   # the session never opened: its handle and range are released
                        self.queued_images.discard(req.session)
                        self.images_inflight -= 1
                        self.strokes.pop(req.session, None)
                        if gc is not None:
                            self._destroy(gc)
                        self.slab.release(off, nbytes)
            finally:
                with self.lock:
                    self.inflight -= 1
                    self.lock.notify_all()


class _DeviceContext:
    """One worker's stream, device staging for the input planes and pinned staging for the
    packed labels, reused across requests in stream order.  Both are sized for `max_pixels`
    when the worker starts (allocation on the request path would stall the device) and grow
    only for a larger image."""

    def __init__(self, torch, device, max_pixels):
        self.torch = torch
        torch.cuda.set_device(device)
        self.device = device
        self.stream = torch.cuda.Stream()
        self.dstage = torch.empty(5 * max_pixels, dtype=torch.int32, device=device)
        self.lstage = torch.empty(max_pixels // 8 + 65536, dtype=torch.uint8, pin_memory=True)

    def _upload(self, gc, planes, w, h):
        torch, n = self.torch, w * h
        if self.dstage.numel() < 5 * n:
            self.dstage = torch.empty(5 * n, dtype=torch.int32, device=self.device)
        if isinstance(planes[-1], tuple):   # (rgba, (fg, bg)): t-links from the models
            import gmm_tlinks
            from GraphCut import _as_rgba32
            img = self.dstage[:n].view(h, w)
            img.copy_(torch.from_numpy(np.ascontiguousarray(_as_rgba32(planes[0])).view(np.int32)),
                      non_blocking=True)
            ex = gmm_tlinks.tlinks(img, *planes[1], out=self.dstage[n:2 * n].view(h, w),
                                   stream=self.stream)
            gc.upload_image(img, ex, stream=self.stream)
            return
        dev = []
        for j, p in enumerate(planes):
            d = self.dstage[j * n:(j + 1) * n].view(h, w)
            src = np.ascontiguousarray(p)
            if src.dtype == np.uint32:
                src = src.view(np.int32)   # the image: same bits, a dtype torch copies
            d.copy_(torch.from_numpy(np.ascontiguousarray(src, dtype=np.int32)), non_blocking=True)
            dev.append(d)
        if len(dev) == 2:   # (rgba, excess): n-links built on the device
            gc.upload_image(dev[0], dev[1], stream=self.stream)
        else:
            gc.upload_capacities(*dev, stream=self.stream)

    def _labels(self, gc, w, h):
        n = h * ((w + 7) // 8)
        if self.lstage.numel() < n:
            self.lstage = self.torch.empty(n, dtype=self.torch.uint8, pin_memory=True)
        buf = self.lstage[:n].numpy().reshape(h, (w + 7) // 8)
        gc.labels_packed_host(out=buf, stream=self.stream)
        return buf.copy()

    def run_image(self, gc, planes, w, h):
        t0 = time.perf_counter()
        with self.torch.cuda.stream(self.stream):
            self._upload(gc, planes, w, h)
            t1 = time.perf_counter()
            gc.cut(stream=self.stream)
            t2 = time.perf_counter()
            labels = self._labels(gc, w, h)
        t3 = time.perf_counter()
        return gc.flow, labels, (1e3 * (t1 - t0), 1e3 * (t2 - t1), 1e3 * (t3 - t2))

    def run_stroke(self, gc, req, w, h):
        t0 = time.perf_counter()
        with self.torch.cuda.stream(self.stream):
            gc.edit_stroke(req.xs, req.ys, req.radius, req.value, stream=self.stream)
            t1 = time.perf_counter()
            gc.cut(stream=self.stream)
            t2 = time.perf_counter()
            labels = self._labels(gc, w, h)
        t3 = time.perf_counter()
        return gc.flow, labels, (1e3 * (t1 - t0), 1e3 * (t2 - t1), 1e3 * (t3 - t2))


def poisson_trace(rng, rate_hz, duration_s, n_images, p_new=0.3):
    """(time, kind, image index) tuples of a Poisson stream: a new image with probability
    p_new, else a stroke on a resident session."""
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate_hz)
        if t >= duration_s:
            return out
        out.append((t, "image" if rng.random() < p_new else "stroke", int(rng.integers(n_images))))


class _PoolSession:
    def __init__(self, sid, slot, tile0, width, height):
        self.sid, self.slot, self.tile0 = sid, slot, tile0
        self.width, self.height = width, height
        self.last_use = time.perf_counter()


class BatchingServer:
    """Continuous batching on one GPU: every session lives in one SessionPool, and each tick
    of the worker solves all the requests that are ready at that moment in one launch.

    A tick takes, under the lock, the head stroke of every resident session with queued
    strokes (one per session, so strokes of a session stay in order) and the queued new
    images in arrival order, as far as free tiles, free slots (evicting least-recently-used
    idle sessions) and `tick_pixels` allow (at least one image per tick).  It uploads the
    images and applies the strokes, solves all of them together (gcp_solve), and reads every
    flow and bit-packed cut back.  Requests that arrive meanwhile join the next tick, so the
    solves of different sizes overlap on the device inside one launch instead of on
    concurrent streams, and no request waits for a CUDA-graph construction: the pool's graph
    is built at start-up.  Results do not depend on the mix: each session's flow value and
    canonical cut are unique for its graph.

    Same request / result interface as GraphCutServer (submit, drain, close, results,
    misses, evictions)."""

    def __init__(self, hbm_budget: int = 16 << 30, device: int = 0, max_sessions: int = 512,
                 tick_pixels: int = 24 << 20, solver_kw=None, warm_up: bool = True):
        import torch

        from session_pool import SessionPool
        self.torch = torch
        self.device = device
        self.tick_pixels = int(tick_pixels)
        max_tiles = self._tiles_for(hbm_budget, max_sessions)
        self.budget = SessionPool.arena_bytes(max_tiles, max_sessions)
        self.pool = SessionPool(max_tiles, max_sessions, device=device, **(solver_kw or {}))
        self.lock = threading.Condition()
        self.images = collections.deque()              # (NewImage, arrival)
        self.strokes = collections.defaultdict(collections.deque)  # session -> (Stroke, arrival)
        self.sessions: dict[int, _PoolSession] = {}
        self.lru = collections.OrderedDict()           # resident sessions, oldest first
        self.free_slots = list(range(max_sessions - 1, -1, -1))
        self.queued_images = set()
        self.results: list[Result] = []
        self.misses = 0
        self.evictions = 0
        self.ticks = 0
        self.errors = []
        self.stop = False
        self.inflight = 0
        with torch.cuda.device(device):
            self.stream = torch.cuda.Stream()
            # staging for a tick of tick_pixels (grown on demand, see _reserve)
            self.dstage = torch.empty(2 * self.tick_pixels, dtype=torch.int32, device=device)
            nb = self.tick_pixels // 4 + (1 << 20)
            self.dbits = torch.empty(nb, dtype=torch.uint8, device=device)
            self.hbits = torch.empty(nb, dtype=torch.uint8, pin_memory=True)
        self._cursor = 0
        if warm_up:
            self._warm_up()
        self.worker = threading.Thread(target=self._worker, daemon=True)
        self.worker.start()

    @staticmethod
    def _tiles_for(budget, max_sessions):
        """The most tiles whose pool fits in `budget` bytes."""
        from session_pool import SessionPool
        lo, hi = 1, 1 << 26
        if SessionPool.arena_bytes(lo, max_sessions) > budget:
            raise MemoryError("the HBM budget does not hold a session pool")
        while lo < hi:
            mid = (lo + hi + 1) // 2
            if SessionPool.arena_bytes(mid, max_sessions) <= budget:
                lo = mid
            else:
                hi = mid - 1
        return lo

    def _warm_up(self):
        """Builds the pool's CUDA graphs before the first request: a fresh solve and a warm
        one of a small image."""
        torch = self.torch
        t0 = self.pool.alloc_tiles(64, 64)
        slot = self.free_slots[-1]
        z = torch.zeros((64, 64), dtype=torch.int32, device=self.pool.device)
        ex = torch.zeros((64, 64), dtype=torch.int32, device=self.pool.device)
        ex[0, 0], ex[-1, -1] = 5, -5
        with torch.cuda.stream(self.stream):
            self.pool.open(slot, 64, 64, t0, stream=self.stream)
            self.pool.upload_capacities(slot, z + 1, z + 1, z + 1, z + 1, ex, stream=self.stream)
            self.pool.solve([slot], stream=self.stream)
            self.pool.edit_stroke(slot, [3], [3], 2, 7, stream=self.stream)
            self.pool.solve([slot], stream=self.stream)
        self.pool.close(slot)
        self.pool.free_tiles(t0, 64, 64)

    # ---- client side ------------------------------------------------------------
    def submit(self, request, arrival=None):
        arrival = time.perf_counter() if arrival is None else arrival
        with self.lock:
            sid = request.session
            if isinstance(request, Stroke):
                if sid not in self.sessions and sid not in self.queued_images:
                    self.misses += 1      # evicted (or never opened)
                    return
                self.strokes[sid].append((request, arrival))
            else:
                self.queued_images.add(sid)
                self.images.append((request, arrival))
            self.lock.notify()

    def drain(self, timeout=600.0):
        t0 = time.perf_counter()
        with self.lock:
            while ((self.images or self.inflight or
                    any(q and (s in self.sessions or s in self.queued_images)
                        for s, q in self.strokes.items()))
                   and time.perf_counter() - t0 < timeout):
                self.lock.wait(0.05)
        if self.errors:
            raise self.errors[0]

    def close(self):
        with self.lock:
            self.stop = True
            self.lock.notify_all()
        self.worker.join()
        self.pool.close_pool()

    @property
    def used_tiles(self) -> int:
        """Tiles of the pool held by resident sessions."""
        return self.pool.tiles.used

    # ---- scheduling (under self.lock) ---------------------------------------------
    def _evict_one(self, keep):
        for sid, s in self.lru.items():
            if sid in keep or self.strokes.get(sid):
                continue
            del self.lru[sid]
            del self.sessions[sid]
            self.strokes.pop(sid, None)
            self.pool.close(s.slot)
            self.pool.free_tiles(s.tile0, s.width, s.height)
            self.free_slots.append(s.slot)
            self.evictions += 1
            return True
        return False

    def _take_tick(self):
        """(strokes, images) of the next tick, or None."""
        strokes = []
        for sid, q in self.strokes.items():
            if q and sid in self.sessions:
                req, arr = q.popleft()
                strokes.append((req, arr, self.sessions[sid]))
        keep = {req.session for req, _, _ in strokes}
        images, px = [], 0
        while self.images:
            req, arr = self.images[0]
            h, w = req.shape
            if images and px + w * h > self.tick_pixels:
                break
            from session_pool import tiles_of
            if tiles_of(w, h) > self.pool.max_tiles:
                self.images.popleft()
                self.queued_images.discard(req.session)
                self.strokes.pop(req.session, None)
                self.errors.append(MemoryError(f"session {req.session}: {w}x{h} needs more "
                                               "than the pool holds"))
                continue
            t0 = self.pool.alloc_tiles(w, h)
            while (t0 is None or not self.free_slots) and self._evict_one(keep):
                if t0 is None:
                    t0 = self.pool.alloc_tiles(w, h)
            if t0 is None or not self.free_slots:
                if t0 is not None:
                    self.pool.free_tiles(t0, w, h)
                break
            self.images.popleft()
            slot = self.free_slots.pop()
            s = _PoolSession(req.session, slot, t0, w, h)
            images.append((req, arr, s))
            keep.add(req.session)
            px += w * h
        if not strokes and not images:
            return None
        return strokes, images

    # ---- worker -----------------------------------------------------------------------
    def _worker(self):
        torch = self.torch
        while True:
            with self.lock:
                tick = None
                while not self.stop:
                    tick = self._take_tick()
                    if tick is not None:
                        break
                    self.lock.wait(0.02)
                if tick is None:
                    return
                strokes, images = tick
                self.inflight += len(strokes) + len(images)
            try:
                start = time.perf_counter()
                jobs = images + strokes
                with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
                    self._reserve(images, jobs)
                    for req, _, s in images:
                        self.pool.open(s.slot, s.width, s.height, s.tile0, stream=self.stream)
                        self._upload(s, req.planes)
                    for req, _, s in strokes:
                        self.pool.edit_stroke(s.slot, req.xs, req.ys, req.radius, req.value,
                                              stream=self.stream)
                    t1 = time.perf_counter()
                    # the solve and every job's packed labels into one device buffer, one
                    # host wait; then one copy of that buffer to the pinned staging
                    outs, spans = self._label_views(jobs)
                    self.pool.solve_labels([s.slot for _, _, s in jobs], outs=outs,
                                           stream=self.stream)
                    t2 = time.perf_counter()
                    flows = [self.pool.flow(s.slot) for _, _, s in jobs]
                    total = spans[-1][0] + spans[-1][1]
                    self.hbits[:total].copy_(self.dbits[:total], non_blocking=True)
                    self.stream.synchronize()
                    hb = self.hbits.numpy()
                    host = [hb[off:off + n].reshape(s.height, (s.width + 7) // 8).copy()
                            for (off, n), (_, _, s) in zip(spans, jobs)]
                done = time.perf_counter()
                phases = (1e3 * (t1 - start), 1e3 * (t2 - t1), 1e3 * (done - t2))
                with self.lock:
                    self.ticks += 1
                    for (req, arr, s), f, bits in zip(jobs, flows, host):
                        kind = "stroke" if isinstance(req, Stroke) else "image"
                        self.results.append(Result(s.sid, kind, f, bits, s.width, arr,
                                                   start, done, s.width * s.height, phases))
                        if kind == "image":
                            self.sessions[s.sid] = s
                            self.queued_images.discard(s.sid)
                        s.last_use = done
                        self.lru.pop(s.sid, None)
                        self.lru[s.sid] = s
            except Exception as exc:  # surfaced by drain()
                with self.lock:
                    self.errors.append(exc)
                    for req, _, s in images:
                        self.queued_images.discard(req.session)
                        if s.sid not in self.sessions:
                            try:
                                self.pool.close(s.slot)
                            except Exception:
                                pass
                            self.pool.free_tiles(s.tile0, s.width, s.height)
                            self.free_slots.append(s.slot)
            finally:
                with self.lock:
                    self.inflight -= len(strokes) + len(images)
                    self.lock.notify_all()

    # ---- staging (worker thread) ------------------------------------------------------
    # Device memory for the tick's input planes and its packed labels, and pinned host memory
    # for the labels' copy back: reused tick after tick (the previous tick's work finished
    # before this one starts) and grown, before the tick's first copy, only when a tick needs
    # more.  Allocating per request instead (fresh device tensors, a fresh pinned block for
    # every result) stalled ticks for up to a quarter of a second.
    @staticmethod
    def _planes_of(req) -> int:
        return 2 if len(req.planes) == 2 else 5

    def _reserve(self, images, jobs):
        torch = self.torch
        need = sum(self._planes_of(req) * s.width * s.height for req, _, s in images)
        if need > self.dstage.numel():
            self.dstage = torch.empty(need + (need >> 2), dtype=torch.int32, device=self.pool.device)
        nbits = sum(self._bits_span(s) for _, _, s in jobs)
        if nbits > self.dbits.numel():
            n = nbits + (nbits >> 2)
            self.dbits = torch.empty(n, dtype=torch.uint8, device=self.pool.device)
            self.hbits = torch.empty(n, dtype=torch.uint8, pin_memory=True)
        self._cursor = 0

    @staticmethod
    def _bits_span(s) -> int:
        return (s.height * ((s.width + 7) // 8) + 15) & ~15   # 16-byte aligned slices

    def _label_views(self, jobs):
        outs, spans, off = [], [], 0
        for _, _, s in jobs:
            n = s.height * ((s.width + 7) // 8)
            outs.append(self.dbits[off:off + n].view(s.height, (s.width + 7) // 8))
            spans.append((off, n))
            off += self._bits_span(s)
        return outs, spans

    def _stage(self, n):
        v = self.dstage[self._cursor:self._cursor + n]
        self._cursor += n
        return v

    def _upload(self, s, planes):
        """A new session's inputs (the same three forms as GraphCutServer's) to its slot,
        through the tick's device staging."""
        torch = self.torch
        w, h = s.width, s.height
        n = w * h
        if isinstance(planes[-1], tuple):   # (rgba, (fg, bg)): t-links from the models
            import gmm_tlinks
            from GraphCut import _as_rgba32
            img = self._stage(n).view(h, w)
            img.copy_(torch.from_numpy(np.ascontiguousarray(_as_rgba32(planes[0])).view(np.int32)),
                      non_blocking=True)
            ex = gmm_tlinks.tlinks(img, *planes[1], out=self._stage(n).view(h, w),
                                   stream=self.stream)
            self.pool.upload_image(s.slot, img, ex, stream=self.stream)
            return
        dev = []
        for p in planes:
            src = np.ascontiguousarray(p)
            if src.dtype == np.uint32:
                src = src.view(np.int32)
            d = self._stage(n).view(h, w)
            d.copy_(torch.from_numpy(np.ascontiguousarray(src, dtype=np.int32)), non_blocking=True)
            dev.append(d)
        if len(dev) == 2:
            self.pool.upload_image(s.slot, dev[0], dev[1], stream=self.stream)
        else:
            self.pool.upload_capacities(s.slot, *dev, stream=self.stream)
