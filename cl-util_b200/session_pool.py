"""SessionPool: many resident graphs in one tile pool, any subset solved by one launch.

The serving loop keeps every session's residual graph on the device between requests.
With one solver handle per session, concurrent requests need concurrent streams and every
new image size a CUDA-graph construction of its own.  A session pool (gcp_* in
include/gcut.h) holds all sessions in one arena instead: a session opens on a slot with a
range of the pool's tiles, and a solve takes a list of slots, so the requests that are
ready at one moment (new images of different sizes, brush strokes on resident sessions) are
solved together by one launch of the pool's CUDA graph, built once for the pool.

    pool = SessionPool(max_tiles=65536, max_sessions=256)
    t0 = pool.alloc_tiles(w, h)             # a range of tiles (None when full)
    pool.open(slot, w, h, t0)
    pool.upload_image(slot, rgba, excess)   # or upload_capacities
    pool.edit_stroke(other_slot, xs, ys, radius, value)
    pool.solve([slot, other_slot])
    pool.flow(slot), pool.labels_packed(slot)
    pool.close(slot); pool.free_tiles(t0, w, h)
"""
from __future__ import annotations

import ctypes

import numpy as np

import _gcut
from _gcut import check, lib, ptr, stream_handle
from GraphCut import _as_i32_device, _as_rgba32, _on

TILE = 32


def tiles_of(width: int, height: int) -> int:
    return -(-int(width) // TILE) * -(-int(height) // TILE)


class RangeAllocator:
    """Best-fit allocator of [0, size) in integer units; freed ranges merge with free
    neighbours.  Host bookkeeping only."""

    def __init__(self, size: int):
        self.size = int(size)
        self.free = {0: self.size} if self.size > 0 else {}   # offset -> length
        self.used = 0

    def alloc(self, n: int):
        n = int(n)
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
        n = int(n)
        self.used -= n
        end = off + n
        if end in self.free:
            n += self.free.pop(end)
        prev = next((o for o, ln in self.free.items() if o + ln == off), None)
        if prev is not None:
            self.free[prev] += n
        else:
            self.free[off] = n


class SessionPool:
    def __init__(self, max_tiles: int, max_sessions: int, device: int = 0, arena=None,
                 discharge_iters=None, bfs=None, initial_relabel=None, max_cycles=None,
                 max_bfs_rounds=None, use_graph=None):
        import torch
        self.torch = torch
        self.device = torch.device("cuda", device)
        self.max_tiles, self.max_sessions = int(max_tiles), int(max_sessions)
        if discharge_iters is None and bfs is None and initial_relabel is None:
            # the autotuner's choice for pools of many grids
            import autotune
            sched = autotune.default_tuner().schedule(device, 0, 0, kind="batch",
                                                      pixels=self.max_tiles * TILE * TILE)
            discharge_iters, bfs = sched["discharge_iters"], sched["pulses_per_relabel"]
            initial_relabel = bool(sched["initial_relabel"])
        self.opts = _gcut.default_opts(device=device, discharge_iters=discharge_iters,
                                       pulses_per_relabel=bfs,
                                       initial_relabel=None if initial_relabel is None else int(initial_relabel),
                                       max_cycles=max_cycles, max_bfs_rounds=max_bfs_rounds,
                                       use_graph=None if use_graph is None else int(use_graph))
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            if arena is None:
                check(lib().gcp_create(self.max_tiles, self.max_sessions, ctypes.byref(self.opts),
                                       ctypes.byref(h)))
            else:
                addr, nbytes = ((arena.data_ptr(), arena.numel() * arena.element_size())
                                if hasattr(arena, "data_ptr") else arena)
                check(lib().gcp_create_in(self.max_tiles, self.max_sessions,
                                          ctypes.byref(self.opts), ctypes.c_void_p(addr),
                                          int(nbytes), ctypes.byref(h)))
        self._arena = arena
        self._h = h
        self.tiles = RangeAllocator(self.max_tiles)
        self.shape = {}          # slot -> (width, height)
        self._keep = {}

    @staticmethod
    def arena_bytes(max_tiles: int, max_sessions: int) -> int:
        out = ctypes.c_int64()
        check(lib().gcp_arena_bytes(int(max_tiles), int(max_sessions), ctypes.byref(out)))
        return out.value

    def close_pool(self):
        if getattr(self, "_h", None):
            lib().gcp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close_pool()
        except Exception:
            pass

    # ---- slots -------------------------------------------------------------------
    def alloc_tiles(self, width: int, height: int):
        """First tile of a free range for a width x height image, or None."""
        return self.tiles.alloc(tiles_of(width, height))

    def free_tiles(self, tile0: int, width: int, height: int):
        self.tiles.release(tile0, tiles_of(width, height))

    def open(self, slot: int, width: int, height: int, tile0: int, stream=None):
        check(lib().gcp_open(self._h, int(slot), int(width), int(height), int(tile0),
                             stream_handle(stream)))
        self.shape[int(slot)] = (int(width), int(height))

    def close(self, slot: int):
        check(lib().gcp_close(self._h, int(slot)))
        self.shape.pop(int(slot), None)
        self._keep.pop(int(slot), None)

    # ---- input ---------------------------------------------------------------------
    def upload_capacities(self, slot, up, down, left, right, excess, stream=None):
        w, h = self.shape[int(slot)]
        planes = (up, down, left, right, excess)
        if any(tuple(p.shape) != (h, w) for p in planes):
            raise ValueError("plane shape differs from the slot's")
        with _on(stream):
            dev = [_as_i32_device(p, self.device) for p in planes]
        check(lib().gcp_upload(self._h, int(slot), *[ptr(d) for d in dev], stream_handle(stream)))
        self._keep[int(slot)] = dev

    def upload_image(self, slot, rgba, excess, stream=None):
        """The n-links from the image on the device (floor(50 exp(-beta |dI|^2) + 0.5), as
        GraphCut.upload_image), t-links from `excess`."""
        torch = self.torch
        w, h = self.shape[int(slot)]
        rgba = _as_rgba32(rgba)
        if tuple(rgba.shape) != (h, w) or tuple(excess.shape) != (h, w):
            raise ValueError("image / excess shape differs from the slot's")
        with _on(stream):
            if not (isinstance(rgba, torch.Tensor) and rgba.is_cuda):
                host = rgba.cpu().numpy() if isinstance(rgba, torch.Tensor) else rgba
                rgba = torch.from_numpy(np.ascontiguousarray(host).view(np.int32)).to(self.device)
            img = rgba.contiguous()
            ex = _as_i32_device(excess, self.device)
        check(lib().gcp_upload_rgba(self._h, int(slot), ptr(img), ptr(ex), stream_handle(stream)))
        self._keep[int(slot)] = (img, ex)

    def _edit(self, fn, slot, xs, ys, radius, value, stream):
        xs = np.ascontiguousarray(xs, dtype=np.int32)
        ys = np.ascontiguousarray(ys, dtype=np.int32)
        if xs.shape != ys.shape or xs.ndim != 1:
            raise ValueError("xs and ys must be 1-D arrays of the same length")
        check(fn(self._h, int(slot), ptr(xs), ptr(ys), int(xs.shape[0]), int(radius),
                 int(value), stream_handle(stream)))

    def edit_stroke(self, slot, xs, ys, radius: int, value: int, stream=None):
        """Pixels within `radius` of the polyline get t-link `value` (gc_edit_stroke)."""
        self._edit(lib().gcp_edit_stroke, slot, xs, ys, radius, value, stream)

    def edit_brush(self, slot, xs, ys, radius: int, value: int, stream=None):
        """The reference brush's pixel set gets t-link `value` (gc_edit_brush)."""
        self._edit(lib().gcp_edit_brush, slot, xs, ys, radius, value, stream)

    # ---- solve and results ---------------------------------------------------------
    def solve(self, slots, stream=None):
        """Solves the listed slots together (one launch); returns when done."""
        arr = (ctypes.c_int * len(slots))(*[int(s) for s in slots])
        with self.torch.cuda.device(self.device):
            check(lib().gcp_solve(self._h, arr, len(slots), stream_handle(stream)))
        for s in slots:
            self._keep.pop(int(s), None)

    def solve_labels(self, slots, outs=None, packed=True, stream=None):
        """solve() and every slot's labels (bit-packed by default) with one host wait
        (gcp_solve_labels); returns the label tensors in the order of `slots`."""
        torch = self.torch
        if outs is None:
            outs = []
            for s in slots:
                w, h = self.shape[int(s)]
                shape = (h, (w + 7) // 8) if packed else (h, w)
                outs.append(torch.empty(shape, dtype=torch.uint8, device=self.device))
        arr = (ctypes.c_int * len(slots))(*[int(s) for s in slots])
        bufs = (ctypes.c_void_p * len(slots))(*[o.data_ptr() for o in outs])
        with torch.cuda.device(self.device):
            check(lib().gcp_solve_labels(self._h, arr, len(slots), bufs, int(bool(packed)),
                                         stream_handle(stream)))
        for s in slots:
            self._keep.pop(int(s), None)
        return outs

    def flow(self, slot) -> int:
        f = ctypes.c_int64(0)
        check(lib().gcp_flow(self._h, int(slot), ctypes.byref(f)))
        return int(f.value)

    def labels(self, slot, out=None, stream=None):
        w, h = self.shape[int(slot)]
        if out is None:
            out = self.torch.empty((h, w), dtype=self.torch.uint8, device=self.device)
        check(lib().gcp_labels(self._h, int(slot), ptr(out), stream_handle(stream)))
        return out

    def labels_packed(self, slot, out=None, stream=None):
        w, h = self.shape[int(slot)]
        if out is None:
            out = self.torch.empty((h, (w + 7) // 8), dtype=self.torch.uint8, device=self.device)
        check(lib().gcp_labels_packed(self._h, int(slot), ptr(out), stream_handle(stream)))
        return out

    def stats(self) -> dict:
        st = _gcut.GcStats()
        check(lib().gcp_get_stats(self._h, ctypes.byref(st)))
        return st.as_dict()
