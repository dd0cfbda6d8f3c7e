"""GraphCut: the solver class of the reference (GraphCut.pyx:29-437) on libgcut.

The reference class is built from an OpenCL context and an RGBA image and derives its
n-link capacities on the device (``GraphCut(context, devices, dImg, lamda)``,
GraphCut.pyx:80; load_tiles, graphcut.cl:1033-1132); its ``cut(dExcess, bfs)`` mutates the
excess buffer in place and returns nothing (GraphCut.pyx:348-418).  Here the capacities are
uploaded (int32 planes, see include/gcut.h), and the solve yields the max-flow value and
the canonical minimum cut:

    gc = GraphCut(width, height)
    gc.upload_capacities(up, down, left, right, excess)   # torch CUDA int32 or numpy int32
    gc.cut()
    gc.flow, gc.labels()                                   # int, torch.uint8 [H, W] on device

The reference's stepping methods keep their names: ``push``, ``relabel``, ``startBfs``,
``isCompleted``; its read-only device planes ``dUp, dDown, dLeft, dRight, dHeight`` and
``dExcess`` are materialised as row-major tensors on access.
"""
from __future__ import annotations

import ctypes

import numpy as np

import _gcut
from _gcut import check, lib, ptr, stream_handle

BFS_DEFAULT = 5  # GraphCut.pyx:27


def _as_i32_device(a, device):
    import torch
    if isinstance(a, torch.Tensor):
        if a.dtype != torch.int32:
            raise TypeError("capacity planes must be int32")
        return a.to(device).contiguous()
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.int32)).to(device)


def _device_guard(device):
    """torch.cuda.device(device), or nothing when `device` is already current: the library
    selects the device itself, and the guard only restores the caller's afterwards."""
    import contextlib
    import torch
    if torch.cuda.current_device() == device.index:
        return contextlib.nullcontext()
    return torch.cuda.device(device)


def _on(stream):
    """Makes `stream` torch's current stream (no-op for None), so that torch copies made for
    a call are ordered before the library's kernels on that stream."""
    import contextlib
    import torch
    return contextlib.nullcontext() if stream is None else torch.cuda.stream(stream)


def _as_rgba32(img):
    """uint32 [H, W] view of an RGB(A) image (R in the low byte); torch or numpy."""
    import torch
    if isinstance(img, torch.Tensor):
        if img.dtype == torch.uint8 and img.dim() == 3:
            if img.shape[2] == 3:
                img = torch.cat([img, torch.full_like(img[..., :1], 255)], dim=2)
            return img.contiguous().view(torch.int32).squeeze(-1)
        if img.dtype not in (torch.int32,):
            raise TypeError("rgba must be uint8 [H, W, 3|4] or 32-bit [H, W]")
        return img
    a = np.asarray(img)
    if a.dtype == np.uint8 and a.ndim == 3:
        if a.shape[2] == 3:
            a = np.concatenate([a, np.full(a.shape[:2] + (1,), 255, np.uint8)], axis=2)
        return np.ascontiguousarray(a).view(np.uint32)[..., 0]
    if a.dtype not in (np.uint32, np.int32):
        raise TypeError("rgba must be uint8 [H, W, 3|4] or 32-bit [H, W]")
    return a


def unpack_labels(bits: np.ndarray, width: int) -> np.ndarray:
    """uint8 [H, W] labels from the packed rows of GraphCut.labels_packed*."""
    return np.unpackbits(np.asarray(bits), axis=1, count=width, bitorder="little")


class GraphCut:
    """Tiled push-relabel graph cut on one width x height 4-connected grid."""

    def __init__(self, width: int, height: int, device: int = 0, bfs: int | None = None,
                 discharge_iters: int | None = None, initial_relabel: bool | None = None,
                 max_cycles: int | None = None, max_bfs_rounds: int | None = None,
                 use_graph: bool | None = None, arena=None):
        import torch
        self.width, self.height = int(width), int(height)
        self.device = torch.device("cuda", device)
        if bfs is None and discharge_iters is None and initial_relabel is None:
            # the run-time autotuner's choice for this size class on this device
            import autotune
            sched = autotune.default_tuner().schedule(device, self.width, self.height)
            bfs, discharge_iters = sched["pulses_per_relabel"], sched["discharge_iters"]
            initial_relabel = bool(sched["initial_relabel"])
        opts = _gcut.default_opts(device=device, discharge_iters=discharge_iters,
                                  pulses_per_relabel=bfs,
                                  initial_relabel=None if initial_relabel is None else int(initial_relabel),
                                  max_cycles=max_cycles, max_bfs_rounds=max_bfs_rounds,
                                  use_graph=None if use_graph is None else int(use_graph))
        self.opts = opts
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            if arena is None:
                check(lib().gc_create(self.width, self.height, ctypes.byref(opts),
                                      ctypes.byref(h)))
            else:   # (device address, bytes) of caller-owned memory, or a CUDA tensor
                addr, nbytes = ((arena.data_ptr(), arena.numel() * arena.element_size())
                                if hasattr(arena, "data_ptr") else arena)
                check(lib().gc_create_in(self.width, self.height, ctypes.byref(opts),
                                         ctypes.c_void_p(addr), int(nbytes), ctypes.byref(h)))
        self._arena = arena   # the memory must outlive the handle
        self._h = h
        self._solved = False

    @staticmethod
    def arena_bytes(width: int, height: int) -> int:
        """Device bytes of a width x height handle (what `arena=` must provide)."""
        out = ctypes.c_int64()
        check(lib().gc_arena_bytes(int(width), int(height), ctypes.byref(out)))
        return out.value

    def close(self):
        if getattr(self, "_h", None):
            lib().gc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- input ------------------------------------------------------------------
    def upload_capacities(self, up, down, left, right, excess, stream=None):
        """Uploads the capacity planes; torch CUDA tensors are read in place, anything else
        is copied to the device first.  Resets the residual graph."""
        import torch
        planes = (up, down, left, right, excess)
        for p in planes:
            if tuple(p.shape) != (self.height, self.width):
                raise ValueError(f"plane shape {tuple(p.shape)} != {(self.height, self.width)}")
        if all(isinstance(p, torch.Tensor) and p.is_cuda for p in planes):
            if all(p.dtype == torch.int32 and p.device == self.device and p.is_contiguous()
                   for p in planes):
                dev = planes      # read in place: no conversion to order before the kernel
            else:
                with _on(stream):   # conversions are ordered before the upload kernel
                    dev = [_as_i32_device(p, self.device) for p in planes]
            check(lib().gc_upload(self._h, *[ptr(d) for d in dev], stream_handle(stream)))
            self._keep = dev  # the upload kernel reads them asynchronously
        else:
            host = [np.ascontiguousarray(p.cpu().numpy() if isinstance(p, torch.Tensor) else p,
                                         dtype=np.int32) for p in planes]
            with torch.cuda.device(self.device):
                check(lib().gc_upload_host(self._h, *[ptr(a) for a in host], stream_handle(stream)))
        self._solved = False

    def upload_image(self, rgba, excess, stream=None, lamda=None):
        """Builds the capacities on the device from an image and the t-links (gc_upload_rgba):
        n-link = floor(50 * exp(-beta * |dI|^2) + 0.5), beta = 1 / (2 * mean |dI|^2).  With
        `lamda` (an integer, the reference's LAMBDA; 60 in GraphCut.pyx:25) the n-links follow
        the reference's own rule instead, lamda / (0.1 * sqrt(|dI|^2) + 0.05) rounded to the
        nearest integer (gc_upload_rgba_lambda; graphcut.cl:1018-1031).  `rgba` is uint32
        [H, W] (RGBA bytes viewed as uint32) or uint8 [H, W, 3|4]; `excess` int32 [H, W], or a
        pair (fg, bg) of colour models (gmm_tlinks.Mixture) from which the t-links are
        computed on the device (gc_tlinks_gmm, 100 * (score_bg - score_fg) rounded).  Torch
        CUDA tensors are read in place; numpy arrays are copied."""
        import torch
        if lamda is not None and (int(lamda) != lamda or not 1 <= lamda <= 1000):
            raise ValueError("lamda must be an integer in [1, 1000]")
        rgba = _as_rgba32(rgba)
        if isinstance(excess, tuple):
            import gmm_tlinks
            fg, bg = excess
            with _on(stream), torch.cuda.device(self.device):
                if not (isinstance(rgba, torch.Tensor) and rgba.is_cuda):
                    host = rgba.cpu().numpy() if isinstance(rgba, torch.Tensor) else rgba
                    rgba = torch.from_numpy(np.ascontiguousarray(host).view(np.int32)).to(self.device)
                rgba = rgba.contiguous()
                if tuple(rgba.shape) != (self.height, self.width):
                    raise ValueError("image shape differs from the graph")
                excess = gmm_tlinks.tlinks(rgba, fg, bg, stream=stream)
        if tuple(rgba.shape) != (self.height, self.width) or tuple(excess.shape) != (self.height, self.width):
            raise ValueError("image / excess shape differs from the graph")
        if isinstance(rgba, torch.Tensor) and rgba.is_cuda and isinstance(excess, torch.Tensor) and excess.is_cuda:
            with _on(stream):
                ex = _as_i32_device(excess, self.device)
                img = rgba.contiguous()
            if lamda is None:
                check(lib().gc_upload_rgba(self._h, ptr(img), ptr(ex), stream_handle(stream)))
            else:
                check(lib().gc_upload_rgba_lambda(self._h, ptr(img), ptr(ex), int(lamda),
                                                  stream_handle(stream)))
            self._keep = (img, ex)
        else:
            img = np.ascontiguousarray(rgba.cpu().numpy() if isinstance(rgba, torch.Tensor) else rgba)
            ex = np.ascontiguousarray(excess.cpu().numpy() if isinstance(excess, torch.Tensor) else excess,
                                      dtype=np.int32)
            with torch.cuda.device(self.device):
                if lamda is None:
                    check(lib().gc_upload_rgba_host(self._h, ptr(img), ptr(ex),
                                                    stream_handle(stream)))
                else:
                    check(lib().gc_upload_rgba_lambda_host(self._h, ptr(img), ptr(ex),
                                                           int(lamda), stream_handle(stream)))
        self._solved = False

    # ---- solve ------------------------------------------------------------------
    def cut(self, stream=None):
        """Runs push-relabel to the final cut (GraphCut.cut, GraphCut.pyx:348-418)."""
        with _device_guard(self.device):
            check(lib().gc_solve(self._h, stream_handle(stream)))
        self._solved = True
        return self

    def cut_labels(self, out=None, packed=False, stream=None):
        """cut() and labels() (or labels_packed() with packed=True) in one call with one host
        wait: the labels kernel follows the solve on the stream (gc_solve_labels).  Returns
        the label tensor."""
        import torch
        if out is None:
            shape = (self.height, (self.width + 7) // 8) if packed else (self.height, self.width)
            out = torch.empty(shape, dtype=torch.uint8, device=self.device)
        with _device_guard(self.device):
            check(lib().gc_solve_labels(self._h, ptr(out), int(bool(packed)), stream_handle(stream)))
        self._solved = True
        return out

    def push(self, stream=None):
        check(lib().gc_push(self._h, stream_handle(stream)))

    def relabel(self, stream=None):
        check(lib().gc_relabel(self._h, stream_handle(stream)))

    def startBfs(self, stream=None):
        check(lib().gc_start_bfs(self._h, stream_handle(stream)))

    def isCompleted(self, stream=None) -> bool:
        done = ctypes.c_int(0)
        check(lib().gc_is_completed(self._h, ctypes.byref(done), stream_handle(stream)))
        if done.value:
            self._solved = True
        return bool(done.value)

    # ---- results ----------------------------------------------------------------
    @property
    def flow(self) -> int:
        f = ctypes.c_int64(0)
        check(lib().gc_flow(self._h, ctypes.byref(f)))
        return int(f.value)

    def labels(self, out=None, stream=None):
        """Canonical cut: uint8 [H, W] device tensor, 1 = source side."""
        import torch
        if out is None:
            out = torch.empty((self.height, self.width), dtype=torch.uint8, device=self.device)
        check(lib().gc_labels(self._h, ptr(out), stream_handle(stream)))
        return out

    def labels_packed(self, out=None, stream=None):
        """Bit-packed canonical labels as a torch uint8 CUDA tensor [H, (W + 7) // 8]:
        pixel x of a row is bit x % 8 of byte x // 8 (``unpack_labels`` inverts it)."""
        import torch
        if out is None:
            out = torch.empty((self.height, (self.width + 7) // 8), dtype=torch.uint8,
                              device=self.device)
        check(lib().gc_labels_packed(self._h, ptr(out), stream_handle(stream)))
        return out

    def labels_packed_host(self, out=None, stream=None) -> np.ndarray:
        """labels_packed into host memory (numpy; `out` may be a pinned buffer)."""
        if out is None:
            out = np.empty((self.height, (self.width + 7) // 8), np.uint8)
        check(lib().gc_labels_packed_host(self._h, ptr(out), stream_handle(stream)))
        return out

    def labels_host(self, out=None, stream=None) -> np.ndarray:
        """Canonical labels in host memory, uint8 [H, W]; `out` may be a (pinned) buffer of
        that shape, written in place."""
        if out is None:
            out = np.empty((self.height, self.width), np.uint8)
        elif out.shape != (self.height, self.width) or out.dtype != np.uint8 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous uint8 array of shape (height, width)")
        check(lib().gc_labels_host(self._h, ptr(out), stream_handle(stream)))
        return out

    def stats(self) -> dict:
        st = _gcut.GcStats()
        check(lib().gc_get_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def set_profile(self, on: bool):
        """Per-kernel CUDA-event timing and tile counters for the following calls."""
        check(lib().gc_set_profile(self._h, int(on)))

    def profile(self) -> dict:
        return _gcut.kernel_profile(lib().gc_get_profile, self._h)

    def set_trace(self, on: bool, stream=None):
        """Device-side trace of the following solves (gc_set_trace): see trace()."""
        check(lib().gc_set_trace(self._h, int(on), stream_handle(stream)))

    def trace(self, stream=None):
        """[(kernel kind, start ns)] recorded since set_trace(True), in launch order."""
        return _gcut.read_trace(lib().gc_get_trace, self._h, stream)

    def set_collect_stats(self, on: bool):
        check(lib().gc_set_collect_stats(self._h, int(on)))

    # ---- warm start -------------------------------------------------------------
    def edit_tlinks(self, idx, values, stream=None):
        """Sets t-links of pixels idx (flat y*W+x, distinct) to values; warm-starts cut()."""
        import torch
        with _on(stream):   # the copies are ordered before the edit kernel
            idx = torch.as_tensor(np.asarray(idx.cpu() if isinstance(idx, torch.Tensor) else idx),
                                  dtype=torch.int32).to(self.device).contiguous()
            vals = torch.as_tensor(np.asarray(values.cpu() if isinstance(values, torch.Tensor) else values),
                                   dtype=torch.int32).to(self.device).contiguous()
        if idx.numel() != vals.numel():
            raise ValueError("idx and values differ in length")
        check(lib().gc_edit_tlinks(self._h, ptr(idx), ptr(vals), int(idx.numel()),
                                   stream_handle(stream)))
        self._keep_edit = (idx, vals)
        self._solved = False

    def edit_stroke(self, xs, ys, radius: int, value: int, stream=None):
        """Every pixel within `radius` of the polyline gets t-link `value` (device raster)."""
        xs = np.ascontiguousarray(xs, dtype=np.int32)
        ys = np.ascontiguousarray(ys, dtype=np.int32)
        if xs.shape != ys.shape or xs.ndim != 1:
            raise ValueError("xs and ys must be 1-D arrays of the same length")
        check(lib().gc_edit_stroke(self._h, ptr(xs), ptr(ys), int(xs.shape[0]), int(radius),
                                   int(value), stream_handle(stream)))
        self._solved = False

    def edit_brush(self, xs, ys, radius: int, value: int, stream=None):
        """Every pixel the reference Brush covers for the polyline (brush.pyx:138-161: line
        pixels widened by the disc of the radius, centred; pixels outside the image skipped)
        gets t-link `value`; warm-starts cut()."""
        xs = np.ascontiguousarray(xs, dtype=np.int32)
        ys = np.ascontiguousarray(ys, dtype=np.int32)
        if xs.shape != ys.shape or xs.ndim != 1:
            raise ValueError("xs and ys must be 1-D arrays of the same length")
        check(lib().gc_edit_brush(self._h, ptr(xs), ptr(ys), int(xs.shape[0]), int(radius),
                                  int(value), stream_handle(stream)))
        self._solved = False

    # ---- read-only planes (GraphCut.pyx:57-79) ----------------------------------
    def _plane(self, which: int):
        import torch
        out = torch.empty((self.height, self.width), dtype=torch.int32, device=self.device)
        args = [None] * 6
        args[which] = ptr(out)
        check(lib().gc_download_state(self._h, *args, stream_handle(None)))
        return out

    _PLANES = {"excess": 0, "height": 1, "up": 2, "down": 3, "left": 4, "right": 5}

    def execute(self, input):
        """GraphCut.execute (GraphCut.pyx:423-437, filter_transpose graphcut.cl:1134-1170): the
        reference turns one of its planes (its left / right capacities are stored
        tile-transposed) into image layout as float32 for display.  Every plane here
        (dExcess, dHeight, dUp, dDown, dLeft, dRight) is already in image layout, so this
        returns `input` as a float32 [H, W] device tensor; a plane name ("excess", "height",
        "up", "down", "left", "right") reads that plane first."""
        import torch
        if isinstance(input, str):
            if input not in self._PLANES:
                raise ValueError(f"plane must be one of {sorted(self._PLANES)}")
            input = self._plane(self._PLANES[input])
        if tuple(input.shape) != (self.height, self.width):
            raise ValueError(f"plane shape {tuple(input.shape)} != {(self.height, self.width)}")
        return torch.as_tensor(input, device=self.device).to(torch.float32)

    @property
    def dExcess(self):
        return self._plane(0)

    @property
    def dHeight(self):
        return self._plane(1)

    @property
    def dUp(self):
        return self._plane(2)

    @property
    def dDown(self):
        return self._plane(3)

    @property
    def dLeft(self):
        return self._plane(4)

    @property
    def dRight(self):
        return self._plane(5)
