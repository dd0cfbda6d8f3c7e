"""SolvePipeline: a stream of same-size images from host memory to flows and cuts, with the
host<->device copies of one image overlapping the solve of the previous one.

The reference solves one image at a time with blocking calls (test_GraphCut.py:78-99).  A
caller that feeds a sequence of frames (video, a batch of photos, a server's queue of one
size class) pays the PCIe copy of every frame on top of its solve.  Here one solver handle
and one compute stream run the uploads, solves and label packing in order, while a second
stream copies the next frame's RGBA image and t-links from pinned host memory into one of
two device staging slots, and copies the previous frame's packed labels back:

    pipe = SolvePipeline(width, height)
    for flow, bits in pipe.run(frames):      # frames: (rgba uint32 [H, W], excess int32 [H, W])
        ...                                  # bits: packed labels, GraphCut.unpack_labels(bits, W)

A frame may carry two colour models instead of the t-links, (rgba, (fg, bg)) with
gmm_tlinks.Mixture models: then only the image is copied (4 bytes per pixel) and the t-links
are computed on the device (gc_tlinks_gmm), as the reference scores the image under its
models on the device before the cut (GMM.score, test_GraphCut.py:44-47).

Only copies overlap kernels; the solver's kernels never run concurrently with each other.
Frames should be in pinned host memory (``torch.empty(..., pin_memory=True).numpy()``) for the
copies to be asynchronous; pageable arrays work, with the copy done on the calling thread.
"""
from __future__ import annotations

import numpy as np

from GraphCut import GraphCut, _as_rgba32


class SolvePipeline:
    def __init__(self, width: int, height: int, device: int = 0, lamda=None, **solver_kw):
        import torch
        self.torch = torch
        self.width, self.height = int(width), int(height)
        self.lamda = lamda
        self.dev = torch.device("cuda", device)
        self.gc = GraphCut(width, height, device=device, **solver_kw)
        with torch.cuda.device(self.dev):
            self.compute = torch.cuda.Stream(self.dev)
            self.copy = torch.cuda.Stream(self.dev)
            n = self.width * self.height
            nb = self.height * ((self.width + 7) // 8)
            self.stage_img = [torch.empty((self.height, self.width), dtype=torch.int32,
                                          device=self.dev) for _ in range(2)]
            self.stage_exc = [torch.empty((self.height, self.width), dtype=torch.int32,
                                          device=self.dev) for _ in range(2)]
            self.dbits = [torch.empty((self.height, (self.width + 7) // 8), dtype=torch.uint8,
                                      device=self.dev) for _ in range(2)]
            self.hbits = [torch.empty(nb, dtype=torch.uint8, pin_memory=True)
                          .view(self.height, (self.width + 7) // 8) for _ in range(2)]
            ev = lambda: torch.cuda.Event()   # noqa: E731
            self.copied = [ev() for _ in range(2)]     # inputs of the slot are on the device
            self.consumed = [ev() for _ in range(2)]   # the upload kernel has read the slot
            self.packed = [ev() for _ in range(2)]     # packed labels of the slot are ready
            self.landed = [ev() for _ in range(2)]     # packed labels are in host memory
            for e in self.consumed + self.landed:
                e.record(self.compute)
        self.models = [None, None]
        self._n = n

    def _host_i32(self, a):
        torch = self.torch
        if isinstance(a, torch.Tensor):
            return a if a.dtype == torch.int32 else a.view(torch.int32)
        a = np.ascontiguousarray(a)
        if a.dtype == np.uint32:
            a = a.view(np.int32)
        return torch.from_numpy(a)

    def _copy_in(self, j, rgba, excess):
        """Queues the host->device copies of one frame into slot j (after the slot's last
        upload has read it); colour models stay on the host until the t-links are built."""
        rgba = _as_rgba32(rgba)
        models = isinstance(excess, tuple)
        if tuple(rgba.shape) != (self.height, self.width) or \
                (not models and tuple(excess.shape) != (self.height, self.width)):
            raise ValueError("frame shape differs from the pipeline's")
        with self.torch.cuda.stream(self.copy):
            self.copy.wait_event(self.consumed[j])
            self.stage_img[j].copy_(self._host_i32(rgba), non_blocking=True)
            if not models:
                self.stage_exc[j].copy_(self._host_i32(excess), non_blocking=True)
            self.copied[j].record(self.copy)
        self.models[j] = excess if models else None

    def run(self, frames):
        """Yields (flow, packed labels) for every (rgba, excess) frame, in order.  The packed
        labels are a fresh numpy array [H, (W + 7) // 8] (pixel x in bit x % 8 of byte x // 8)."""
        torch = self.torch
        it = iter(frames)
        nxt = next(it, None)
        k = 0
        pending = None   # (slot, flow) whose labels are on their way to the host
        with torch.cuda.device(self.dev):
            if nxt is not None:
                self._copy_in(0, *nxt)
            while nxt is not None:
                j = k & 1
                following = next(it, None)
                if following is not None:
                    self._copy_in(j ^ 1, *following)   # overlaps this frame's solve
                with torch.cuda.stream(self.compute):
                    self.compute.wait_event(self.copied[j])
                    self.compute.wait_event(self.landed[j])   # dbits[j] / hbits[j] are free
                    if self.models[j] is not None:            # t-links from the two models
                        import gmm_tlinks
                        gmm_tlinks.tlinks(self.stage_img[j], *self.models[j],
                                          out=self.stage_exc[j], stream=self.compute)
                    self.gc.upload_image(self.stage_img[j], self.stage_exc[j], stream=self.compute,
                                         lamda=self.lamda)
                    self.consumed[j].record(self.compute)
                    # returns when the solve and the packed labels are done (one host wait)
                    self.gc.cut_labels(out=self.dbits[j], packed=True, stream=self.compute)
                    flow = self.gc.flow
                    self.packed[j].record(self.compute)
                with torch.cuda.stream(self.copy):
                    self.copy.wait_event(self.packed[j])
                    self.hbits[j].copy_(self.dbits[j], non_blocking=True)
                    self.landed[j].record(self.copy)
                if pending is not None:
                    pj, pflow = pending
                    self.landed[pj].synchronize()
                    yield pflow, self.hbits[pj].numpy().copy()
                pending = (j, flow)
                nxt = following
                k += 1
            if pending is not None:
                pj, pflow = pending
                self.landed[pj].synchronize()
                yield pflow, self.hbits[pj].numpy().copy()

    def close(self):
        self.gc.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
