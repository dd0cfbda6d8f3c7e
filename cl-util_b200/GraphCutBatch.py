"""Many independent grids solved together in one tile pool (one tile queue over all grids).

    b = GraphCutBatch([(w0, h0), (w1, h1), ...])
    for i, g in enumerate(graphs): b.upload(i, g.up, g.down, g.left, g.right, g.excess)
    b.cut()
    b.flow(i), b.labels(i)

Every kernel launch of the solve covers the active tiles of all grids at once, so small
grids share launches instead of paying one launch sequence each.
"""
from __future__ import annotations

import ctypes

import numpy as np

import _gcut
from _gcut import check, lib, ptr, stream_handle


class GraphCutBatch:
    def __init__(self, shapes, device: int = 0, bfs=None, discharge_iters=None,
                 initial_relabel=None, max_cycles=None, max_bfs_rounds=None,
                 use_graph=None):
        import torch
        self.shapes = [(int(w), int(h)) for (w, h) in shapes]
        self.device = torch.device("cuda", device)
        if discharge_iters is None and bfs is None and initial_relabel is None:
            # the run-time autotuner's choice for a pool of this many pixels on this device
            import autotune
            sched = autotune.default_tuner().schedule(
                device, 0, 0, kind="batch", pixels=sum(w * h for w, h in self.shapes))
            discharge_iters, bfs = sched["discharge_iters"], sched["pulses_per_relabel"]
            initial_relabel = bool(sched["initial_relabel"])
        opts = _gcut.default_opts(device=device, discharge_iters=discharge_iters,
                                  pulses_per_relabel=bfs,
                                  initial_relabel=None if initial_relabel is None else int(initial_relabel),
                                  max_cycles=max_cycles, max_bfs_rounds=max_bfs_rounds,
                                  use_graph=None if use_graph is None else int(use_graph))
        n = len(self.shapes)
        ws = (ctypes.c_int * n)(*[w for w, _ in self.shapes])
        hs = (ctypes.c_int * n)(*[h for _, h in self.shapes])
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            check(lib().gcb_create(n, ws, hs, ctypes.byref(opts), ctypes.byref(h)))
        self._h = h
        self._keep = {}

    def close(self):
        if getattr(self, "_h", None):
            lib().gcb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return len(self.shapes)

    def upload(self, i, up, down, left, right, excess, stream=None):
        import torch
        w, h = self.shapes[i]
        dev = []
        for p in (up, down, left, right, excess):
            if tuple(p.shape) != (h, w):
                raise ValueError(f"plane shape {tuple(p.shape)} != {(h, w)}")
            t = p if isinstance(p, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(p, dtype=np.int32))
            dev.append(t.to(self.device, dtype=torch.int32).contiguous())
        check(lib().gcb_upload(self._h, int(i), *[ptr(d) for d in dev], stream_handle(stream)))
        self._keep[i] = dev

    def cut(self, stream=None):
        import torch
        with torch.cuda.device(self.device):
            check(lib().gcb_solve(self._h, stream_handle(stream)))
        self._keep.clear()
        return self

    def flow(self, i) -> int:
        f = ctypes.c_int64(0)
        check(lib().gcb_flow(self._h, int(i), ctypes.byref(f)))
        return int(f.value)

    def labels(self, i, out=None, stream=None):
        import torch
        w, h = self.shapes[i]
        if out is None:
            out = torch.empty((h, w), dtype=torch.uint8, device=self.device)
        check(lib().gcb_labels(self._h, int(i), ptr(out), stream_handle(stream)))
        return out

    def set_profile(self, on: bool):
        check(lib().gcb_set_profile(self._h, int(on)))

    def profile(self) -> dict:
        return _gcut.kernel_profile(lib().gcb_get_profile, self._h)

    def stats(self) -> dict:
        st = _gcut.GcStats()
        check(lib().gcb_get_stats(self._h, ctypes.byref(st)))
        return st.as_dict()
