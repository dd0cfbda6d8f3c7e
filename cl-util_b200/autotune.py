"""Autotuner for the solver schedule, used at run time by GraphCut and GraphCutBatch.

Knobs: discharge iterations inside a tile per launch, discharge launches (pulses) between
global relabels, and whether the solve starts with an exact global relabel.  The tile is
fixed at 32x32 pixels: a warp row is one 128-byte line of a plane and the BFS works on
32-bit row masks, so other shapes would change the data layout, not a launch parameter.

A schedule is chosen per device and per size class (grids are grouped by pixel count, a
batch by the pixel count of the whole pool):

* ``Autotuner.schedule(device, width, height)`` returns the cached choice for the class, or
  the built-in default when the class was never tuned on this device;
* ``Autotuner.ensure(...)`` tunes the class when it has no cached choice: every candidate
  schedule solves the same sample grid(s) (a synthetic grid of the class's representative
  size, or the caller's planes), all candidates must give the same flow value and canonical
  cut, and the fastest (CUDA events on the solver's stream, inputs resident) is kept;
* choices are cached in memory and in a JSON file keyed by the device (name and SM count),
  ``$GCUT_TUNE_CACHE`` or ``~/.cache/gcut/schedules.json``, so later processes reuse them.

GraphCut / GraphCutBatch ask ``default_tuner().schedule(...)`` when no schedule argument is
given.  Offline: ``python cl-util_b200/autotune.py [--size 2048] [--batch 0]`` tunes one
class on the full grid and prints the table.
"""
from __future__ import annotations

import argparse
import itertools
import json
import os
import sys
import threading

KNOBS = ("discharge_iters", "pulses_per_relabel", "initial_relabel")

# the full offline grid and the smaller one tuned at run time
DEFAULT_GRID = {
    "discharge_iters": [1, 2, 3, 4, 8, 16],
    "pulses_per_relabel": [1, 2, 4, 6, 8, 12],
    "initial_relabel": [0, 1],
}
RUNTIME_GRID = {
    "discharge_iters": [2, 3, 4, 6],
    "pulses_per_relabel": [1, 2, 4],
    "initial_relabel": [0, 1],
}

# size classes by pixel count (upper bounds, inclusive) with a representative square side
SIZE_CLASSES = ((1 << 18, 384), (1 << 20, 768), (1 << 22, 1536), (None, 4096))

# built-in choices (offline tuning on synthetic grids) used until a class is tuned: one grid
# 3 x 2 is the best candidate at 2048^2 (0.257 ms against 0.281 for 4 x 2, upload and solve
# of seed 1000) and at 4096^2 (1.09 ms against 1.21 for 4 x 2; 4 x 1 is not among the best
# six), and within a few
# percent of the best on smaller grids; pools of many grids 4 x 2 (the pool choice depends on
# the instance: on one sample of 64 grids of 256^2 to 1536^2 the tuner preferred 3 x 4, 8.82
# against 10.57 ms, while the benchmark's 64 grids take 5.97 ms with 3 x 4 and 5.33 with 4 x 2)
BUILTIN = {
    "single": [dict(discharge_iters=3, pulses_per_relabel=2, initial_relabel=0)] * 4,
    "batch": [dict(discharge_iters=4, pulses_per_relabel=2, initial_relabel=0)] * 4,
}


def size_class(pixels: int) -> int:
    for k, (hi, _) in enumerate(SIZE_CLASSES):
        if hi is None or pixels <= hi:
            return k
    return len(SIZE_CLASSES) - 1


def _solve_time(make, planes_list, repeats, torch):
    solver = make()
    stream = torch.cuda.Stream()
    times = []
    with torch.cuda.stream(stream):
        for rep in range(repeats + 1):
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            if hasattr(solver, "shapes"):
                for i, planes in enumerate(planes_list):
                    solver.upload(i, *planes, stream=stream)
            else:
                solver.upload_capacities(*planes_list[0], stream=stream)
            solver.cut(stream=stream)
            ev1.record(stream)
            ev1.synchronize()
            if rep:
                times.append(ev0.elapsed_time(ev1))
        if hasattr(solver, "shapes"):
            results = [(solver.flow(i), solver.labels(i).cpu()) for i in range(len(solver))]
        else:
            results = [(solver.flow, solver.labels().cpu())]
    solver.close()
    return min(times), results


def _same(a, b):
    import torch
    return all(f0 == f1 and torch.equal(l0, l1) for (f0, l0), (f1, l1) in zip(a, b))


def tune(graphs, grid=None, repeats=3, device=0, batch=None, verbose=False, planes=None,
         runner=None):
    """Times every schedule of `grid` on `graphs` (synth.Graph objects, or `planes`: lists of
    the five device planes with (width, height) from `graphs`) and returns (best option
    dict, table of {opts, ms}).  With batch=True the grids are solved together in one pool.
    Raises RuntimeError when two schedules give different results.  `runner(opts)` replaces
    the device timing ((ms, results) per candidate; used by host-side tests)."""
    grid = dict(DEFAULT_GRID if grid is None else grid)
    batch = len(graphs) > 1 if batch is None else batch
    if runner is None:
        import torch

        from GraphCut import GraphCut
        from GraphCutBatch import GraphCutBatch
        dev = torch.device("cuda", device)
        if planes is None:
            planes = [[torch.from_numpy(p).to(dev) for p in g.planes()] for g in graphs]
        shapes = [(g.width, g.height) for g in graphs]

        def runner(o):
            kw = dict(device=device, bfs=o["pulses_per_relabel"],
                      discharge_iters=o["discharge_iters"],
                      initial_relabel=bool(o["initial_relabel"]))
            if batch:
                make = lambda: GraphCutBatch(shapes, **kw)   # noqa: E731
            else:
                make = lambda: GraphCut(shapes[0][0], shapes[0][1], **kw)   # noqa: E731
            return _solve_time(make, planes, repeats, torch)
        same = _same
    else:
        def same(a, b):
            return a == b
    table, ref = [], None
    keys = list(grid)
    for combo in itertools.product(*(grid[k] for k in keys)):
        o = dict(zip(keys, combo))
        ms, res = runner(o)
        if ref is None:
            ref = res
        elif not same(ref, res):
            raise RuntimeError(f"schedule {o} changed the result")
        table.append({"opts": o, "ms": ms})
        if verbose:
            print(json.dumps(table[-1]), file=sys.stderr, flush=True)
    best = min(table, key=lambda r: r["ms"])
    return best["opts"], table


def device_key(device: int) -> str:
    import torch
    p = torch.cuda.get_device_properties(device)
    return f"{p.name}/{p.multi_processor_count}sm"


class Autotuner:
    """Per-device, per-size-class schedule choices (see the module docstring)."""

    def __init__(self, cache_path: str | None = None, grid=None, repeats: int = 2,
                 runner_factory=None, device_key_fn=None):
        if cache_path is None:
            cache_path = os.environ.get("GCUT_TUNE_CACHE") or os.path.join(
                os.path.expanduser("~"), ".cache", "gcut", "schedules.json")
        self.cache_path = cache_path
        self.grid = dict(RUNTIME_GRID if grid is None else grid)
        self.repeats = repeats
        self.runner_factory = runner_factory      # (device, kind, shapes, planes) -> runner
        self.device_key_fn = device_key_fn or device_key
        self.tunings = 0                          # classes tuned by this object
        self._lock = threading.Lock()
        self._cache = self._load()

    def _load(self) -> dict:
        try:
            with open(self.cache_path) as f:
                data = json.load(f)
            return data if isinstance(data, dict) else {}
        except (OSError, ValueError):
            return {}

    def _save(self):
        try:
            os.makedirs(os.path.dirname(self.cache_path) or ".", exist_ok=True)
            tmp = f"{self.cache_path}.{os.getpid()}.tmp"
            with open(tmp, "w") as f:
                json.dump(self._cache, f, indent=1, sort_keys=True)
            os.replace(tmp, self.cache_path)
        except OSError:
            pass   # an unwritable cache only costs a re-tune in the next process

    @staticmethod
    def _key(dev_key: str, kind: str, pixels: int) -> str:
        return f"{dev_key}|{kind}|{size_class(pixels)}"

    def cached(self, device: int, pixels: int, kind: str = "single"):
        with self._lock:
            return self._cache.get(self._key(self.device_key_fn(device), kind, pixels))

    def schedule(self, device: int, width: int, height: int, kind: str = "single",
                 pixels: int | None = None) -> dict:
        """The schedule for a grid (or, kind "batch", a pool of `pixels` pixels): the cached
        choice of its class on this device, else the built-in default."""
        px = int(width) * int(height) if pixels is None else int(pixels)
        hit = self.cached(device, px, kind)
        if hit is not None:
            return {k: int(hit[k]) for k in KNOBS}
        return dict(BUILTIN[kind][size_class(px)])

    def ensure(self, device: int, width: int, height: int, kind: str = "single",
               graphs=None, planes=None) -> dict:
        """The class's cached choice; when there is none, tunes it now (on `graphs` /
        `planes` when given, else on a synthetic grid of the class's representative size)
        and caches the result."""
        px = int(width) * int(height) if graphs is None or kind == "single" else \
            sum(g.width * g.height for g in graphs)
        hit = self.cached(device, px, kind)
        if hit is not None:
            return {k: int(hit[k]) for k in KNOBS}
        if graphs is None:
            if kind == "batch":
                raise ValueError("tuning a batch class needs its sample grids")
            import synth
            side = SIZE_CLASSES[size_class(px)][1]
            graphs = [synth.make_graph(side, side, 4242)]
        runner = None
        if self.runner_factory is not None:
            runner = self.runner_factory(device, kind, [(g.width, g.height) for g in graphs],
                                         planes)
        best, table = tune(graphs, grid=self.grid, repeats=self.repeats, device=device,
                           batch=kind == "batch", planes=planes, runner=runner)
        entry = dict(best, ms=min(r["ms"] for r in table), candidates=len(table),
                     sample=[[g.width, g.height] for g in graphs][:4])
        with self._lock:
            self._cache[self._key(self.device_key_fn(device), kind, px)] = entry
            self.tunings += 1
            self._save()
        return {k: int(best[k]) for k in KNOBS}


_default = None
_default_lock = threading.Lock()


def default_tuner() -> Autotuner:
    global _default
    with _default_lock:
        if _default is None:
            _default = Autotuner()
        return _default


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=2048)
    ap.add_argument("--seed", type=int, default=1000)
    ap.add_argument("--batch", type=int, default=0, help="tune a pool of N mixed-size grids")
    ap.add_argument("--repeats", type=int, default=3)
    args = ap.parse_args()
    import synth
    if args.batch:
        shapes = synth.batch_shapes(args.batch, args.seed)
        graphs = [synth.make_graph(w, h, args.seed + i) for i, (w, h) in enumerate(shapes)]
    else:
        graphs = [synth.make_graph(args.size, args.size, args.seed)]
    best, table = tune(graphs, repeats=args.repeats, verbose=True)
    print(json.dumps({"best": best, "ms": min(r["ms"] for r in table), "table": table}))


if __name__ == "__main__":
    main()
