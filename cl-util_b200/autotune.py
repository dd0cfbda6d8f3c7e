"""Autotuner for the solver schedule.

Knobs: discharge iterations inside a tile per launch, discharge launches (pulses) between
global relabels, and whether the solve starts with an exact global relabel.  The tile is
fixed at 32x32 pixels: a warp row is one 128-byte line of a plane and the BFS works on
32-bit row masks, so other shapes would change the data layout, not a launch parameter.

Every candidate schedule is timed on full solves of sample grids (inputs resident on the
device, CUDA events on the solver's stream) and must give the same flow value and the same
canonical cut as every other candidate; the fastest is returned.

    python cl-util_b200/autotune.py [--size 2048] [--seed 1000] [--batch 0]
"""
from __future__ import annotations

import argparse
import itertools
import json
import sys

DEFAULT_GRID = {
    "discharge_iters": [1, 2, 3, 4, 8, 16],
    "pulses_per_relabel": [1, 2, 4, 6, 8, 12],
    "initial_relabel": [0, 1],
}


def _solve_time(make, planes_list, repeats, torch):
    solver = make()
    stream = torch.cuda.Stream()
    results = None
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


def tune(graphs, grid=None, repeats=3, device=0, batch=None, verbose=False):
    """Returns (best option dict, table of {opts, ms}).  `graphs` are synth.Graph objects;
    with batch=True they are solved together in one pool."""
    import torch

    from GraphCut import GraphCut
    from GraphCutBatch import GraphCutBatch
    grid = dict(DEFAULT_GRID, **(grid or {}))
    batch = len(graphs) > 1 if batch is None else batch
    dev = torch.device("cuda", device)
    planes_list = [[torch.from_numpy(p).to(dev) for p in g.planes()] for g in graphs]
    table, ref = [], None
    keys = list(grid)
    for combo in itertools.product(*(grid[k] for k in keys)):
        o = dict(zip(keys, combo))
        kw = dict(device=device, bfs=o["pulses_per_relabel"], discharge_iters=o["discharge_iters"],
                  initial_relabel=bool(o["initial_relabel"]))
        if batch:
            make = lambda kw=kw: GraphCutBatch([(g.width, g.height) for g in graphs], **kw)
        else:
            make = lambda kw=kw: GraphCut(graphs[0].width, graphs[0].height, **kw)
        ms, res = _solve_time(make, planes_list, repeats, torch)
        if ref is None:
            ref = res
        else:
            for (f0, l0), (f1, l1) in zip(ref, res):
                if f0 != f1 or not torch.equal(l0, l1):
                    raise RuntimeError(f"schedule {o} changed the result: flow {f1} vs {f0}")
        table.append({"opts": o, "ms": ms})
        if verbose:
            print(json.dumps(table[-1]), file=sys.stderr, flush=True)
    best = min(table, key=lambda r: r["ms"])
    return best["opts"], table


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
