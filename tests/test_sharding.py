"""Multi-rank host logic on the CPU: the LPT split of a batch over ranks and the reductions
of per-rank timings and checks, run as two gloo processes."""
import os
import socket

import numpy as np
import pytest

from sharding import lpt_assign, reduce_max, reduce_min, reduce_sum


def test_lpt_covers_every_grid_once_and_balances():
    rng = np.random.default_rng(0)
    for n in (1, 2, 3, 8):
        w = [int(x) for x in rng.integers(1, 1000, 64)]
        split = lpt_assign(w, n)
        flat = sorted(i for part in split for i in part)
        assert flat == list(range(64))
        loads = [sum(w[i] for i in part) for part in split]
        # LPT: no rank exceeds the average load by more than the largest single weight
        assert max(loads) <= sum(w) / n + max(w)
        assert lpt_assign(w, n) == split   # deterministic


def test_lpt_more_ranks_than_grids():
    split = lpt_assign([5, 3], 4)
    assert split == [[0], [1], [], []]


def test_lpt_rejects_no_ranks():
    with pytest.raises(ValueError):
        lpt_assign([1], 0)


def test_reductions_without_a_process_group():
    assert reduce_max(3.5) == 3.5 and reduce_min(2.0) == 2.0 and reduce_sum(1.0) == 1.0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        sizes = [w * h for w, h in [(256, 384), (1536, 1024), (512, 512), (1280, 256),
                                    (768, 1536), (384, 384), (1024, 1024)]]
        mine = lpt_assign(sizes, world)[rank]
        # each rank times its own share (here: pixels as a stand-in for milliseconds)
        ms = float(sum(sizes[i] for i in mine))
        res = (reduce_max(ms), reduce_min(1.0 if rank != 0 else 0.0), reduce_sum(len(mine)))
        out.put((rank, mine, res))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_and_reduce():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    (r0, mine0, res0), (r1, mine1, res1) = results
    assert sorted(mine0 + mine1) == list(range(7)) and not set(mine0) & set(mine1)
    sizes = [w * h for w, h in [(256, 384), (1536, 1024), (512, 512), (1280, 256),
                                (768, 1536), (384, 384), (1024, 1024)]]
    loads = [sum(sizes[i] for i in m) for m in (mine0, mine1)]
    assert res0 == res1 == (float(max(loads)), 0.0, 7.0)
