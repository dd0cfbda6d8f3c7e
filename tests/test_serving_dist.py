"""Serving over several GPUs, host logic on the CPU: sticky placement of sessions on ranks
(SessionRouter) and the request forwarding of DistributedServer, run as two gloo processes
with the fake solver of the scheduling tests standing in for each rank's GPU."""
import os
import socket

import numpy as np
import pytest

from serving import NewImage, Stroke
from serving_dist import SessionRouter


def test_router_places_by_load_and_sticks():
    r = SessionRouter(3)
    assert [r.place(s, px) for s, px in [(0, 100), (1, 50), (2, 70), (3, 10)]] == [0, 1, 2, 1]
    assert r.load == [100, 60, 70]
    assert r.place(0, 999) == 0 and r.load[0] == 100     # already placed: sticky, no new load
    assert r.route(2) == 2 and r.route(42) is None
    r.release(0)
    assert r.load == [0, 60, 70] and r.route(0) is None
    assert r.place(4, 5) == 0
    with pytest.raises(ValueError):
        SessionRouter(0)


def _trace(seed=3, n=60):
    """(request) list: 14 sessions of mixed sizes, strokes on open sessions, a stroke on a
    session that never opened."""
    rng = np.random.default_rng(seed)
    reqs, opened = [], []
    for k in range(n):
        if not opened or rng.random() < 0.25:
            sid = len(opened)
            w, h = int(rng.integers(1, 9)) * 32, int(rng.integers(1, 9)) * 32
            t = rng.integers(-5, 6, (h, w)).astype(np.int32)
            reqs.append(NewImage(sid, (t, t, t, t, t)))
            opened.append(sid)
        else:
            sid = int(rng.choice(opened))
            reqs.append(Stroke(sid, np.array([1], np.int32), np.array([1], np.int32), 3,
                               int(rng.integers(1, 100))))
    reqs.append(Stroke(999, np.array([0], np.int32), np.array([0], np.int32), 1, 1))
    return reqs


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
        from serving_dist import DistributedServer
        from test_serving_sched import FakeServer
        ds = DistributedServer(lambda: FakeServer(slots=2, hbm_budget=1 << 30))
        if rank == 0:
            for req in _trace():
                ds.submit(req)
        results = ds.finish(timeout=60)
        if rank == 0:
            out.put(([(r, res.session, res.kind, res.flow) for r, res in results],
                     ds.router.owner, ds.counters, ds.forwarded))
        ds.close()
    finally:
        dist.destroy_process_group()


def test_two_ranks_serve_sessions_sticky_and_same_as_one():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results, owner, counters, forwarded = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    reqs = _trace()
    # every request of an opened session was served, on the rank it was placed on
    n_served = sum(1 for r in reqs if r.session in owner)
    assert len(results) == n_served and forwarded > 0
    assert {s for _, s, _, _ in results} == set(owner)
    for rank, sid, _, _ in results:
        assert rank == owner[sid]
    assert set(owner.values()) == {0, 1}
    # the miss of the never-opened session was counted once, on rank 0
    assert sum(c["misses"] for c in counters) == 1 and counters[0]["misses"] == 1
    # results equal one server's: the fake session state is the running sum of its requests
    from test_serving_sched import FakeServer
    srv = FakeServer(slots=2, hbm_budget=1 << 30)
    for req in reqs:
        srv.submit(req)
    srv.drain(60)
    one = sorted((r.session, r.kind, r.flow) for r in srv.results)
    srv.close()
    assert sorted((s, k, f) for _, s, k, f in results) == one
