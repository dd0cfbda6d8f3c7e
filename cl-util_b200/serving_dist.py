"""Serving on several GPUs of one node: one process per GPU, each with its own GraphCutServer,
and sessions sticky to the GPU that holds their residual graph.

Rank 0 is the front end.  A new image is placed on the rank with the fewest resident
pixels (``SessionRouter``); every later request of that session goes to the same rank, since
its heights, flow and t-links live in that GPU's memory.  Requests for other ranks are
forwarded as small host messages (``torch.distributed`` point-to-point object messages; gloo
or NCCL process group alike); nothing of the solve crosses between GPUs.  At the end every
rank drains its server and the results are gathered on rank 0, each tagged with the rank
that served it.

    with DistributedServer(lambda: GraphCutServer(hbm_budget=...)) as ds:
        if ds.rank == 0:
            for req in requests: ds.submit(req)
        results = ds.finish()          # rank 0: every result; other ranks: []
"""
from __future__ import annotations

import threading

from serving import NewImage, Stroke


class SessionRouter:
    """Placement of sessions on ranks: a new session goes to the rank with the smallest
    resident load (pixels of the sessions placed there; ties to the lower rank) and stays
    there.  Host bookkeeping only, deterministic."""

    def __init__(self, world: int):
        if world < 1:
            raise ValueError("world must be >= 1")
        self.load = [0] * world
        self.owner = {}       # session -> rank
        self.pixels = {}      # session -> pixels

    def place(self, session, pixels: int) -> int:
        if session in self.owner:
            return self.owner[session]
        r = min(range(len(self.load)), key=lambda k: (self.load[k], k))
        self.owner[session] = r
        self.pixels[session] = int(pixels)
        self.load[r] += int(pixels)
        return r

    def route(self, session):
        """The rank holding the session, or None for a session never placed."""
        return self.owner.get(session)

    def release(self, session):
        """The session left its GPU (closed or evicted): its pixels leave the rank's load."""
        r = self.owner.pop(session, None)
        if r is not None:
            self.load[r] -= self.pixels.pop(session)


_STOP = "stop"


class DistributedServer:
    """One server per rank of the default process group (see the module docstring)."""

    def __init__(self, make_server, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.server = make_server()
        self.router = SessionRouter(self.world) if self.rank == 0 else None
        self.forwarded = 0
        self._rx = None
        if self.rank != 0:
            self._rx = threading.Thread(target=self._receive, daemon=True)
            self._rx.start()

    def _receive(self):
        while True:
            box = [None]
            self.dist.recv_object_list(box, src=0, group=self.group)
            msg = box[0]
            if msg == _STOP:
                return
            req, arrival = msg
            self.server.submit(req, arrival=arrival)

    def submit(self, request, arrival=None):
        """Rank 0: routes one request to the rank that holds (or will hold) its session."""
        if self.rank != 0:
            raise RuntimeError("requests enter at rank 0")
        if isinstance(request, NewImage):
            h, w = request.shape
            r = self.router.place(request.session, w * h)
        elif isinstance(request, Stroke):
            r = self.router.route(request.session)
            if r is None:   # never opened: rank 0's server counts the miss
                r = 0
        else:
            raise TypeError("request must be a NewImage or a Stroke")
        if r == 0:
            self.server.submit(request, arrival=arrival)
        else:
            self.dist.send_object_list([(request, arrival)], dst=r, group=self.group)
            self.forwarded += 1

    def finish(self, timeout=600.0):
        """Every rank: ends the request stream, drains its server and sends its results to
        rank 0, which returns them all as (rank, Result) pairs; other ranks return []."""
        if self.rank == 0:
            for r in range(1, self.world):
                self.dist.send_object_list([_STOP], dst=r, group=self.group)
        elif self._rx is not None:
            self._rx.join()
        self.server.drain(timeout)
        mine = [(self.rank, res) for res in self.server.results]
        counters = {"misses": self.server.misses, "evictions": self.server.evictions}
        out = [None] * self.world if self.rank == 0 else None
        self.dist.gather_object((mine, counters), out, dst=0, group=self.group)
        if self.rank != 0:
            return []
        self.counters = [c for _, c in out]
        return [x for part, _ in out for x in part]

    def close(self):
        self.server.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
