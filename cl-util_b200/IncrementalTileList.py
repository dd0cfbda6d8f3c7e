"""IncrementalTileList on libgcut's single-pass scan; StreamCompact and PrefixSum live in
their own modules, as in the reference, and are re-exported here.

A mirror of the reference class beneath GraphCut (IncrementalTileList.pyx:26-208) with the
same method names and argument meaning.  Buffers are torch int32 CUDA tensors; every
build / compact / scan is one kernel launch (decoupled look-back) instead of the
reference's flag + copy + 1-3 scan launches + scatter.  Each object owns its look-back
state (as each reference object owns its buffers), so objects on different streams do not
interfere; a look-back error of an earlier call raises GCError at the next call, and a
compacted length of -1 (a wait that gave up) raises when `length` is read.
"""
from __future__ import annotations

import _gcut
from _gcut import ScanState, check, lib, ptr, stream_handle
from PrefixSum import PrefixSum, _i32  # noqa: F401  (PrefixSum re-exported)
from StreamCompact import StreamCompact  # noqa: F401  (re-exported)


class Operator:
    """Stamp comparisons (IncrementalTileList.pyx:26-31)."""
    EQUAL = 0
    GT = 1
    LT = 2
    GTE = 3
    LTE = 4


class Logical:
    """Combination of two predicates (IncrementalTileList.pyx:33-35)."""
    AND = 0
    OR = 1


class IncrementalTileList:
    """Per-tile iteration stamps and the compacted list of tiles matching a predicate
    (IncrementalTileList.pyx:37-208)."""

    def __init__(self, global_dim, tiles_dim, device=0):
        import torch
        self.global_dim = tuple(int(v) for v in global_dim)
        self.tiles_dim = tuple(int(v) for v in tiles_dim)
        self.dim = (self.global_dim[0] // self.tiles_dim[0], self.global_dim[1] // self.tiles_dim[1])
        self.device = torch.device("cuda", device) if isinstance(device, int) else device
        n = self.dim[0] * self.dim[1]
        self.d_tiles = torch.zeros((self.dim[1], self.dim[0]), dtype=torch.int32, device=self.device)
        self.state = ScanState(self.device.index or 0, n)
        self.d_list = _i32(n, self.device)
        self.d_length = _i32(1, self.device)
        self.init_iteration = -1
        self.is_dirty = True
        self._length = 0
        self.reset()

    @property
    def n_tiles(self) -> int:
        return self.dim[0] * self.dim[1]

    @property
    def length(self) -> int:
        """Number of tiles in d_list (one device->host read when dirty)."""
        if self.is_dirty:
            n = int(self.d_length[0].item())
            if n < 0:
                raise _gcut.GCError(_gcut.GC_ERR_INTERNAL, "the tile-list compaction gave up "
                                    f"a bounded look-back wait (error {self.state.error()})")
            self._length = n
            self.is_dirty = False
        return self._length

    def increment(self) -> int:
        self.iteration += 1
        return self.iteration

    def build(self, operator=None, operand=None, stream=None):
        """d_list = row-major ids of tiles with `stamp operator operand` (default: EQUAL to
        the current iteration)."""
        if operator is None:
            operator = Operator.EQUAL
        if operand is None:
            operand = self.iteration
        check(lib().gc_tiles_build(self.state.handle, ptr(self.d_tiles), int(operator),
                                   int(operand), ptr(self.d_list), ptr(self.d_length),
                                   self.n_tiles, stream_handle(stream)))
        self.is_dirty = True

    def incorporate(self, d_tiles2, operator1, operand1, operator2, operand2, logical,
                    stream=None):
        """Stamps the current iteration where (stamp op1 a1) LOGICAL (tiles2 op2 a2)."""
        check(lib().gc_tiles_incorporate(ptr(self.d_tiles), ptr(d_tiles2), int(operator1),
                                         int(operand1), int(operator2), int(operand2),
                                         int(logical), int(self.iteration), self.n_tiles,
                                         stream_handle(stream)))

    def buildLogical(self, d_tiles2, operator1, operand1, operator2, operand2, logical,
                     stream=None):
        check(lib().gc_tiles_build_logical(self.state.handle, ptr(self.d_tiles),
                                           ptr(d_tiles2), int(operator1), int(operand1),
                                           int(operator2), int(operand2), int(logical),
                                           ptr(self.d_list), ptr(self.d_length), self.n_tiles,
                                           stream_handle(stream)))
        self.is_dirty = True

    def execute(self, out=None, stream=None):
        """The display layer of the list (IncrementalTileList.execute,
        IncrementalTileList.pyx:191-208): 32-bit RGBA words [H, W] on the device, opaque red
        (0xFF0000FF) on the tiles stamped with the current iteration, opaque black elsewhere.
        Written into `out` (a contiguous 32-bit [H, W] tensor) when given."""
        import torch
        w, h = self.global_dim
        if out is None:
            out = torch.empty((h, w), dtype=torch.int32, device=self.device)
        elif tuple(out.shape) != (h, w) or out.element_size() != 4 or not out.is_contiguous():
            raise ValueError("out must be a contiguous 32-bit [H, W] tensor")
        check(lib().gc_tiles_view(ptr(self.d_tiles), self.dim[0], self.dim[1],
                                  self.tiles_dim[0], self.tiles_dim[1], int(self.iteration),
                                  w, h, ptr(out), stream_handle(stream)))
        return out

    def reset(self, stream=None):
        self.iteration = self.init_iteration + 1
        check(lib().gc_tiles_fill(ptr(self.d_tiles), int(self.init_iteration), self.n_tiles,
                                  stream_handle(stream)))
        self.is_dirty = True
