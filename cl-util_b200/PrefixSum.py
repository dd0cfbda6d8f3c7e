"""PrefixSum on libgcut's single-pass scan (PrefixSum.pyx:121-226, prefixsum.cl).

The reference's exclusive int32 scan with the same method names, argument meaning and
ValueError on capacity overflow.  Buffers are torch int32 CUDA tensors, and a scan is one
kernel launch (decoupled look-back) instead of the reference's 1-3 launches.  Each object
owns its look-back state (as each reference object owns its buffers), so objects on
different streams do not interfere; a look-back error of an earlier call raises GCError at
the next call.
"""
from __future__ import annotations

from _gcut import ScanState, check, lib, ptr, stream_handle


def _i32(n, device):
    import torch
    return torch.zeros(max(1, n), dtype=torch.int32, device=device)


def _pow2gt(x: int) -> int:
    """Smallest power of two >= x (clutil.pyx:15-20)."""
    i = 1
    while i < x:
        i <<= 1
    return i


class PrefixSum:
    """Exclusive int32 scan (PrefixSum.pyx:121-226, prefixsum.cl)."""

    def __init__(self, capacity: int, device=0):
        import torch
        self.capacity = int(capacity)
        self.device = torch.device("cuda", device) if isinstance(device, int) else device
        self.state = ScanState(self.device.index or 0, self.capacity)

    def factory(self, length=None):
        """A scan buffer; its size is rounded up to a power of two (PrefixSum.pyx:168-176)."""
        if length is None:
            length = self.capacity
        elif length > self.capacity:
            raise ValueError(f"length > self.capacity: {length}, {self.capacity}")
        return _i32(_pow2gt(length), self.device)

    def scan(self, dArray, dTotal, length=None, stream=None):
        """In-place exclusive scan of dArray[:length]; the sum goes to dTotal[0]."""
        if length is None:
            length = dArray.numel()
        if length > self.capacity:
            raise ValueError(f"length > self.capacity: {length}, {self.capacity}")
        check(lib().gc_scan_exclusive(self.state.handle, ptr(dArray), ptr(dArray), ptr(dTotal),
                                      int(length), stream_handle(stream)))
