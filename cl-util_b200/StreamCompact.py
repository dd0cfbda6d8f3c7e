"""StreamCompact on libgcut's single-pass scan (StreamCompact.pyx:22-82, streamcompact.cl).

The reference's compaction of int32 flags into the list of flagged indices, with the same
method names, argument meaning and ValueError on capacity overflow.  One kernel launch per
compaction (the scan and the scatter together) instead of the reference's copy + scan +
scatter, and the list never aliases the flags (the reference's in-place aliasing,
StreamCompact.pyx:77-81, is not kept).  Each object owns its look-back state.
"""
from __future__ import annotations

from _gcut import ScanState, check, lib, ptr, stream_handle
from PrefixSum import _i32, _pow2gt


class StreamCompact:
    """Stream compaction of int32 flags (StreamCompact.pyx:22-82)."""

    def __init__(self, capacity: int, device=0):
        import torch
        self.capacity = int(capacity)
        self.device = torch.device("cuda", device) if isinstance(device, int) else device
        self.state = ScanState(self.device.index or 0, self.capacity)

    def flagFactory(self, length=None):
        if length is None:
            length = self.capacity
        elif length > self.capacity:
            raise ValueError(f"length > self.capacity: {length}, {self.capacity}")
        return _i32(length, self.device)

    def listFactory(self, length=None):
        if length is None:
            length = self.capacity
        elif length > self.capacity:
            raise ValueError(f"length > self.capacity: {length}, {self.capacity}")
        return _i32(_pow2gt(length), self.device)

    def compact(self, dFlags, dList, dLength, length=None, stream=None):
        """dList[:n] = indices of the non-zero flags (increasing), dLength[0] = n."""
        if length is None:
            length = dFlags.numel()
        elif length > self.capacity:
            raise ValueError(f"length > self.capacity: {length}, {self.capacity}")
        check(lib().gc_compact(self.state.handle, ptr(dFlags), ptr(dList), ptr(dLength),
                               int(length), stream_handle(stream)))
