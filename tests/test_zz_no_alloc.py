"""gc_compact_noalloc: the compaction entry point for callers that cannot allocate.

Callers that must keep a fixed device-memory footprint, or that cannot risk the implicit
synchronisation of cudaMalloc / cudaFree while other work runs on the GPU, use this variant
of gc_compact; its look-back scratch is a fixed array inside the library instead of memory
allocated on first use.  This test calls it through the C ABI and checks that it returns
exactly what gc_compact returns (and the indices of the non-zero flags), on calls in a row
(each finds the previous call's leftovers in the shared array), from an input that fills the
whole array down to an empty one, and that inputs above its stated maximum are refused.  The file name makes pytest collect it after every other test file.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_compact_matches_compact_twice(cuda):
    torch = cuda
    import _gcut
    L = _gcut.lib()
    stream = _gcut.stream_handle()
    rng = np.random.default_rng(2024)
    # calls in a row: the whole array (every chunk in use), then a larger input than the
    # next, then a smaller one with another density, then an empty one
    cases = ((_gcut.GC_COMPACT_NOALLOC_MAX_N, 0.5), (1_000_003, 0.3), (262_147, 0.7), (0, 0.5))
    for n, density in cases:
        flags = (rng.random(n) < density).astype(np.int32)
        d_flags = torch.from_numpy(flags).cuda() if n else torch.zeros(1, dtype=torch.int32, device="cuda")
        ref_list = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
        ref_len = torch.full((1,), -7, dtype=torch.int32, device="cuda")
        got_list = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
        got_len = torch.full((1,), -7, dtype=torch.int32, device="cuda")
        _gcut.check(L.gc_compact(None, _ptr(d_flags), _ptr(ref_list), _ptr(ref_len), n, stream))
        _gcut.check(L.gc_compact_noalloc(_ptr(d_flags), _ptr(got_list), _ptr(got_len), n, stream))
        torch.cuda.synchronize()
        m = int(ref_len.item())
        assert m == int(flags.sum())
        assert int(got_len.item()) == m
        assert torch.equal(got_list[:m], ref_list[:m])
        assert np.array_equal(got_list[:m].cpu().numpy(), np.flatnonzero(flags))


def test_noalloc_compact_rejects_inputs_above_its_maximum(cuda):
    torch = cuda
    import _gcut
    L = _gcut.lib()
    buf = torch.zeros(16, dtype=torch.int32, device="cuda")
    out = torch.zeros(16, dtype=torch.int32, device="cuda")
    length = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = L.gc_compact_noalloc(_ptr(buf), _ptr(out), _ptr(length),
                              _gcut.GC_COMPACT_NOALLOC_MAX_N + 1, _gcut.stream_handle())
    assert rc == _gcut.GC_ERR_INVALID
    assert b"GC_COMPACT_NOALLOC_MAX_N" in L.gc_last_error()
