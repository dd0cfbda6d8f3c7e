"""ctypes binding of libgcut.so (the C ABI declared in include/gcut.h).

The library must have been built (``python cl-util_b200/gcut_build.py``); loading fails loudly
otherwise - there is no fallback implementation.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgcut.so")

GC_OK, GC_ERR_INVALID, GC_ERR_OOM, GC_ERR_NOT_CONVERGED, GC_ERR_CUDA, GC_ERR_INTERNAL, \
    GC_ERR_STATE = range(7)

ERROR_NAMES = {
    GC_ERR_INVALID: "GC_ERR_INVALID", GC_ERR_OOM: "GC_ERR_OOM",
    GC_ERR_NOT_CONVERGED: "GC_ERR_NOT_CONVERGED", GC_ERR_CUDA: "GC_ERR_CUDA",
    GC_ERR_INTERNAL: "GC_ERR_INTERNAL", GC_ERR_STATE: "GC_ERR_STATE",
}


class GCError(RuntimeError):
    """A non-zero status returned by libgcut."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {message}")
        self.code = code


class GcOpts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("discharge_iters", ctypes.c_int),
                ("pulses_per_relabel", ctypes.c_int), ("initial_relabel", ctypes.c_int),
                ("max_cycles", ctypes.c_int), ("max_bfs_rounds", ctypes.c_int),
                ("use_graph", ctypes.c_int)]


class GcStats(ctypes.Structure):
    _fields_ = [("cycles", ctypes.c_int64), ("pulses", ctypes.c_int64),
                ("bfs_rounds", ctypes.c_int64), ("flood_rounds", ctypes.c_int64),
                ("launches", ctypes.c_int64), ("tiles_discharged", ctypes.c_int64)]

    def as_dict(self):
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


class GcKernelProf(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_int64), ("ms", ctypes.c_double), ("tiles", ctypes.c_int64)]


class GcGauss(ctypes.Structure):
    """One colour-model component: log(w N(x | mean, S)) = c - 0.5 |Li (x - mean)|^2."""
    _fields_ = [("c", ctypes.c_double), ("mean", ctypes.c_double * 3),
                ("li", ctypes.c_double * 6)]


class GcGmmFitResult(ctypes.Structure):
    """gc_gmm_fit's result: the model (covariances as lower triangles) and how the fit ended."""
    _fields_ = [("weights", ctypes.c_double * 8), ("means", (ctypes.c_double * 3) * 8),
                ("covars", (ctypes.c_double * 6) * 8), ("log_likelihood", ctypes.c_double),
                ("iterations", ctypes.c_int32), ("converged", ctypes.c_int32),
                ("status", ctypes.c_int32), ("n_components", ctypes.c_int32),
                ("components", GcGauss * 8)]


GC_NKERN = 10
GC_COMPACT_NOALLOC_MAX_N = 4194304
GC_GMM_MAX_COMPONENTS = 8

_P = ctypes.c_void_p
_I = ctypes.c_int
_I32 = ctypes.c_int32

# name -> argument types (all functions return int unless listed in _RESTYPE)
SIGNATURES = {
    "gc_opts_default": [_P],
    "gc_create": [_I, _I, _P, _P],
    "gc_destroy": [_P],
    "gc_arena_bytes": [_I, _I, _P],
    "gc_create_in": [_I, _I, _P, _P, ctypes.c_int64, _P],
    "gc_size": [_P, _P, _P],
    "gc_upload": [_P] * 6 + [_P],
    "gc_upload_host": [_P] * 6 + [_P],
    "gc_upload_rgba": [_P, _P, _P, _P],
    "gc_upload_rgba_host": [_P, _P, _P, _P],
    "gc_upload_rgba_lambda": [_P, _P, _P, _I32, _P],
    "gc_upload_rgba_lambda_host": [_P, _P, _P, _I32, _P],
    "gc_tlinks_gmm": [_P, _I, _I, _I, _P, _I, _P, _I, ctypes.c_double, _I32, _P, _P],
    "gc_gmm_fit": [_P, _I, _I, _I, ctypes.c_double, ctypes.c_double, ctypes.c_double, _I,
                   _P, _P],
    "gc_solve": [_P, _P],
    "gc_solve_labels": [_P, _P, _I, _P],
    "gc_push": [_P, _P],
    "gc_relabel": [_P, _P],
    "gc_start_bfs": [_P, _P],
    "gc_is_completed": [_P, _P, _P],
    "gc_flow": [_P, _P],
    "gc_labels": [_P, _P, _P],
    "gc_labels_host": [_P, _P, _P],
    "gc_labels_packed": [_P, _P, _P],
    "gc_labels_packed_host": [_P, _P, _P],
    "gc_edit_tlinks": [_P, _P, _P, _I, _P],
    "gc_edit_stroke": [_P, _P, _P, _I, _I, _I32, _P],
    "gc_edit_brush": [_P, _P, _P, _I, _I, _I32, _P],
    "gc_download_state": [_P] * 7 + [_P],
    "gc_get_stats": [_P, _P],
    "gc_set_trace": [_P, _I, _P],
    "gc_get_trace": [_P, _P, _I, _P, _P],
    "gcb_set_trace": [_P, _I, _P],
    "gcb_get_trace": [_P, _P, _I, _P, _P],
    "gcp_set_trace": [_P, _I, _P],
    "gcp_get_trace": [_P, _P, _I, _P, _P],
    "gc_set_collect_stats": [_P, _I],
    "gc_set_profile": [_P, _I],
    "gc_get_profile": [_P, _P, _I],
    "gc_kernel_name": [_I],
    "gc_last_error": [],
    "gc_scan_state_create": [_I, _I, _P],
    "gc_scan_state_destroy": [_P],
    "gc_scan_state_error": [_P, _P, _P],
    "gc_scan_state_selftest": [_P, _I, _P, _P],
    "gc_scan_exclusive": [_P, _P, _P, _P, _I, _P],
    "gc_compact": [_P, _P, _P, _P, _I, _P],
    "gc_compact_noalloc": [_P, _P, _P, _I, _P],
    "gc_tiles_build": [_P, _P, _I, _I32, _P, _P, _I, _P],
    "gc_tiles_build_logical": [_P, _P, _P, _I, _I32, _I, _I32, _I, _P, _P, _I, _P],
    "gc_tiles_incorporate": [_P, _P, _I, _I32, _I, _I32, _I, _I32, _I, _P],
    "gc_tiles_fill": [_P, _I32, _I, _P],
    "gc_tiles_view": [_P, _I, _I, _I, _I, _I32, _I, _I, _P, _P],
    "gc_view_colorize": [_P, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P],
    "gcb_create": [_I, _P, _P, _P, _P],
    "gcb_destroy": [_P],
    "gcb_upload": [_P, _I] + [_P] * 5 + [_P],
    "gcb_solve": [_P, _P],
    "gcb_flow": [_P, _I, _P],
    "gcb_labels": [_P, _I, _P, _P],
    "gcb_get_stats": [_P, _P],
    "gcb_set_profile": [_P, _I],
    "gcb_get_profile": [_P, _P, _I],
    "gcp_arena_bytes": [_I, _I, _P],
    "gcp_create": [_I, _I, _P, _P],
    "gcp_create_in": [_I, _I, _P, _P, ctypes.c_int64, _P],
    "gcp_destroy": [_P],
    "gcp_open": [_P, _I, _I, _I, _I, _P],
    "gcp_close": [_P, _I],
    "gcp_upload": [_P, _I] + [_P] * 5 + [_P],
    "gcp_upload_rgba": [_P, _I, _P, _P, _P],
    "gcp_edit_stroke": [_P, _I, _P, _P, _I, _I, _I32, _P],
    "gcp_edit_brush": [_P, _I, _P, _P, _I, _I, _I32, _P],
    "gcp_solve": [_P, _P, _I, _P],
    "gcp_solve_labels": [_P, _P, _I, _P, _I, _P],
    "gcp_flow": [_P, _I, _P],
    "gcp_labels": [_P, _I, _P, _P],
    "gcp_labels_packed": [_P, _I, _P, _P],
    "gcp_get_stats": [_P, _P],
}
_RESTYPE = {"gc_last_error": ctypes.c_char_p, "gc_kernel_name": ctypes.c_char_p}

_lib = None


def lib():
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with "
                               "`python cl-util_b200/gcut_build.py` (no fallback exists)")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RESTYPE.get(name, ctypes.c_int)
        _lib = L
    return _lib


def check(rc: int):
    if rc != GC_OK:
        msg = lib().gc_last_error()
        raise GCError(rc, msg.decode() if msg else "")


class ScanState:
    """One look-back state of the scan primitives (gc_scan_state): every PrefixSum,
    StreamCompact and IncrementalTileList owns one, as each reference object owns its own
    buffers, so objects used on different streams never share look-back words."""

    def __init__(self, device: int, max_items: int):
        h = ctypes.c_void_p()
        check(lib().gc_scan_state_create(int(device), int(max_items), ctypes.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def error(self, stream=None) -> int:
        """The error word (0: none; 1: a look-back wait gave up; 2: a scatter index was out
        of range), read synchronously and cleared."""
        e = ctypes.c_int(0)
        check(lib().gc_scan_state_error(self._h, ctypes.byref(e), stream_handle(stream)))
        return int(e.value)

    def selftest(self, spins: int, stream=None) -> int:
        """Runs gc_scan_state_selftest: a bounded look-back wait that must run out."""
        e = ctypes.c_int(0)
        check(lib().gc_scan_state_selftest(self._h, int(spins), ctypes.byref(e),
                                           stream_handle(stream)))
        return int(e.value)

    def close(self):
        if getattr(self, "_h", None):
            lib().gc_scan_state_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def default_opts(**overrides) -> GcOpts:
    o = GcOpts()
    check(lib().gc_opts_default(ctypes.byref(o)))
    for k, v in overrides.items():
        if v is not None:
            setattr(o, k, int(v))
    return o


def stream_handle(stream=None):
    """cudaStream_t of a torch stream (current stream when None) as a ctypes pointer."""
    import torch
    s = torch.cuda.current_stream() if stream is None else stream
    return ctypes.c_void_p(s.cuda_stream)


def ptr(t):
    """Device/host address of a tensor or numpy array."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return ctypes.c_void_p(t.data_ptr())
    return t.ctypes.data_as(ctypes.c_void_p)


TRACE_KINDS = ("begin", "active_list", "discharge", "masks", "flood_first", "flood", "check",
               "bfs_first", "bfs", "upload", "labels", "end")
GC_TRACE_MAX = 2048


def read_trace(get_fn, handle, stream=None):
    """[(kind name, start ns)] of a handle's device-side trace (gc_get_trace and kin)."""
    import numpy as np
    buf = np.zeros(2 * GC_TRACE_MAX, np.uint64)
    n = ctypes.c_int(0)
    check(get_fn(handle, buf.ctypes.data_as(ctypes.c_void_p), GC_TRACE_MAX, ctypes.byref(n),
                 stream_handle(stream)))
    k = min(n.value, GC_TRACE_MAX)
    return [(TRACE_KINDS[int(buf[2 * i + 1])] if int(buf[2 * i + 1]) < len(TRACE_KINDS)
             else str(int(buf[2 * i + 1])), int(buf[2 * i])) for i in range(k)]


def trace_summary(entries):
    """{kind: [count, total ns]} from consecutive start times (each kernel's span runs to the
    next entry's start; the last entry closes the trace)."""
    out = {}
    for (k, t0), (_, t1) in zip(entries, entries[1:]):
        a = out.setdefault(k, [0, 0])
        a[0] += 1
        a[1] += t1 - t0
    return out


def kernel_profile(get_fn, handle) -> dict:
    """{kernel name: {launches, ms, tiles}} from gc_get_profile / gcb_get_profile."""
    arr = (GcKernelProf * GC_NKERN)()
    check(get_fn(handle, arr, GC_NKERN))
    out = {}
    for k in range(GC_NKERN):
        name = lib().gc_kernel_name(k).decode()
        out[name] = {"launches": int(arr[k].launches), "ms": float(arr[k].ms),
                     "tiles": int(arr[k].tiles)}
    return out
