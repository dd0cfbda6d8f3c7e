"""The reference's own graph-cut kernels on the host.  TEST INFRASTRUCTURE ONLY.

``oracle/_ref/librefcl.so`` holds graphcut.cl compiled unchanged as C, with the reference's
host loop (GraphCut.cut, GraphCut.pyx:348-418) around it; ``refcl_host.c`` says how it is
run.  The library is built only where the reference checkout is present (``make -C oracle
ref REF=<checkout>``), and ``available()`` is false elsewhere.  The parity tests use it to
pin the oracle to the reference's own kernels; ``tests/golden/make_refcl_golden.py`` writes
its answers into fixtures, which pin the oracle and the CUDA path where the checkout is
absent.

The kernels' image size is fixed in their source (graphcut.cl:15-16): 800 x 608.  A second
library, ``librefcl_512x512.so``, is built from a copy with those two lines set to 512 x 512
(the reference's CPU-sized configuration); ``cut`` picks the library by the planes' shape.
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_PATH = os.path.join(_HERE, "_ref", "librefcl.so")
_PATHS = {(800, 608): _PATH,
          (512, 512): os.path.join(_HERE, "_ref", "librefcl_512x512.so")}
_LIBS = {}

WIDTH, HEIGHT = 800, 608     # the size fixed in graphcut.cl
SIZES = tuple(_PATHS)        # (width, height) of every library
STAT_NAMES = ("iterations", "relabels", "bfs_rounds", "launches", "guard_bytes_dirty",
              "barriers_without_fibers", "divergent_barrier_passes", "non_integral_values")


def build(reference_dir: str | None = None) -> bool:
    """Build the libraries from the reference checkout (the Makefile's default location
    when reference_dir is None); False when the checkout's kernel sources are not there."""
    cmd = ["make", "-s", "-C", _HERE, "ref"]
    if reference_dir is not None:
        if not os.path.exists(os.path.join(reference_dir, "graphcut.cl")):
            return False
        cmd.append(f"REF={reference_dir}")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        if re.search(r"No rule to make target '[^']*\.cl'", r.stderr):
            return False   # a reference kernel source is missing: no checkout here
        raise RuntimeError(f"building the reference kernels failed:\n{r.stderr}")
    return all(os.path.exists(p) for p in _PATHS.values()) and scan_available()


def available(size=(WIDTH, HEIGHT)) -> bool:
    return os.path.exists(_PATHS[tuple(size)])


def lib(size=(WIDTH, HEIGHT)):
    size = tuple(size)
    if size not in _LIBS:
        path = _PATHS[size]
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -C oracle ref REF=<checkout>)")
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        L.refcl_cut.argtypes = ([P] * 5 + [ctypes.c_int, ctypes.c_longlong] + [P] * 6 +
                                [ctypes.c_int, P])
        L.refcl_cut.restype = ctypes.c_int
        if (L.refcl_width(), L.refcl_height()) != size:
            raise RuntimeError(f"{path} was built for another size")
        _LIBS[size] = L
    return _LIBS[size]


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


SCHEDULE_LOCKSTEP, SCHEDULE_SERIAL = 0, 1


def cut(up, down, left, right, excess, bfs: int = 5, max_iters: int = 100_000,
        schedule: int = SCHEDULE_LOCKSTEP):
    """Run GraphCut.cut with the reference's kernels on an integer graph of one of SIZES
    (800 x 608, the kernels' own size, or 512 x 512).

    schedule: SCHEDULE_LOCKSTEP (the work-items of a group make each access to
    bfs_intratile's loop flag together -- all test, all reset, then the changed ones set --
    as a GPU warp's lanes do) or SCHEDULE_SERIAL (work-items strictly one after another
    between barriers, as a CPU OpenCL runtime runs them; the race on that flag,
    graphcut.cl:925-990, then ends the in-tile BFS early).

    Returns a dict: the final residual planes ``up``/``down``/``left``/``right`` and
    ``excess`` (int32, row-major, true residuals: tiles never loaded get their capacities
    added), ``height``, and ``stats`` (a dict over STAT_NAMES).  Raises on a bad argument
    or when max_iters push iterations do not finish."""
    planes = [np.ascontiguousarray(a, dtype=np.int32) for a in (up, down, left, right, excess)]
    shape = planes[4].shape
    size = (shape[1], shape[0]) if len(shape) == 2 else None
    if size not in _PATHS or any(a.shape != shape for a in planes):
        raise ValueError(f"the reference kernels take planes of one of {SIZES} "
                         f"(width, height), got {[a.shape for a in planes]}")
    out = [np.zeros(shape, np.int32) for _ in range(6)]
    stats = np.zeros(len(STAT_NAMES), np.int64)
    rc = lib(size).refcl_cut(*[_p(a) for a in planes], int(bfs), int(max_iters),
                         *[_p(a) for a in out], int(schedule), _p(stats))
    if rc == 1:
        raise ValueError("refcl_cut: bad argument (capacities must be in [0, 2^24), "
                         "|excess| < 2^24)")
    if rc == 2:
        raise MemoryError("refcl_cut: out of memory")
    if rc == 3:
        raise RuntimeError(f"refcl_cut: not finished after {max_iters} push iterations")
    if rc != 0:
        raise RuntimeError(f"refcl_cut failed ({rc})")
    names = ("up", "down", "left", "right", "excess", "height")
    res = dict(zip(names, out))
    res["stats"] = {k: int(v) for k, v in zip(STAT_NAMES, stats)}
    return res


# ---------------------------------------------------------------------------------------
# The reference's scan and compaction kernels (prefixsum.cl, streamcompact.cl) under the
# restated PrefixSum / StreamCompact host code (refcl_scan.c).
# ---------------------------------------------------------------------------------------
_SCAN_PATH = os.path.join(_HERE, "_ref", "librefcl_scan.so")
SCAN_STAT_NAMES = ("launches", "guard_bytes_dirty", "barriers_without_fibers")


def scan_available() -> bool:
    return os.path.exists(_SCAN_PATH)


def _scan_lib():
    if "scan" not in _LIBS:
        if not scan_available():
            raise FileNotFoundError(f"{_SCAN_PATH} is not built (make -C oracle ref REF=<checkout>)")
        L = ctypes.CDLL(_SCAN_PATH)
        P = ctypes.c_void_p
        for name in ("refcl_scan", "refcl_compact"):
            f = getattr(L, name)
            f.argtypes = [P, ctypes.c_int, ctypes.c_int, P, P, P]
            f.restype = ctypes.c_int
        _LIBS["scan"] = L
    return _LIBS["scan"]


def _scan_rc(rc, what):
    if rc == 1:
        raise ValueError(f"{what}: bad argument (length >= 1 and capacity >= length)")
    if rc == 2:
        raise MemoryError(f"{what}: out of memory")
    if rc == 4:
        raise IndexError(f"{what}: the reference's host code indexes a partial-sum level "
                         "that does not exist")
    if rc != 0:
        raise RuntimeError(f"{what} failed ({rc})")


def scan(values, capacity=None):
    """PrefixSum(capacity).scan on the reference's kernels: (exclusive scan, total, stats).
    The reference cannot scan an empty array, so len(values) >= 1."""
    a = np.ascontiguousarray(values, dtype=np.int32).ravel()
    out = np.zeros_like(a)
    total = np.zeros(1, np.int32)
    stats = np.zeros(len(SCAN_STAT_NAMES), np.int64)
    cap = a.size if capacity is None else int(capacity)
    _scan_rc(_scan_lib().refcl_scan(_p(a), a.size, cap, _p(out), _p(total), _p(stats)),
             "refcl_scan")
    return out, int(total[0]), {k: int(v) for k, v in zip(SCAN_STAT_NAMES, stats)}


def compact(flags, capacity=None):
    """StreamCompact(capacity).compact on the reference's kernels: (list, length, stats)."""
    a = np.ascontiguousarray(flags, dtype=np.int32).ravel()
    lst = np.zeros_like(a)
    length = np.zeros(1, np.int32)
    stats = np.zeros(len(SCAN_STAT_NAMES), np.int64)
    cap = a.size if capacity is None else int(capacity)
    _scan_rc(_scan_lib().refcl_compact(_p(a), a.size, cap, _p(lst), _p(length), _p(stats)),
             "refcl_compact")
    n = int(length[0])
    return lst[:n], n, {k: int(v) for k, v in zip(SCAN_STAT_NAMES, stats)}
