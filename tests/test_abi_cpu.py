"""The C-ABI library loads without a GPU and exports every function include/gcut.h
declares; the Python binding declares exactly those functions."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    with open(os.path.join(ROOT, "include", "gcut.h")) as f:
        src = f.read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gc[bp]?_[a-z_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def libgcut():
    import _gcut
    if not os.path.exists(_gcut.LIB_PATH):
        import gcut_build
        gcut_build.build()
    return ctypes.CDLL(_gcut.LIB_PATH)


def test_header_declares_functions():
    names = header_functions()
    assert "gc_solve" in names and "gc_compact" in names and "gcb_solve" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol(libgcut):
    missing = [n for n in header_functions() if not hasattr(libgcut, n)]
    assert not missing, missing


def test_binding_matches_header():
    import _gcut
    assert sorted(_gcut.SIGNATURES) == header_functions()


def test_calls_without_gpu_fail_cleanly(libgcut):
    """No CUDA device here: creating a solver returns an error code, never crashes."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import _gcut
    L = _gcut.lib()
    h = ctypes.c_void_p()
    rc = L.gc_create(64, 64, None, ctypes.byref(h))
    assert rc != 0 and not h.value
    assert L.gc_last_error()
    # invalid arguments are rejected before any CUDA call
    assert L.gc_create(0, 64, None, ctypes.byref(h)) == _gcut.GC_ERR_INVALID
    assert L.gc_solve(None, None) == _gcut.GC_ERR_INVALID
    ramp = (ctypes.c_float * 9)(0, 1, 0, 1, 1, 1, 1, 1, 1)
    assert L.gc_view_colorize(None, 1, 1, 0, 1, 4, 4, ramp, None, None, None) \
        == _gcut.GC_ERR_INVALID                               # cell width 0
    ramp[8] = float("nan")
    assert L.gc_view_colorize(None, 1, 1, 1, 1, 4, 4, ramp, None, None, None) \
        == _gcut.GC_ERR_INVALID                               # opacity not finite
    o = _gcut.GcOpts()
    assert L.gc_opts_default(ctypes.byref(o)) == 0 and o.discharge_iters > 0


def test_arena_bytes_host_only():
    """gc_arena_bytes needs no device: it sizes the arena of a handle from its grid."""
    import _gcut
    lib = _gcut.lib()
    out = ctypes.c_int64()
    sizes = {}
    for w, h in [(1, 1), (32, 32), (33, 32), (512, 512), (4096, 4096)]:
        assert lib.gc_arena_bytes(w, h, ctypes.byref(out)) == 0
        sizes[(w, h)] = out.value
    assert 0 < sizes[(1, 1)] <= sizes[(32, 32)]            # one tile; label staging W*H
    assert sizes[(33, 32)] > sizes[(32, 32)]
    assert sizes[(4096, 4096)] > 28 * 4096 * 4096            # 7 int32 planes at least
    assert sizes[(4096, 4096)] < 32 * 4096 * 4096
    assert lib.gc_arena_bytes(0, 5, ctypes.byref(out)) == 1   # GC_ERR_INVALID


def test_struct_layouts_match_the_c_compiler(tmp_path):
    """The ctypes mirrors of the header's structs have the sizes and field offsets gcc gives
    the C declarations (a drift here would corrupt every call that passes them)."""
    import shutil
    import subprocess

    import _gcut
    if not shutil.which("gcc"):
        pytest.skip("gcc not found")
    fields = {
        "gc_opts": (_gcut.GcOpts, ["device", "discharge_iters", "max_cycles", "use_graph"]),
        "gc_stats": (_gcut.GcStats, ["cycles", "launches", "tiles_discharged"]),
        "gc_gauss": (_gcut.GcGauss, ["c", "mean", "li"]),
        "gc_gmm_fit_result": (_gcut.GcGmmFitResult,
                              ["weights", "means", "covars", "log_likelihood", "iterations",
                               "converged", "status", "n_components", "components"]),
    }
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "gcut.h"', "int main(void) {"]
    for name, (_, fs) in fields.items():
        lines.append(f'  printf("{name} %zu\\n", sizeof({name}));')
        for f in fs:
            lines.append(f'  printf("{name}.{f} %zu\\n", offsetof({name}, {f}));')
    lines.append("  return 0;\n}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)],
                   check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                       text=True).stdout.splitlines())
    for name, (cls, fs) in fields.items():
        assert int(got[name]) == ctypes.sizeof(cls), name
        for f in fs:
            assert int(got[f"{name}.{f}"]) == getattr(cls, f).offset, (name, f)
