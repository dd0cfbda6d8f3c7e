"""Display layers without a graphics stack.

The reference paints its planes and tile maps over the displayed image with OpenCL filters
that read and write GL images (graphcut_filter.cl: tranpose for a plane such as the heights,
tilelist / tilelist_growcut for a tile map; colorizef and HSVtoRGB map a value through an HSV
ramp).  Here the same layer is an RGBA device buffer (gc_view_colorize), written to a file or
shown by whatever the caller uses:

    from views import colorize
    rgba = colorize(gc.dHeight, value_range=(0, 64), hues=(0.0, 0.7), opacity=0.5, base=image)
    tiles = colorize(tile_list.d_tiles, cell=(32, 32), width=W, height=H, value_range=(0, 10))

IncrementalTileList.execute keeps the reference's red-on-black tile view (gc_tiles_view).
"""
from __future__ import annotations

import ctypes

import numpy as np

from _gcut import check, lib, ptr, stream_handle


def colorize(values, width: int | None = None, height: int | None = None, cell=(1, 1),
             value_range=(0.0, 1.0), hues=(0.0, 1.0), sats=(1.0, 1.0), vals=(1.0, 1.0),
             opacity: float = 1.0, base=None, out=None, stream=None):
    """RGBA words (int32 [height, width] CUDA tensor, R in the low byte) of `values` (an int32
    CUDA tensor [rows, cols] of cells, each cell_w x cell_h pixels) mapped through the HSV ramp
    and blended over `base` (RGBA words, or None for all zero) with `opacity`
    (gc_view_colorize).  width / height default to the cell grid's pixel size."""
    import torch
    if not (isinstance(values, torch.Tensor) and values.is_cuda and values.dtype == torch.int32
            and values.dim() == 2):
        raise TypeError("values must be an int32 CUDA tensor [rows, cols]")
    values = values.contiguous()
    cell_w, cell_h = int(cell[0]), int(cell[1])
    rows, cols = values.shape
    width = cols * cell_w if width is None else int(width)
    height = rows * cell_h if height is None else int(height)
    if base is not None:
        if tuple(base.shape) != (height, width):
            raise ValueError("base must be [height, width]")
        base = base.contiguous()
    if out is None:
        out = torch.empty((height, width), dtype=torch.int32, device=values.device)
    ramp = np.array([value_range[0], value_range[1], hues[0], hues[1], sats[0], sats[1],
                     vals[0], vals[1], opacity], dtype=np.float32)
    with torch.cuda.device(values.device):
        check(lib().gc_view_colorize(ptr(values), cols, rows, cell_w, cell_h, width, height,
                                     ramp.ctypes.data_as(ctypes.c_void_p),
                                     ptr(base) if base is not None else None, ptr(out),
                                     stream_handle(stream)))
    return out
