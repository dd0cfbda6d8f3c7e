"""T-links from colour models on the device (gc_tlinks_gmm).

The reference fits a Gaussian mixture to the foreground and to the background strokes
(GMM.fit, GMM.pyx:165-372), scores every pixel under each (GMM.score, GMM.pyx:130-163;
score_buf / score_img2d, gmm.cl:373-491) and passes ``scoreBg - scoreFg`` to the solver as
its excess (test_GraphCut.py:44-47).  Here the fit stays with the caller (its output is a
handful of numbers per component) and one kernel turns the image and the two models into the
solver's int32 excess plane:

    excess = clamp(floor(scale * (s_bg - s_fg) + 0.5), -clamp, clamp),
    s = -log sum_k w_k N(x | mean_k, S_k),  x = (R, G, B)

    fg = Mixture(weights, means, covars)        # covars [K, 3] (diagonal) or [K, 3, 3]
    ex = tlinks(rgba, fg, bg)                   # torch int32 [H, W] on the device
    gc.upload_image(rgba, ex)                   # or gc.upload_image(rgba, (fg, bg))

The result equals a float64 host evaluation of the same expression (``components`` gives the
form it is evaluated in) except where the host's and the device's exp / log differ in the
last bit and that moves ``scale * (s_bg - s_fg) + 0.5`` across an integer.
"""
from __future__ import annotations

import ctypes

import numpy as np

import _gcut
from _gcut import GcGauss, check, lib, ptr, stream_handle

TLINK_SCALE = 100.0
TLINK_CLAMP = 10 ** 6


def components(weights, means, covars) -> np.ndarray:
    """Evaluation form of a Gaussian mixture: float64 [K, 10] rows (c, mean[3], li[6]), the
    layout of ``gc_gauss``.

    ``li`` is the lower triangle (Li00, Li10, Li11, Li20, Li21, Li22) of the inverse of the
    Cholesky factor of the covariance and ``c = log w - 0.5 * (3 log 2pi + log det S)``, so
    that log(w N(x | mean, S)) = c - 0.5 |Li (x - mean)|^2.  ``covars`` is [K, 3] for
    diagonal covariances (GMM.fit's output, GMM.pyx:366-372) or [K, 3, 3].
    """
    w = np.asarray(weights, np.float64).reshape(-1)
    mu = np.asarray(means, np.float64).reshape(len(w), 3)
    cv = np.asarray(covars, np.float64)
    if cv.shape == (len(w), 3):
        cv = np.stack([np.diag(v) for v in cv])
    if cv.shape != (len(w), 3, 3):
        raise ValueError(f"covars must be [K, 3] or [K, 3, 3], got {cv.shape}")
    if not 1 <= len(w) <= _gcut.GC_GMM_MAX_COMPONENTS:
        raise ValueError(f"a model has 1..{_gcut.GC_GMM_MAX_COMPONENTS} components")
    out = np.empty((len(w), 10), np.float64)
    for k in range(len(w)):
        L = np.linalg.cholesky(cv[k])
        Li = np.linalg.inv(L)
        logdet = 2.0 * np.log(np.diag(L)).sum()
        out[k, 0] = np.log(w[k]) - 0.5 * (3 * np.log(2 * np.pi) + logdet)
        out[k, 1:4] = mu[k]
        out[k, 4:10] = (Li[0, 0], Li[1, 0], Li[1, 1], Li[2, 0], Li[2, 1], Li[2, 2])
    return out


class Mixture:
    """A fitted colour model (weights [K], means [K, 3], covars [K, 3] or [K, 3, 3])."""

    def __init__(self, weights, means, covars):
        self.comps = components(weights, means, covars)

    @classmethod
    def from_components(cls, comps) -> "Mixture":
        m = cls.__new__(cls)
        m.comps = np.ascontiguousarray(comps, np.float64).reshape(-1, 10)
        return m

    def __len__(self):
        return self.comps.shape[0]

    def as_c(self):
        arr = (GcGauss * len(self))()
        ctypes.memmove(arr, self.comps.ctypes.data, self.comps.nbytes)
        return arr


def _mixture(m) -> Mixture:
    return m if isinstance(m, Mixture) else Mixture.from_components(m)


def tlinks(rgba, fg, bg, scale: float = TLINK_SCALE, clamp: int = TLINK_CLAMP, out=None,
           stream=None, device=None):
    """int32 [H, W] excess plane on the device from an image and two colour models.

    ``rgba`` is a torch CUDA or numpy array, uint32 [H, W] (R in the low byte) or uint8
    [H, W, 3|4]; a strided torch row layout (unit column stride) is read in place.  ``fg`` and
    ``bg`` are ``Mixture`` objects or [K, 10] ``components`` arrays.  ``out`` (torch int32
    [H, W], contiguous, on the device) receives the result when given.
    """
    import torch

    from GraphCut import _as_rgba32
    img = _as_rgba32(rgba)
    if not (isinstance(img, torch.Tensor) and img.is_cuda):
        dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        img = torch.from_numpy(np.ascontiguousarray(
            img.cpu().numpy() if isinstance(img, torch.Tensor) else img).view(np.int32)).to(dev)
    if img.dim() != 2 or img.stride(1) != 1:
        img = img.contiguous()
    h, w = img.shape
    if out is None:
        out = torch.empty((h, w), dtype=torch.int32, device=img.device)
    elif out.dtype != torch.int32 or tuple(out.shape) != (h, w) or not out.is_contiguous():
        raise ValueError("out must be a contiguous int32 [H, W] tensor")
    f, b = _mixture(fg), _mixture(bg)
    fc, bc = f.as_c(), b.as_c()
    with torch.cuda.device(img.device):
        check(lib().gc_tlinks_gmm(ptr(img), w, h, img.stride(0) if h > 0 else w, fc, len(f),
                                  bc, len(b), float(scale), int(clamp), ptr(out),
                                  stream_handle(stream)))
    return out
