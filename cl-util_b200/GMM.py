"""GMM: the colour-model class of the reference (GMM.pyx:18-395) on libgcut.

The reference fits a Gaussian mixture to stroke pixels with a chain of OpenCL launches and
host waits per EM iteration (GMM.fit, GMM.pyx:165-372).  Here ``fit`` is one launch of
``gc_gmm_fit`` (a thread-block cluster that runs every iteration on the device) and one
small read-back of the result:

    gmm = GMM(n_iterations=65, n_components=4)
    weights, means, covars = gmm.fit(d_samples, retParams=True)
    fg = gmm.mixture()                       # gmm_tlinks.Mixture, for gmm_tlinks.tlinks

Samples are RGBA words (R in the low byte) as torch CUDA int32/uint32 tensors or numpy
arrays.  Arithmetic is float64; covariances are diagonal as in the reference unless
``full_covariance`` is set.
"""
from __future__ import annotations

import ctypes

import numpy as np

import _gcut
from _gcut import GcGmmFitResult, check, lib, ptr, stream_handle

MIN_COVAR = 1e-3     # GMM.pyx:10, passed to gmm.cl as -D MIN_COVAR (GMM.pyx:66-71)
INIT_COVAR = 30.0    # GMM.pyx:9, passed as -D INIT_COVAR
TOLERANCE = 0.01     # GMM.pyx:329


class GMM:
    """``GMM(n_iterations, n_components, cap_samples, min_covar, init_covar)`` as in the
    reference (GMM.pyx:59-93).  ``cap_samples`` is accepted and ignored: the reference sizes
    its per-sample responsibility buffers with it, and the device fit keeps no per-sample
    state."""

    def __init__(self, n_iterations: int, n_components: int, cap_samples=None,
                 min_covar=None, init_covar=None, tolerance: float = TOLERANCE,
                 full_covariance: bool = False, device=0):
        if not 1 <= n_components <= _gcut.GC_GMM_MAX_COMPONENTS:
            raise ValueError(f"n_components must be 1..{_gcut.GC_GMM_MAX_COMPONENTS}")
        self.n_iterations = int(n_iterations)
        self.n_components = int(n_components)
        self.cap_samples = cap_samples
        self.min_covar = MIN_COVAR if min_covar is None else float(min_covar)
        self.init_covar = INIT_COVAR if init_covar is None else float(init_covar)
        self.tolerance = float(tolerance)
        self.full_covariance = bool(full_covariance)
        self.device = device
        self.has_converged = False
        self.iterations = 0
        self.log_likelihood = None
        self.weights = self.means = self.covars = None
        self._result = None

    def fit(self, d_samples, nSamples=None, retParams=None, stream=None):
        """EM on the device (gc_gmm_fit).  Returns (weights [K], means [K, 3], covars [K, 3]
        or [K, 3, 3]) when ``retParams``, as the reference does."""
        import torch
        if isinstance(d_samples, torch.Tensor) and d_samples.is_cuda:
            if d_samples.element_size() != 4:
                raise TypeError("samples must be 32-bit RGBA words")
            dev = d_samples.reshape(-1).contiguous()
        else:
            host = d_samples.cpu().numpy() if isinstance(d_samples, torch.Tensor) else d_samples
            host = np.ascontiguousarray(np.asarray(host).reshape(-1)).view(np.int32)
            dev = torch.from_numpy(host).to(torch.device("cuda", self.device)
                                            if isinstance(self.device, int) else self.device)
        n = dev.numel() if nSamples is None else int(nSamples)
        if n < self.n_components:
            raise ValueError(f"nSamples < nComp: {n}, {self.n_components}")  # GMM.pyx:169-171
        if n > dev.numel():
            raise ValueError("nSamples exceeds the samples given")
        if self._result is None or self._result.device != dev.device:
            self._result = torch.empty(ctypes.sizeof(GcGmmFitResult), dtype=torch.uint8,
                                       device=dev.device)
        from GraphCut import _on
        with torch.cuda.device(dev.device), _on(stream):
            # the fit and the read-back on one stream: the copy waits for the fit
            check(lib().gc_gmm_fit(ptr(dev), n, self.n_components, self.n_iterations,
                                   self.tolerance, self.min_covar, self.init_covar,
                                   int(self.full_covariance), ptr(self._result),
                                   stream_handle(stream)))
            host = self._result.cpu().numpy()
        r = GcGmmFitResult.from_buffer_copy(host.tobytes())
        K = self.n_components
        self.weights = np.array(r.weights[:K])
        self.means = np.array([list(r.means[k]) for k in range(K)])
        tri = np.array([list(r.covars[k]) for k in range(K)])
        full = np.empty((K, 3, 3))
        for k in range(K):
            s00, s10, s11, s20, s21, s22 = tri[k]
            full[k] = [[s00, s10, s20], [s10, s11, s21], [s20, s21, s22]]
        self.covars = full if self.full_covariance else np.stack([np.diag(m) for m in full])
        self.iterations = int(r.iterations)
        self.has_converged = bool(r.converged)
        self.log_likelihood = float(r.log_likelihood)
        # the model's evaluation form as the device computed it ([K, 10] rows of gc_gauss)
        self.device_components = np.array(
            [[r.components[k].c, *r.components[k].mean, *r.components[k].li] for k in range(K)])
        if r.status:
            raise _gcut.GCError(_gcut.GC_ERR_NOT_CONVERGED,
                                "gc_gmm_fit: a covariance stopped being positive definite "
                                f"after {self.iterations} iterations")
        if retParams:
            return self.weights, self.means, self.covars

    def mixture(self):
        """The fitted model as a gmm_tlinks.Mixture (components of weight 0 left out)."""
        from gmm_tlinks import Mixture
        if self.weights is None:
            raise RuntimeError("fit first")
        keep = self.weights > 0
        return Mixture(self.weights[keep], self.means[keep], self.covars[keep])
