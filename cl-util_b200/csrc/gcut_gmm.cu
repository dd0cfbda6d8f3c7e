// T-links from two colour models, computed on the device (gc_tlinks_gmm).
//
// The reference scores each pixel under a foreground and a background Gaussian mixture
// (GMM.score, GMM.pyx:130-163, running score_buf / score_img2d, gmm.cl:373-491) and feeds
// the solver excess = scoreBg - scoreFg (test_GraphCut.py:44-47).  Here the two scores, their
// difference and the int32 rounding are one pass over the image: 4 bytes read and 4 written
// per pixel, the rest is float64 arithmetic on registers.
//
// The models are full-covariance (a diagonal model is the special case the reference fits).
// Each component is evaluated as c - 0.5 * |Li (x - mean)|^2 with Li the inverse Cholesky
// factor, every add and multiply rounded on its own in a fixed order (the __d*_rn intrinsics
// are never contracted into fused multiply-adds), so a float64 host evaluation in the same
// order gives the same bits up to the last-bit differences of exp and log.
#include <cmath>
#include <cstdio>

#include "gcut_internal.h"

namespace {

constexpr int kMaxComp = GC_GMM_MAX_COMPONENTS;
constexpr int kThreads = 256;

struct GmmArgs {
  gc_gauss comp[2][kMaxComp];  // [0] foreground, [1] background
  int n[2];
  double scale;
  double clamp;
};

// log(w N(x | mean, S)) of one component.
__device__ __forceinline__ double component_log_density(const gc_gauss& g, double r, double gr,
                                                        double b) {
  const double d0 = __dsub_rn(r, g.mean[0]);
  const double d1 = __dsub_rn(gr, g.mean[1]);
  const double d2 = __dsub_rn(b, g.mean[2]);
  const double y0 = __dmul_rn(g.li[0], d0);
  const double y1 = __dadd_rn(__dmul_rn(g.li[1], d0), __dmul_rn(g.li[2], d1));
  const double y2 = __dadd_rn(__dadd_rn(__dmul_rn(g.li[3], d0), __dmul_rn(g.li[4], d1)),
                              __dmul_rn(g.li[5], d2));
  const double q = __dadd_rn(__dadd_rn(__dmul_rn(y0, y0), __dmul_rn(y1, y1)), __dmul_rn(y2, y2));
  return __dsub_rn(g.c, __dmul_rn(0.5, q));
}

// exp(x) for x below this is under 2^-57, so 1 plus up to seven such terms, added in any
// order, rounds to exactly 1 in float64.
constexpr double kNegligible = -40.0;

// -log sum_k w_k N(x | mean_k, S_k) = -(m + log(sum_k exp(e_k - m))), m = max_k e_k, for a
// model of n <= KMAX components.
template <int KMAX>
__device__ __forceinline__ double mixture_score(const gc_gauss* comp, int n, double r, double g,
                                                double b) {
  double e[KMAX];
  double m = -INFINITY;
#pragma unroll
  for (int k = 0; k < KMAX; ++k) {
    if (k < n) {
      e[k] = component_log_density(comp[k], r, g, b);
      m = fmax(m, e[k]);
    }
  }
  int near = 0;
#pragma unroll
  for (int k = 0; k < KMAX; ++k)
    if (k < n && __dsub_rn(e[k], m) >= kNegligible) ++near;
  // Only the largest term counts: the sum is exactly exp(0) = 1 and log(1) = 0, which is
  // what the full evaluation below gives too; skipping it saves the exp and log calls.
  if (near == 1) return -__dadd_rn(m, 0.0);
  double sum = 0.0;
#pragma unroll
  for (int k = 0; k < KMAX; ++k)
    if (k < n) sum = __dadd_rn(sum, exp(__dsub_rn(e[k], m)));
  return -__dadd_rn(m, log(sum));
}

// KMAX: the larger of the two models' component counts, rounded up to 2, 4 or 8 (fewer
// registers for the common small models).
template <int KMAX>
__global__ void __launch_bounds__(kThreads)
k_tlinks_gmm(const uint32_t* __restrict__ rgba, int width, long long n, int pitch,
             const GmmArgs a, int32_t* __restrict__ excess) {
  for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n;
       i += (long long)gridDim.x * kThreads) {
    const long long y = i / width;
    const long long x = i - y * width;
    const uint32_t px = __ldg(rgba + y * pitch + x);
    const double r = (double)(px & 0xFFu);
    const double g = (double)((px >> 8) & 0xFFu);
    const double b = (double)((px >> 16) & 0xFFu);
    const double s_fg = mixture_score<KMAX>(a.comp[0], a.n[0], r, g, b);
    const double s_bg = mixture_score<KMAX>(a.comp[1], a.n[1], r, g, b);
    double t = floor(__dadd_rn(__dmul_rn(a.scale, __dsub_rn(s_bg, s_fg)), 0.5));
    t = fmin(fmax(t, -a.clamp), a.clamp);
    excess[i] = (int32_t)t;
  }
}

int tlinks_fail(const char* msg) { return gcut::set_last_error(GC_ERR_INVALID, msg); }

bool finite_within(double v, double bound) { return std::isfinite(v) && std::fabs(v) <= bound; }

int check_model(const gc_gauss* m, int n, const char* which) {
  static thread_local char buf[160];
  if (n < 1 || n > kMaxComp) {
    snprintf(buf, sizeof buf, "gc_tlinks_gmm: %s model needs 1..%d components", which, kMaxComp);
    return tlinks_fail(buf);
  }
  if (!m) {
    snprintf(buf, sizeof buf, "gc_tlinks_gmm: %s model is null", which);
    return tlinks_fail(buf);
  }
  for (int k = 0; k < n; ++k) {
    bool ok = finite_within(m[k].c, 0x1p64);
    for (int j = 0; j < 3; ++j) ok = ok && finite_within(m[k].mean[j], 0x1p32);
    for (int j = 0; j < 6; ++j) ok = ok && finite_within(m[k].li[j], 0x1p32);
    if (!ok) {
      snprintf(buf, sizeof buf,
               "gc_tlinks_gmm: %s component %d has a non-finite or out-of-range parameter", which, k);
      return tlinks_fail(buf);
    }
  }
  return GC_OK;
}

}  // namespace

extern "C" int gc_tlinks_gmm(const uint32_t* rgba, int width, int height, int pitch,
                             const gc_gauss* fg, int n_fg, const gc_gauss* bg, int n_bg,
                             double scale, int32_t clamp, int32_t* excess, void* stream) {
  gcut::set_last_error(GC_OK, "");
  if (width < 0 || height < 0) return tlinks_fail("gc_tlinks_gmm: negative size");
  if (pitch < width) return tlinks_fail("gc_tlinks_gmm: pitch < width");
  if (!finite_within(scale, 0x1p32)) return tlinks_fail("gc_tlinks_gmm: |scale| > 2^32 or not finite");
  if (clamp < 0 || clamp > (1 << 30)) return tlinks_fail("gc_tlinks_gmm: clamp outside [0, 2^30]");
  int r = check_model(fg, n_fg, "foreground");
  if (r != GC_OK) return r;
  r = check_model(bg, n_bg, "background");
  if (r != GC_OK) return r;
  const long long n = (long long)width * height;
  if (n == 0) return GC_OK;
  if (!rgba || !excess) return tlinks_fail("gc_tlinks_gmm: null image or output");

  GmmArgs a{};
  for (int k = 0; k < n_fg; ++k) a.comp[0][k] = fg[k];
  for (int k = 0; k < n_bg; ++k) a.comp[1][k] = bg[k];
  a.n[0] = n_fg;
  a.n[1] = n_bg;
  a.scale = scale;
  a.clamp = (double)clamp;
  const long long blocks = (n + kThreads - 1) / kThreads;
  const unsigned grid = (unsigned)(blocks < (1LL << 30) ? blocks : (1LL << 30));
  const int kmax = n_fg > n_bg ? n_fg : n_bg;
  cudaStream_t s = (cudaStream_t)stream;
  if (kmax <= 2)
    k_tlinks_gmm<2><<<grid, kThreads, 0, s>>>(rgba, width, n, pitch, a, excess);
  else if (kmax <= 4)
    k_tlinks_gmm<4><<<grid, kThreads, 0, s>>>(rgba, width, n, pitch, a, excess);
  else
    k_tlinks_gmm<8><<<grid, kThreads, 0, s>>>(rgba, width, n, pitch, a, excess);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return gcut::set_last_error(GC_ERR_CUDA, cudaGetErrorString(e));
  return GC_OK;
}
