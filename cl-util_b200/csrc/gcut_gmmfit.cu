// Colour-model fit on the device (gc_gmm_fit): expectation-maximisation of a Gaussian mixture
// over pixel colours, the reference's GMM.fit (GMM.pyx:165-372; initA, em1, em2, eval and
// check_converge, gmm.cl:33-372), in float64.
//
// The reference runs every EM iteration as a chain of launches separated by host waits: em1
// writes per-sample responsibilities to global memory, em2 halves them log2(n) times, eval
// and check_converge sum the log-likelihood, and the host reads it back to decide whether
// to go on.  Here the whole fit is ONE launch of one thread-block cluster (8 blocks of 256
// threads on 8 SMs):
//   * each block folds its share of the samples into per-thread sums held in registers (the
//     responsibilities never leave the SM), then into one row of block sums in shared memory;
//   * the blocks read one another's rows through distributed shared memory, every block in
//     the same fixed order, so every block holds bit-identical totals and takes the same
//     decisions (no broadcast is needed, and a run is deterministic);
//   * two cluster barriers per iteration: after the block sums are written, and after every
//     block has read them.
// All barriers are hardware cluster barriers that every thread of every block reaches the
// same number of times: the loop's exit decisions come from the identical totals.
#include <cooperative_groups.h>

#include <cmath>

#include "gcut_internal.h"

namespace cg = cooperative_groups;

namespace {

constexpr int kMaxK = GC_GMM_MAX_COMPONENTS;
constexpr int kCluster = 8;                  // blocks in the cluster (the portable maximum)
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kStats = 10;                   // per component: r, r x (3), r x x^T (6)
constexpr int kLsum = kMaxK * kStats;        // index of the log-likelihood sum
constexpr int kVals = kLsum + 1;
constexpr double kLog2Pi = 1.8378770664093453;  // log(2 pi)

struct FitShared {
  double stats[kVals];          // this block's sums, read by the cluster's other blocks
  double tot[kVals];            // cluster totals (identical in every block)
  double wpart[kWarps][kVals];  // per-warp sums
  double w[kMaxK], mu[kMaxK][3], S[kMaxK][6];   // current model (S: lower triangle)
  double c[kMaxK], li[kMaxK][6];                // its evaluation form
  double lprev, lcur;
  int stop, status, iterations, converged;
};

// Evaluation form of component k: c = log w - 0.5 (3 log 2pi + log det S) and Li, the
// inverse of the lower Cholesky factor of S.  Returns false when S is not positive definite.
__device__ bool component_form(FitShared& sh, int k) {
  const double* S = sh.S[k];
  const double l00 = sqrt(S[0]);
  const double l10 = S[1] / l00, l20 = S[3] / l00;
  const double d11 = S[2] - l10 * l10;
  const double l11 = sqrt(d11);
  const double l21 = (S[4] - l20 * l10) / l11;
  const double d22 = S[5] - l20 * l20 - l21 * l21;
  const double l22 = sqrt(d22);
  const double i00 = 1.0 / l00, i11 = 1.0 / l11, i22 = 1.0 / l22;
  const double i10 = -l10 * i00 * i11;
  const double i21 = -l21 * i11 * i22;
  const double i20 = -(l20 * i00 + l21 * i10) * i22;
  const double logdet = 2.0 * (log(l00) + log(l11) + log(l22));
  sh.c[k] = log(sh.w[k]) - 0.5 * (3.0 * kLog2Pi + logdet);
  sh.li[k][0] = i00; sh.li[k][1] = i10; sh.li[k][2] = i11;
  sh.li[k][3] = i20; sh.li[k][4] = i21; sh.li[k][5] = i22;
  return S[0] > 0.0 && d11 > 0.0 && d22 > 0.0 && isfinite(logdet);
}

// M-step of one component from the cluster totals (em2, gmm.cl:183-312): weight N_k / sum N,
// mean sum r x / N_k, covariance sum r x x^T / N_k - mean mean^T + min_covar I.
__device__ void m_step(FitShared& sh, int K, double min_covar, int full) {
  double sum_n = 0.0;
  for (int k = 0; k < K; ++k) sum_n += sh.tot[k * kStats];
  for (int k = 0; k < K; ++k) {
    const double* t = sh.tot + k * kStats;
    const double nk = t[0];
    if (!(nk > 0.0)) {  // no responsibility left: weight 0, the rest unchanged
      sh.w[k] = 0.0;
      continue;
    }
    sh.w[k] = nk / sum_n;
    const double m0 = t[1] / nk, m1 = t[2] / nk, m2 = t[3] / nk;
    sh.mu[k][0] = m0; sh.mu[k][1] = m1; sh.mu[k][2] = m2;
    double* S = sh.S[k];
    S[0] = t[4] / nk - m0 * m0 + min_covar;
    S[2] = t[6] / nk - m1 * m1 + min_covar;
    S[5] = t[9] / nk - m2 * m2 + min_covar;
    if (full) {
      S[1] = t[5] / nk - m1 * m0;
      S[3] = t[7] / nk - m2 * m0;
      S[4] = t[8] / nk - m2 * m1;
    } else {
      S[1] = S[3] = S[4] = 0.0;
    }
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// One cluster of kCluster blocks.  KMAX: the component count rounded up to 2, 4 or 8.  The
// per-thread sums of up to 4 components (40 doubles) stay in registers in one pass over the
// samples; models of 5 to 8 components take passes of 2 components each, which recompute
// the responsibilities rather than spill.
template <int KMAX>
__global__ void __cluster_dims__(kCluster, 1, 1) __launch_bounds__(kThreads, 1)
k_gmm_fit(const uint32_t* __restrict__ samples, int n, int K, int max_iter, double tol,
          double min_covar, double init_covar, int full, gc_gmm_fit_result* __restrict__ out) {
  constexpr int CH = KMAX <= 4 ? KMAX : 2;
  __shared__ FitShared sh;
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int stride = kCluster * kThreads;

  // initA (gmm.cl:33-72): evenly spaced samples as means.  Its green channel goes through
  // the mask 0xFF0 (gmm.cl:54), a typo for 0xFF00; the full green byte is used here.
  if (tid == 0) {
    for (int k = 0; k < K; ++k) {
      const int idx = K > 1 ? (int)((long long)k * (n - 1) / (K - 1)) : 0;
      const uint32_t px = samples[idx];
      sh.w[k] = 1.0 / K;
      sh.mu[k][0] = (double)(px & 0xFFu);
      sh.mu[k][1] = (double)((px >> 8) & 0xFFu);
      sh.mu[k][2] = (double)((px >> 16) & 0xFFu);
      double* S = sh.S[k];
      S[0] = S[2] = S[5] = init_covar;
      S[1] = S[3] = S[4] = 0.0;
    }
    sh.lprev = sh.lcur = 0.0;
    sh.stop = sh.status = sh.iterations = sh.converged = 0;
  }
  __syncthreads();

  for (int t = 0;; ++t) {
    if (tid < K && !component_form(sh, tid)) sh.status = 1;
    __syncthreads();
    if (sh.status) break;  // the same in every block: the totals and models are identical

    // E-step (em1): responsibilities and their moment sums, CH components per pass
#pragma unroll
    for (int p = 0; p < KMAX / CH; ++p) {
      if (p * CH >= K) break;
      double acc[CH * kStats];
#pragma unroll
      for (int v = 0; v < CH * kStats; ++v) acc[v] = 0.0;
      double lsum = 0.0;
      for (int i = rank * kThreads + tid; i < n; i += stride) {
        const uint32_t px = samples[i];
        const double x0 = (double)(px & 0xFFu), x1 = (double)((px >> 8) & 0xFFu),
                     x2 = (double)((px >> 16) & 0xFFu);
        double e[KMAX];
        double m = -INFINITY;
#pragma unroll
        for (int k = 0; k < KMAX; ++k) {
          if (k < K) {
            const double d0 = x0 - sh.mu[k][0], d1 = x1 - sh.mu[k][1], d2 = x2 - sh.mu[k][2];
            const double* L = sh.li[k];
            const double y0 = L[0] * d0;
            const double y1 = L[1] * d0 + L[2] * d1;
            const double y2 = L[3] * d0 + L[4] * d1 + L[5] * d2;
            e[k] = sh.c[k] - 0.5 * (y0 * y0 + y1 * y1 + y2 * y2);
            m = fmax(m, e[k]);
          }
        }
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < KMAX; ++k)
          if (k < K) s += exp(e[k] - m);
        const double lpr = m + log(s);
        if (p == 0) lsum += lpr;
#pragma unroll
        for (int j = 0; j < CH; ++j) {
          const int k = p * CH + j;
          if (k < K) {
            const double r = exp(e[k] - lpr);
            const double r0 = r * x0, r1 = r * x1, r2 = r * x2;
            double* a = acc + j * kStats;
            a[0] += r;
            a[1] += r0; a[2] += r1; a[3] += r2;
            a[4] += r0 * x0; a[5] += r1 * x0; a[6] += r1 * x1;
            a[7] += r2 * x0; a[8] += r2 * x1; a[9] += r2 * x2;
          }
        }
      }
      // block sums: warps first (lane 0's butterfly result), then warps in order
#pragma unroll
      for (int v = 0; v < CH * kStats; ++v) {
        const double a = warp_sum(acc[v]);
        if (lane == 0) sh.wpart[warp][p * CH * kStats + v] = a;
      }
      if (p == 0) {
        const double a = warp_sum(lsum);
        if (lane == 0) sh.wpart[warp][kLsum] = a;
      }
    }
    __syncthreads();
    if (tid < kVals) {
      double s = 0.0;
      if (tid < K * kStats || tid == kLsum)
        for (int w = 0; w < kWarps; ++w) s += sh.wpart[w][tid];
      sh.stats[tid] = s;
    }
    cluster.sync();  // every block's sums are written

    // cluster totals (em2's reduction): every block adds the blocks' rows in rank order
    if (tid < kVals) {
      double s = 0.0;
      for (int r = 0; r < kCluster; ++r) s += cluster.map_shared_rank(sh.stats, r)[tid];
      sh.tot[tid] = s;
    }
    __syncthreads();
    if (tid == 0) {
      // eval + check_converge (GMM.pyx:283-329): the sum just formed is L of the model that
      // produced the responsibilities, i.e. of iteration t - 1
      const double L = sh.tot[kLsum];
      int stop = 0;
      if (t >= 1) {
        if (t - 1 > 1 && fabs(L - sh.lprev) < tol) {
          stop = 1;
          sh.converged = 1;
        }
        sh.lprev = L;
      }
      if (!stop && t == max_iter) stop = 1;
      sh.lcur = L;
      sh.iterations = t;
      if (!stop) m_step(sh, K, min_covar, full);
      sh.stop = stop;
    }
    cluster.sync();  // every block has read the others' sums; the new model is visible
    if (sh.stop) break;
  }

  if (rank == 0 && tid == 0) {
    for (int k = 0; k < kMaxK; ++k) {
      const bool on = k < K;
      out->weights[k] = on ? sh.w[k] : 0.0;
      for (int j = 0; j < 3; ++j) out->means[k][j] = on ? sh.mu[k][j] : 0.0;
      for (int j = 0; j < 6; ++j) out->covars[k][j] = on ? sh.S[k][j] : 0.0;
    }
    // the evaluation form computed at the top of the last iteration belongs to the returned
    // model: the loop stops before an M-step
    for (int k = 0; k < kMaxK; ++k) {
      const bool on = k < K && !sh.status;
      out->components[k].c = on ? sh.c[k] : 0.0;
      for (int j = 0; j < 3; ++j) out->components[k].mean[j] = on ? sh.mu[k][j] : 0.0;
      for (int j = 0; j < 6; ++j) out->components[k].li[j] = on ? sh.li[k][j] : 0.0;
    }
    out->log_likelihood = sh.lcur;
    out->iterations = sh.iterations;
    out->converged = sh.converged;
    out->status = sh.status;
    out->n_components = K;
  }
}

int fit_fail(const char* msg) { return gcut::set_last_error(GC_ERR_INVALID, msg); }

}  // namespace

extern "C" int gc_gmm_fit(const uint32_t* samples, int n, int n_components, int max_iterations,
                          double tolerance, double min_covar, double init_covar,
                          int full_covariance, gc_gmm_fit_result* result, void* stream) {
  gcut::set_last_error(GC_OK, "");
  if (n_components < 1 || n_components > kMaxK)
    return fit_fail("gc_gmm_fit: n_components must be 1..GC_GMM_MAX_COMPONENTS");
  if (n < n_components) return fit_fail("gc_gmm_fit: fewer samples than components");
  if (max_iterations < 1 || max_iterations > 100000)
    return fit_fail("gc_gmm_fit: max_iterations must be 1..100000");
  if (!std::isfinite(tolerance) || tolerance < 0.0) return fit_fail("gc_gmm_fit: bad tolerance");
  if (!std::isfinite(min_covar) || min_covar < 0.0) return fit_fail("gc_gmm_fit: bad min_covar");
  if (!std::isfinite(init_covar) || !(init_covar > 0.0))
    return fit_fail("gc_gmm_fit: init_covar must be > 0");
  if (!samples || !result) return fit_fail("gc_gmm_fit: null samples or result");
  cudaStream_t s = (cudaStream_t)stream;
  const int full = full_covariance ? 1 : 0;
  if (n_components <= 2)
    k_gmm_fit<2><<<kCluster, kThreads, 0, s>>>(samples, n, n_components, max_iterations,
                                                tolerance, min_covar, init_covar, full, result);
  else if (n_components <= 4)
    k_gmm_fit<4><<<kCluster, kThreads, 0, s>>>(samples, n, n_components, max_iterations,
                                                tolerance, min_covar, init_covar, full, result);
  else
    k_gmm_fit<8><<<kCluster, kThreads, 0, s>>>(samples, n, n_components, max_iterations,
                                                tolerance, min_covar, init_covar, full, result);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return gcut::set_last_error(GC_ERR_CUDA, cudaGetErrorString(e));
  return GC_OK;
}
