// Single-pass decoupled look-back scan and stream compaction (sm_100a).
//
// Replaces the reference's multi-launch Blelloch scan (prefixsum.cl:81-212, driven by
// PrefixSum.pyx:83-129), the scatter of streamcompact.cl:1-14 (StreamCompact.pyx:66-82)
// and the stamp predicates of incremental_tile_list.cl:40-154 (IncrementalTileList.pyx:
// 119-176).  One launch per scan/compaction: each CTA takes a chunk of 4096 items by
// arrival ticket, reduces it, publishes its aggregate and looks back over its
// predecessors' published prefixes.  The predicate is evaluated while loading, so the
// "flag" kernel of the reference disappears into the scan.  Compaction writes to a list
// separate from the flags (the reference scans in place into the list and then scatters
// into the same buffer, StreamCompact.pyx:72-81).
#include "gcut_common.cuh"
#include "gcut_internal.h"

namespace gcut {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 16;
constexpr int SCAN_CHUNK = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ bool op_apply(int op, int32_t v, int32_t a) {
  switch (op) {
    case 0: return v == a;   // OPERATOR_EQUAL
    case 1: return v > a;    // OPERATOR_GT
    case 2: return v < a;    // OPERATOR_LT
    case 3: return v >= a;   // OPERATOR_GTE
    default: return v <= a;  // OPERATOR_LTE
  }
}

struct ScanArgs {
  const int32_t* in;
  const int32_t* in2;
  int32_t* clear;        // optional: zeroed after reading (consumed flags)
  int32_t* scan_out;     // MODE_SCAN: exclusive scan
  int32_t* list_out;     // compaction modes: selected indices
  int32_t* total_out;    // scan total / list length
  int n;
  int mode;
  int op1, op2;
  int32_t a1, a2;
  int logical;           // 0 AND, 1 OR
};

__global__ void __launch_bounds__(SCAN_THREADS) k_scan(ScanArgs a, ScanState st) {
  __shared__ int32_t sm[32];
  __shared__ int32_t s_chunk, s_excl;
  __shared__ uint32_t s_tag;
  if (threadIdx.x == 0) {
    s_chunk = atomicAdd(st.ticket, 1);
    s_tag = *((volatile uint32_t*)st.seq);
  }
  __syncthreads();
  const int chunk = s_chunk;
  const int nchunks = (a.n + SCAN_CHUNK - 1) / SCAN_CHUNK > 0 ? (a.n + SCAN_CHUNK - 1) / SCAN_CHUNK : 1;
  const long long base = (long long)chunk * SCAN_CHUNK + (long long)threadIdx.x * SCAN_ITEMS;

  int32_t v[SCAN_ITEMS];
  int32_t raw[SCAN_ITEMS], raw2[SCAN_ITEMS];
  const bool vec = base + SCAN_ITEMS <= a.n && ((reinterpret_cast<uintptr_t>(a.in) & 15) == 0) &&
                   (a.mode != GC_SCAN_MODE_LOGICAL || (reinterpret_cast<uintptr_t>(a.in2) & 15) == 0);
  if (vec) {
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k += 4) {
      const int4 q = *reinterpret_cast<const int4*>(a.in + base + k);
      raw[k] = q.x; raw[k + 1] = q.y; raw[k + 2] = q.z; raw[k + 3] = q.w;
      if (a.mode == GC_SCAN_MODE_LOGICAL) {
        const int4 q2 = *reinterpret_cast<const int4*>(a.in2 + base + k);
        raw2[k] = q2.x; raw2[k + 1] = q2.y; raw2[k + 2] = q2.z; raw2[k + 3] = q2.w;
      }
    }
  } else {
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
      const long long i = base + k;
      raw[k] = i < a.n ? a.in[i] : 0;
      raw2[k] = (i < a.n && a.mode == GC_SCAN_MODE_LOGICAL) ? a.in2[i] : 0;
    }
  }
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    const long long i = base + k;
    int32_t x = 0;
    if (i < a.n) {
      switch (a.mode) {
        case GC_SCAN_MODE_SCAN: x = raw[k]; break;
        case GC_SCAN_MODE_COMPACT: x = raw[k] != 0; break;
        case GC_SCAN_MODE_FLAG: x = op_apply(a.op1, raw[k], a.a1); break;
        default: {
          const bool f1 = op_apply(a.op1, raw[k], a.a1), f2 = op_apply(a.op2, raw2[k], a.a2);
          x = a.logical == 0 ? (f1 && f2) : (f1 || f2);
        }
      }
      if (a.clear) a.clear[i] = 0;
    }
    v[k] = x;
  }
  int32_t tsum = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) tsum += v[k];
  int32_t agg;
  int32_t tex = block_exclusive_scan(tsum, sm, &agg);
  if (threadIdx.x < 32) {
    const int32_t ex = lookback_exclusive_warp(st, s_tag, chunk, agg);
    if (threadIdx.x == 0) s_excl = ex;
  }
  __syncthreads();
  int32_t run = s_excl + tex;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    long long i = base + k;
    if (i < a.n) {
      if (a.mode == GC_SCAN_MODE_SCAN) a.scan_out[i] = run;
      else if (v[k]) {
        if ((unsigned)run < (unsigned)a.n) a.list_out[run] = (int32_t)i;
        else atomicExch(st.err, 2);   // only after a look-back that gave up
      }
    }
    run += v[k];
  }
  if (chunk == nchunks - 1 && threadIdx.x == 0 && a.total_out) *a.total_out = s_excl + agg;
  // The last CTA to finish sees every CTA's error report: a compaction whose look-back gave
  // up returns length -1 (a list length is never negative), so the result itself says so.
  if (threadIdx.x == 0 && scan_finish(st, nchunks) && a.mode != GC_SCAN_MODE_SCAN &&
      a.total_out && *((volatile int32_t*)st.err) != 0)
    *a.total_out = -1;
}

// Exercises the bounded look-back wait.  One warp looks back from chunk 1 to a chunk 0 that
// never publishes (the host cleared its status word, whose tag 0 never matches a launch
// tag), so the wait gives up after st.spin_limit polls, sets the error word and returns.
// The launch then closes like a one-chunk scan (tickets reset, tag bumped), so the status
// word it published cannot be mistaken for a later launch's.
__global__ void k_lookback_selftest(ScanState st) {
  __shared__ uint32_t s_tag;
  if (threadIdx.x == 0) s_tag = *((volatile uint32_t*)st.seq);
  __syncthreads();
  if (threadIdx.x < 32) lookback_exclusive_warp(st, s_tag, 1, 0);
  if (threadIdx.x == 0) scan_finish(st, 1);
}

// IncrementalTileList.incorporate (incremental_tile_list.cl:110-154): stamp `iteration`
// where the combined predicate holds.
__global__ void k_increment_logical(const int32_t* in1, const int32_t* in2, int32_t* out,
                                    int n, int op1, int op2, int32_t a1, int32_t a2,
                                    int logical, int32_t iteration) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  bool f1 = op_apply(op1, in1[i], a1), f2 = op_apply(op2, in2[i], a2);
  if (logical == 0 ? (f1 && f2) : (f1 || f2)) out[i] = iteration;
}

__global__ void k_fill(int32_t* p, int n, int32_t v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

// IncrementalTileList.execute (IncrementalTileList.pyx:191-208; filter,
// incremental_tile_list.cl:156-175): one RGBA word per pixel, opaque red where the pixel's
// tile carries `iteration`, opaque black elsewhere.  Pixels outside the tile grid (an image
// side that is not a multiple of the tile side) are black; the reference has no bounds check
// there and reads past its tile array.
__global__ void k_tiles_view(const int32_t* __restrict__ tiles, int tiles_w, int tiles_h,
                             int tile_w, int tile_h, int32_t iteration, int width, long long n,
                             uint32_t* __restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i / width);
    const int x = (int)(i - (long long)y * width);
    const int tx = x / tile_w, ty = y / tile_h;
    bool on = false;
    if (tx < tiles_w && ty < tiles_h) on = tiles[(long long)ty * tiles_w + tx] == iteration;
    out[i] = on ? 0xFF0000FFu : 0xFF000000u;
  }
}

// Headless counterpart of the reference's display filters (graphcut_filter.cl:5-155: colorizef,
// HSVtoRGB and the tranpose / tilelist / tilelist_growcut kernels): each pixel takes the int32
// value of its cell (cell_w x cell_h pixels share one value: 1 x 1 for a pixel plane, the tile
// size for a tile map), maps it through an HSV ramp and blends the colour over the base image:
// out = base + (colour - base) * opacity per channel, every channel in [0, 1] (byte / 255).
// Below the range the colour is black (tested first, as colorizef, graphcut_filter.cl:29-48,
// does), above it white, inside it the hue, saturation and value run linearly between the
// ends (a range of one value maps it to the start, where the reference divides 0 by 0); its
// alpha is 0, as the reference's.  The arithmetic is float32
// with every rounding written out (no contraction), and the result is rounded to the nearest
// byte (ties to even).  Pixels outside the cell grid keep the base.
struct ViewRamp { float lo, hi, h0, h1, s0, s1, v0, v1, opacity; };

__device__ __forceinline__ float ramp_at(float a, float b, float t) {
  return __fadd_rn(a, __fmul_rn(t, __fsub_rn(b, a)));
}
__device__ __forceinline__ uint32_t unorm8(float f) {
  f = fminf(fmaxf(f, 0.0f), 1.0f);
  return (uint32_t)__float2int_rn(__fmul_rn(f, 255.0f));
}

__global__ void k_view_colorize(const int32_t* __restrict__ values, int values_w, int values_h,
                                int cell_w, int cell_h, int width, long long n, ViewRamp R,
                                const uint32_t* __restrict__ base, uint32_t* __restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i / width);
    const int x = (int)(i - (long long)y * width);
    const int cx = x / cell_w, cy = y / cell_h;
    const uint32_t b = base ? base[i] : 0u;
    if (cx >= values_w || cy >= values_h) { out[i] = b; continue; }
    const float v = __int2float_rn(values[(long long)cy * values_w + cx]);
    float H = 0.0f, S = 0.0f, V = 0.0f;
    if (v < R.lo) {
      // below the range: black
    } else if (v > R.hi) {
      V = 1.0f;
    } else {
      const float t = R.hi > R.lo ? __fdiv_rn(__fsub_rn(v, R.lo), __fsub_rn(R.hi, R.lo)) : 0.0f;
      H = ramp_at(R.h0, R.h1, t);
      S = ramp_at(R.s0, R.s1, t);
      V = ramp_at(R.v0, R.v1, t);
    }
    // HSV -> RGB over the sectors of the hue circle; sector 4 takes sector 5's (v, p, q) as the
    // reference's HSVtoRGB does, so hues 4/6..5/6 show as it shows them
    float c[3] = {0.0f, 0.0f, 0.0f};
    if (V != 0.0f) {
      const float h6 = __fmul_rn(H, 6.0f);
      const int sector = (int)__fsub_rn(h6, 1e-6f);   // truncated toward zero
      const float f = __fsub_rn(h6, (float)sector);
      const float p = __fmul_rn(V, __fsub_rn(1.0f, S));
      const float q = __fmul_rn(V, __fsub_rn(1.0f, __fmul_rn(S, f)));
      const float u = __fmul_rn(V, __fsub_rn(1.0f, __fmul_rn(S, __fsub_rn(1.0f, f))));
      switch (sector) {
        case 0: c[0] = V; c[1] = u; c[2] = p; break;
        case 1: c[0] = q; c[1] = V; c[2] = p; break;
        case 2: c[0] = p; c[1] = V; c[2] = u; break;
        case 3: c[0] = p; c[1] = q; c[2] = V; break;
        default: c[0] = V; c[1] = p; c[2] = q; break;
      }
    }
    uint32_t w = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float cb = __fdiv_rn((float)((b >> (8 * k)) & 0xffu), 255.0f);
      const float co = k < 3 ? c[k] : 0.0f;
      w |= unorm8(__fadd_rn(cb, __fmul_rn(__fsub_rn(co, cb), R.opacity))) << (8 * k);
    }
    out[i] = w;
  }
}

int launch_view_colorize(const int32_t* values, int values_w, int values_h, int cell_w,
                         int cell_h, int width, int height, const float* ramp9,
                         const uint32_t* base, uint32_t* out, cudaStream_t s) {
  const long long n = (long long)width * height;
  if (n <= 0) return GC_OK;
  const ViewRamp R{ramp9[0], ramp9[1], ramp9[2], ramp9[3], ramp9[4], ramp9[5], ramp9[6],
                   ramp9[7], ramp9[8]};
  const long long blocks = (n + 255) / 256;
  const unsigned grid = (unsigned)(blocks < (1LL << 30) ? blocks : (1LL << 30));
  k_view_colorize<<<grid, 256, 0, s>>>(values, values_w, values_h, cell_w, cell_h, width, n, R,
                                       base, out);
  return cudaGetLastError() == cudaSuccess ? GC_OK : GC_ERR_CUDA;
}

int launch_lookback_selftest(const ScanState& st, cudaStream_t s) {
  if (st.max_chunks < 2) return GC_ERR_INVALID;
  if (cudaMemsetAsync(st.status, 0, sizeof(unsigned long long), s) != cudaSuccess) return GC_ERR_CUDA;
  k_lookback_selftest<<<1, 32, 0, s>>>(st);
  return cudaGetLastError() == cudaSuccess ? GC_OK : GC_ERR_CUDA;
}

void preload_scan_kernels() {
  cudaFuncAttributes a;
  cudaFuncGetAttributes(&a, (const void*)k_lookback_selftest);
  cudaFuncGetAttributes(&a, (const void*)k_scan);
  cudaFuncGetAttributes(&a, (const void*)k_increment_logical);
  cudaFuncGetAttributes(&a, (const void*)k_fill);
  cudaFuncGetAttributes(&a, (const void*)k_tiles_view);
  cudaFuncGetAttributes(&a, (const void*)k_view_colorize);
}

int scan_chunks(int n) { return n <= 0 ? 1 : (n + SCAN_CHUNK - 1) / SCAN_CHUNK; }

int launch_scan(int mode, const int32_t* in, const int32_t* in2, int32_t* clear,
                int32_t* scan_out, int32_t* list_out, int32_t* total_out, int n, int op1,
                int32_t a1, int op2, int32_t a2, int logical, const ScanState& st,
                cudaStream_t s) {
  int nch = scan_chunks(n);
  if (nch > st.max_chunks) return GC_ERR_INVALID;
  ScanArgs a{in, in2, clear, scan_out, list_out, total_out, n, mode, op1, op2, a1, a2, logical};
  k_scan<<<nch, SCAN_THREADS, 0, s>>>(a, st);
  return cudaGetLastError() == cudaSuccess ? GC_OK : GC_ERR_CUDA;
}

int launch_increment_logical(const int32_t* in1, const int32_t* in2, int32_t* out, int n,
                             int op1, int op2, int32_t a1, int32_t a2, int logical,
                             int32_t iteration, cudaStream_t s) {
  if (n <= 0) return GC_OK;
  k_increment_logical<<<(n + 255) / 256, 256, 0, s>>>(in1, in2, out, n, op1, op2, a1, a2,
                                                       logical, iteration);
  return cudaGetLastError() == cudaSuccess ? GC_OK : GC_ERR_CUDA;
}

int launch_fill(int32_t* p, int n, int32_t v, cudaStream_t s) {
  if (n <= 0) return GC_OK;
  k_fill<<<(n + 255) / 256, 256, 0, s>>>(p, n, v);
  return cudaGetLastError() == cudaSuccess ? GC_OK : GC_ERR_CUDA;
}

int launch_tiles_view(const int32_t* tiles, int tiles_w, int tiles_h, int tile_w, int tile_h,
                      int32_t iteration, int width, int height, uint32_t* out, cudaStream_t s) {
  const long long n = (long long)width * height;
  if (n <= 0) return GC_OK;
  const long long blocks = (n + 255) / 256;
  const unsigned grid = (unsigned)(blocks < (1LL << 30) ? blocks : (1LL << 30));
  k_tiles_view<<<grid, 256, 0, s>>>(tiles, tiles_w, tiles_h, tile_w, tile_h, iteration, width,
                                    n, out);
  return cudaGetLastError() == cudaSuccess ? GC_OK : GC_ERR_CUDA;
}

}  // namespace gcut
