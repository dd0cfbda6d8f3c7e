// Tiled push-relabel kernels for sm_100a.
//
// Reference path: GraphCut.cut (GraphCut.pyx:348-418) driving graphcut.cl.  The reference
// runs one OpenCL kernel per push direction (push_down/up/right/left, graphcut.cl:158-536)
// with an 8-pixel wave per work-item, merges tile overspill with add_border (:114-156),
// relabels the whole image with a Jacobi pass (:538-577) and computes the global relabel
// with init_bfs/bfs_intratile/bfs_intertile (:582-1016) over compacted tile lists.  Here:
//
//  * k_discharge   one CTA of 256 threads per listed tile (persistent over the device-side
//                  list): the tile's excess, height and four residual planes arrive in shared
//                  memory by bulk copy (the next tile's copy overlaps this tile's work), with
//                  the halo heights, and the CTA runs `iters` rounds of {push along every
//                  admissible edge (all 4 directions), Jacobi relabel}.  Flow leaving the tile
//                  is added to the neighbour's excess and reverse residual with atomics (no
//                  border buffer, no add_border launch); tile-edge pixels rise at most 2 per
//                  launch, so the labelling stays valid whether a neighbouring CTA saw a
//                  pixel's start or final height.  Each finished
//                  tile's bookkeeping (next list, dirty flags) is settled in batches.
//  * k_edge_relabel_build   relabels the active tile-edge pixels (Jacobi) and rebuilds the
//                  active-tile list with the single-pass decoupled look-back compaction in
//                  the same launch (IncrementalTileList.build + StreamCompact + PrefixSum);
//                  the manual relabel step (GraphCut.relabel) only.
//  * k_bfs_round   exact global relabel: per tile, one warp runs a bit-parallel multi-source
//                  BFS (32-bit row masks of residual edges, lane = row) seeded by sink
//                  pixels and by the halo distances, and marks neighbours whose edge
//                  distances changed; the marked tiles form the next frontier.
//  * k_flood_round canonical cut: the same tile rounds flood the set reachable from excess
//                  pixels over residual edges (the minimal source set).
#include <cstdio>
#include <mutex>
#include <unordered_map>

#include "gcut_common.cuh"
#include "gcut_internal.h"

namespace gcut {

constexpr int DIS_THREADS = 256;
constexpr int DIS_LOG = 32;       // tiles per bookkeeping flush in k_discharge (<= DIS_THREADS / 5)
constexpr int WARPS_PER_CTA = 4;   // warp-per-tile kernels (BFS, flood, mask rebuild)

__device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }

// ------------------------------------------------------------------------------------
// Upload: row-major planes -> tile planes; boundary capacities zeroed; padding pixels are
// isolated (all zero).  Heights start at 0 for sink pixels and 1 otherwise (a valid
// labelling).  Replaces init_gc + load_tiles (graphcut.cl:63-112, 1033-1132).
// ------------------------------------------------------------------------------------
// Spreads bits 0..7 of x to bit positions 0, 4, ..., 28.
__device__ __forceinline__ uint32_t spread8(uint32_t x) {
  x &= 0xffu;
  x = (x | (x << 12)) & 0x000F000Fu;
  x = (x | (x << 6)) & 0x03030303u;
  x = (x | (x << 3)) & 0x11111111u;
  return x;
}

// Row mask of row (lane & 3) of this warp's four rows, from the ballots of the four pixels
// each thread holds (thread (g, q) of the warp holds pixels 4q..4q+3 of row g).
__device__ __forceinline__ uint32_t warp_row_mask(uint32_t b0, uint32_t b1, uint32_t b2, uint32_t b3,
                                                  int ri) {
  const int sh = 8 * ri;
  return spread8(b0 >> sh) | (spread8(b1 >> sh) << 1) | (spread8(b2 >> sh) << 2) |
         (spread8(b3 >> sh) << 3);
}

// Row masks of tile t (residual edge up / down / left / right, sink, positive excess) from
// the values the block's 256 threads hold: thread (r, q) holds pixels (r, 4q .. 4q+3).  The
// BFS and the flood read these instead of the planes.  Every thread of the block calls it.
__device__ __forceinline__ void write_tile_masks(const PoolView& P, int t, const int (&e)[4],
                                                 const int (&cu)[4], const int (&cd)[4],
                                                 const int (&cl)[4], const int (&cr)[4]) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned F = 0xffffffffu;
  uint32_t m[6];
  const int* planes4[4] = {cu, cd, cl, cr};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int* v = planes4[k];
    m[k] = warp_row_mask(__ballot_sync(F, v[0] > 0), __ballot_sync(F, v[1] > 0),
                         __ballot_sync(F, v[2] > 0), __ballot_sync(F, v[3] > 0), lane & 3);
  }
  m[4] = warp_row_mask(__ballot_sync(F, e[0] < 0), __ballot_sync(F, e[1] < 0),
                       __ballot_sync(F, e[2] < 0), __ballot_sync(F, e[3] < 0), lane & 3);
  m[5] = warp_row_mask(__ballot_sync(F, e[0] > 0), __ballot_sync(F, e[1] > 0),
                       __ballot_sync(F, e[2] > 0), __ballot_sync(F, e[3] > 0), lane & 3);
  if (lane < 4) {
    const int row = 4 * w + lane;
    uint32_t* mc = P.mcan + (long long)t * 128;
    mc[row] = m[0]; mc[32 + row] = m[1]; mc[64 + row] = m[2]; mc[96 + row] = m[3];
    P.msink[(long long)t * 32 + row] = m[4];
    P.mexc[(long long)t * 32 + row] = m[5];
  }
}

// Tile t's planes changed after its masks were written: the first flood round that covers
// it (or k_masks) rebuilds them.  A plain store: nothing reads the flag until a later kernel.
__device__ __forceinline__ void mark_dirty(const PoolView& P, int t) { P.mdirty[t] = 1; }

// Row masks of one tile row, as write_tile_masks writes them.
struct RowMasks { uint32_t up, down, left, right, sink, exc; };

// Rebuilds tile t's row masks and its sum of max(excess, 0) from its planes with one warp:
// lane c reads column c of four rows at a time (one 128-byte line per row and plane), and a
// ballot over the lanes is the row's mask.  Writes the masks and the sum, clears the dirty
// flag, and returns row `lane`'s masks to each lane and the tile's sum to every lane.
__device__ __forceinline__ RowMasks warp_rebuild_masks(const PoolView& P, int t, int lane,
                                                       long long* tile_pos) {
  const unsigned F = 0xffffffffu;
  const long long base = (long long)t * GC_TILE_PX + lane;
  RowMasks out{0u, 0u, 0u, 0u, 0u, 0u};
  long long pos = 0;
#pragma unroll 1
  for (int r0 = 0; r0 < GC_TILE; r0 += 4) {
    int v[4][5];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const long long o = base + (r0 + k) * GC_TILE;
      v[k][0] = P.exc[o];
      v[k][1] = P.cap[DUP][o];
      v[k][2] = P.cap[DDOWN][o];
      v[k][3] = P.cap[DLEFT][o];
      v[k][4] = P.cap[DRIGHT][o];
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint32_t mu = __ballot_sync(F, v[k][1] > 0), md = __ballot_sync(F, v[k][2] > 0);
      const uint32_t ml = __ballot_sync(F, v[k][3] > 0), mr = __ballot_sync(F, v[k][4] > 0);
      const uint32_t ms = __ballot_sync(F, v[k][0] < 0), me = __ballot_sync(F, v[k][0] > 0);
      if (lane == r0 + k) {
        out.up = mu; out.down = md; out.left = ml; out.right = mr;
        out.sink = ms; out.exc = me;
      }
      pos += v[k][0] > 0 ? v[k][0] : 0;
    }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) pos += __shfl_xor_sync(F, pos, o);
  uint32_t* mc = P.mcan + (long long)t * 128;
  mc[lane] = out.up;
  mc[32 + lane] = out.down;
  mc[64 + lane] = out.left;
  mc[96 + lane] = out.right;
  P.msink[(long long)t * 32 + lane] = out.sink;
  P.mexc[(long long)t * 32 + lane] = out.exc;
  if (lane == 0) {
    P.tpos[t] = pos;
    P.mdirty[t] = 0;
  }
  *tile_pos = pos;
  return out;
}

// Capacity sources of the upload.  PlaneSource: row-major capacity planes (gc_upload).
// RgbaSource: n-links built from an RGBA image and the n-link table (gc_upload_rgba).
struct PlaneSource {
  const int32_t *up, *down, *left, *right, *excess;
  bool vec;   // all planes 16-byte aligned and the width a multiple of 4: int4 row loads
  __device__ __forceinline__ void prepare(int32_t*) const {}
  // the four pixels (x0 .. x0+3, y) at once, all inside the image (x0 + 3 < W)
  __device__ __forceinline__ void pixel4(const ImageDesc& im, int x0, int y, int (&e)[4],
                                         int (&cu)[4], int (&cd)[4], int (&cl)[4],
                                         int (&cr)[4]) const {
    const long long i = (long long)y * im.W + x0;
    const int4 a = *reinterpret_cast<const int4*>(excess + i);
    const int4 b = *reinterpret_cast<const int4*>(up + i);
    const int4 c = *reinterpret_cast<const int4*>(down + i);
    const int4 d = *reinterpret_cast<const int4*>(left + i);
    const int4 f = *reinterpret_cast<const int4*>(right + i);
    e[0] = a.x; e[1] = a.y; e[2] = a.z; e[3] = a.w;
    const bool top = y == 0, bottom = y == im.H - 1;
    cu[0] = top ? 0 : b.x; cu[1] = top ? 0 : b.y; cu[2] = top ? 0 : b.z; cu[3] = top ? 0 : b.w;
    cd[0] = bottom ? 0 : c.x; cd[1] = bottom ? 0 : c.y; cd[2] = bottom ? 0 : c.z; cd[3] = bottom ? 0 : c.w;
    cl[0] = x0 == 0 ? 0 : d.x; cl[1] = d.y; cl[2] = d.z; cl[3] = d.w;
    cr[0] = f.x; cr[1] = f.y; cr[2] = f.z; cr[3] = x0 + 3 == im.W - 1 ? 0 : f.w;
  }
  __device__ __forceinline__ void pixel(const ImageDesc& im, const int32_t*, int x, int y, int& e,
                                        int& cu, int& cd, int& cl, int& cr) const {
    const long long i = (long long)y * im.W + x;
    e = excess[i];
    cu = y > 0 ? up[i] : 0;
    cd = y < im.H - 1 ? down[i] : 0;
    cl = x > 0 ? left[i] : 0;
    cr = x < im.W - 1 ? right[i] : 0;
  }
};

__device__ __forceinline__ int rgb_dist2(uint32_t a, uint32_t b) {
  const int dr = (int)(a & 255u) - (int)(b & 255u);
  const int dg = (int)((a >> 8) & 255u) - (int)((b >> 8) & 255u);
  const int db = (int)((a >> 16) & 255u) - (int)((b >> 16) & 255u);
  return dr * dr + dg * dg + db * db;
}

// Weight of the reference's n-link rule, rounded to an integer: floor(x + 0.5) for
// x = lambda / (0.1 sqrt(d) + 0.05) = 20 lambda / (2 sqrt(d) + 1) (graphcut.cl:1018-1031,
// LAMBDA and EPSILON from GraphCut.pyx:25-26,92-93), exactly.  For k >= 1,
// floor(x + 0.5) >= k  <=>  b = 40 lambda - 2k + 1 >= 0  and  4 (2k - 1)^2 d <= b^2,
// so the weight is the largest k satisfying that integer test (monotone in k).  A double
// estimate of k is settled by the test itself; with lambda <= 1000 and d <= 3 * 255^2 every
// product fits in 64 bits.
__device__ __forceinline__ bool ref_weight_at_least(long long k, long long d, long long a40) {
  if (k < 1) return true;
  const long long b = a40 - 2 * k + 1, a = 2 * k - 1;
  return b >= 0 && 4 * a * a * d <= b * b;
}
__device__ __forceinline__ int ref_weight(int d, int lambda) {
  const long long a40 = 40LL * lambda;
  const double sd = sqrt((double)d);
  long long k = (long long)floor(((double)a40 + 1.0 + 2.0 * sd) / (4.0 * sd + 2.0));
  if (k < 0) k = 0;
  while (k > 0 && !ref_weight_at_least(k, d, a40)) --k;
  while (ref_weight_at_least(k + 1, d, a40)) ++k;
  return (int)k;
}

struct RgbaSource {
  const uint32_t* rgba;
  const int32_t* excess;
  const int32_t* tab;   // exp weighting: the 50 thresholds on the device; null: reference rule
  int lambda;           // reference weighting
  static constexpr bool vec = false;
  __device__ __forceinline__ void pixel4(const ImageDesc&, int, int, int (&)[4], int (&)[4],
                                         int (&)[4], int (&)[4], int (&)[4]) const {}
  __device__ __forceinline__ void prepare(int32_t* s_tab) const {
    if (tab && threadIdx.x < GC_NLINK_LEVELS) s_tab[threadIdx.x] = tab[threadIdx.x];
  }
  // exp weighting: the number of table entries >= d (the entries do not increase)
  __device__ __forceinline__ static int table_weight(const int32_t* s_tab, int d) {
    int lo = 0, hi = GC_NLINK_LEVELS;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (s_tab[mid] >= d) lo = mid + 1; else hi = mid;
    }
    return lo;
  }
  __device__ __forceinline__ int weight(const int32_t* s_tab, int d) const {
    return tab ? table_weight(s_tab, d) : ref_weight(d, lambda);
  }
  __device__ __forceinline__ void pixel(const ImageDesc& im, const int32_t* s_tab, int x, int y,
                                        int& e, int& cu, int& cd, int& cl, int& cr) const {
    const long long i = (long long)y * im.W + x;
    const uint32_t c = rgba[i];
    e = excess[i];
    cu = y > 0 ? weight(s_tab, rgb_dist2(c, rgba[i - im.W])) : 0;
    cd = y < im.H - 1 ? weight(s_tab, rgb_dist2(c, rgba[i + im.W])) : 0;
    cl = x > 0 ? weight(s_tab, rgb_dist2(c, rgba[i - 1])) : 0;
    cr = x < im.W - 1 ? weight(s_tab, rgb_dist2(c, rgba[i + 1])) : 0;
  }
};

// The exp weighting's table on the device, from the |dI|^2 sum of k_dsum: weight(d) =
// floor(50 exp(-beta d) + 0.5) with beta = 1 / (2 mean |dI|^2) (0 when the mean is 0) does
// not increase with d, so it is stored as t[k - 1] = the largest d in [0, 3 * 255^2] with
// weight >= k.  Thread k - 1 locates t[k - 1] from the real root of 50 exp(-beta d) + 0.5
// = k and settles it by evaluating the formula itself at the integers around it, in double,
// so the table reproduces a float64 evaluation of the formula pixel by pixel.
__global__ void k_nlink_table(const unsigned long long* __restrict__ sum, long long npairs,
                              int32_t* __restrict__ tab) {
  const int k = (int)threadIdx.x + 1;
  if (k > GC_NLINK_LEVELS) return;
  const long kMax = 3L * 255 * 255;
  const double mean = (double)(*sum) / (double)(npairs > 1 ? npairs : 1);
  const double beta = mean > 0 ? 1.0 / (2.0 * mean) : 0.0;
  if (beta <= 0) { tab[k - 1] = (int32_t)kMax; return; }
  auto w = [&](long d) { return (int)floor(50.0 * exp(-beta * (double)d) + 0.5); };
  const double root = log(50.0 / (k - 0.5)) / beta;   // weight(d) >= k  <=>  d <= root
  long d = root >= (double)kMax ? kMax : (root < 0 ? 0 : (long)floor(root));
  while (d < kMax && w(d + 1) >= k) ++d;
  while (d >= 0 && w(d) < k) --d;
  tab[k - 1] = (int32_t)d;
}

template <class Source>
__global__ void __launch_bounds__(DIS_THREADS)
k_upload(PoolView P, ImageDesc im, int img, Source src, int32_t* __restrict__ tl, ImageAcc* acc) {
  trace_mark(P, TR_UPLOAD);
  __shared__ int32_t s_tab[GC_NLINK_LEVELS];
  src.prepare(s_tab);
  __syncthreads();
  const int bt = blockIdx.x;
  const int tx = bt % im.tw, ty = bt / im.tw;
  const int t = im.tile0 + bt;
  const int r = threadIdx.x >> 3, c0 = (threadIdx.x & 7) * 4;
  const int y = ty * GC_TILE + r;
  int e[4], h[4], cu[4], cd[4], cl[4], cr[4];
  long long pos = 0;
  int bad = 0, anypos = 0;
  const int xb = tx * GC_TILE + c0;
  if (src.vec && y < im.H && xb + 3 < im.W) {
    src.pixel4(im, xb, y, e, cu, cd, cl, cr);
  } else {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int x = xb + j;
      e[j] = cu[j] = cd[j] = cl[j] = cr[j] = 0;
      if (x < im.W && y < im.H) src.pixel(im, s_tab, x, y, e[j], cu[j], cd[j], cl[j], cr[j]);
    }
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    bad |= (cu[j] | cd[j] | cl[j] | cr[j]) < 0;
    h[j] = e[j] < 0 ? 0 : 1;
    pos += e[j] > 0 ? e[j] : 0;
    anypos |= e[j] > 0;
  }
  const long long off = (long long)t * GC_TILE_PX + r * GC_TILE + c0;
  *(int4*)(P.exc + off) = make_int4(e[0], e[1], e[2], e[3]);
  *(int4*)(tl + off) = make_int4(e[0], e[1], e[2], e[3]);
  *(int4*)(P.hgt + off) = make_int4(h[0], h[1], h[2], h[3]);
  *(int4*)(P.cap[DUP] + off) = make_int4(cu[0], cu[1], cu[2], cu[3]);
  *(int4*)(P.cap[DDOWN] + off) = make_int4(cd[0], cd[1], cd[2], cd[3]);
  *(int4*)(P.cap[DLEFT] + off) = make_int4(cl[0], cl[1], cl[2], cl[3]);
  *(int4*)(P.cap[DRIGHT] + off) = make_int4(cr[0], cr[1], cr[2], cr[3]);
  write_tile_masks(P, t, e, cu, cd, cl, cr);
  if (threadIdx.x < 32) P.mreach[(long long)t * 32 + threadIdx.x] = 0u;   // no flood yet
  __shared__ long long wpos[DIS_THREADS / 32];
#pragma unroll
  for (int o = 16; o; o >>= 1) pos += __shfl_xor_sync(0xffffffffu, pos, o);
  if ((threadIdx.x & 31) == 0) wpos[threadIdx.x >> 5] = pos;
  bad = __syncthreads_or(bad);
  anypos = __syncthreads_or(anypos);
  if (threadIdx.x == 0) {
    long long tp = 0;
    for (int k = 0; k < DIS_THREADS / 32; ++k) tp += wpos[k];
    P.tpos[t] = tp;
    // one add per tile: the adds of all of an image's tiles go to one address
    if (tp) atomicAdd(&acc[img].sumpos_t, (unsigned long long)tp);
    if (bad) atomicAdd(&acc[img].bad_caps, 1);
    P.tact[t] = anypos;
    P.touched[t] = 0;
    P.act_int[t] = 0;
    P.mark[0][t] = 0;
    P.mark[1][t] = 0;
    P.inq[0][t] = 0;
    P.inq[1][t] = 0;
    P.img_of[t] = img;
    P.mdirty[t] = 0;     // the masks above are current
  }
}

// Mask rebuild of the selected tiles whose planes changed since their masks were written
// (dirty flag set), one warp per tile.  The solve loops do not need it: their first flood
// round rebuilds the dirty tiles it covers.  It precedes a global relabel that no flood
// precedes (gc_start_bfs).
__global__ void __launch_bounds__(WARPS_PER_CTA * 32)
k_masks(PoolView P) {
  trace_mark(P, TR_MASKS);
  __shared__ int s_n, s_nr;
  if (threadIdx.x == 0) {
    int n = *((volatile int32_t*)&P.nsel[1]), nr = *((volatile int32_t*)&P.nsel[0]);
    if (n < 0 || n > P.nt || nr < 0 || nr > P.nimg) {   // self-check
      record_bad(P, 9, n);
      n = nr = 0;
    }
    s_n = n;
    s_nr = nr;
  }
  __syncthreads();
  const int n = s_n;
  const int lane = threadIdx.x & 31;
  const int i0 = blockIdx.x * WARPS_PER_CTA + (threadIdx.x >> 5);
  const int stride = gridDim.x * WARPS_PER_CTA;
  SelCursor cursor(P, s_nr, i0 < n ? i0 : 0);
  for (int i = i0; i < n; i += stride) {
    const int t = cursor.tile(i);
    if (P.mdirty[t] == 0) continue;   // the same word for every lane: warp-uniform
    long long pos;
    warp_rebuild_masks(P, t, lane, &pos);
    if (lane == 0 && P.ktiles) atomicAdd(&P.ktiles[K_MASKS], 1ull);
  }
}

// ------------------------------------------------------------------------------------
// Discharge.  Thread (r, q) owns pixels (r, 4q .. 4q+3) of the tile.
//
// Every pixel pushes along all admissible edges and relabels, tile-edge pixels included,
// but a tile-edge pixel rises by at most 2 above its height at the start of the launch.
// A neighbouring CTA that pushes into an edge pixel v saw either v's start height or its
// final height; with h_final(v) <= h_start(v) + 2 every such push leaves a valid labelling
// (h(v) <= h(u) + 1 on the new residual edge v -> u), and pushes out of the tile read the
// neighbour's height under the same bound.  Flow leaving the tile is added to the
// neighbour's excess and reverse residual with atomics at the end of the tile.
//
// Active tiles form a worklist: the launch reads queue[c] (c = pulse parity, device-side)
// and appends, deduplicated by inq[c ^ 1], every tile that is still active or received flow
// to queue[c ^ 1]; the last CTA advances the parity.  One launch per pulse, no compaction.
// ------------------------------------------------------------------------------------
struct DisSmem {
  int32_t hs[GC_TILE_PX];   // heights
  int32_t fu[GC_TILE_PX];   // flow pushed up by each pixel this round
  int32_t fd[GC_TILE_PX];   // flow pushed down
  int32_t fl[GC_TILE * 8];  // flow pushed left by the first pixel of each 4-pixel strip
  int32_t fr[GC_TILE * 8];  // flow pushed right by the last pixel of each strip
  int32_t hu[GC_TILE], hd[GC_TILE], hl[GC_TILE], hr[GC_TILE];  // halo heights
  // launch-start values of the tile-edge pixels that also receive atomics from the
  // neighbouring tiles (written back as deltas against these)
  int32_t eo_top[GC_TILE], eo_bot[GC_TILE], eo_left[GC_TILE], eo_right[GC_TILE];
  int32_t cu_top[GC_TILE], cd_bot[GC_TILE], cl_left[GC_TILE], cr_right[GC_TILE];
  // flow leaving the tile, per edge pixel, delivered at the end of the tile
  int32_t xu[GC_TILE], xd[GC_TILE], xl[GC_TILE], xr[GC_TILE];
};

__device__ __forceinline__ void worklist_add(const PoolView& P, int nxt, int t) {
  if (*((volatile int32_t*)&P.inq[nxt][t]) != 0) return;   // common case: already queued
  if (atomicExch(&P.inq[nxt][t], 1) == 0) {
    const int pos = atomicAdd(&P.qcount[nxt], 1);
    if (pos < P.nt) P.queue[nxt][pos] = t;   // inq deduplicates, so pos < nt always holds
    else record_bad(P, 1, pos);
  }
}

__device__ __forceinline__ int4 lds4(const int32_t* p) { return *reinterpret_cast<const int4*>(p); }
__device__ __forceinline__ void sts4(int32_t* p, int a, int b, int c, int d) {
  *reinterpret_cast<int4*>(p) = make_int4(a, b, c, d);
}

// Bulk copies global -> shared memory (cp.async.bulk, completion on an mbarrier).  The
// copies are plain (no cluster multicast); every wait on the mbarrier is bounded.
__device__ __forceinline__ void mbar_init(uint64_t* mbar, unsigned count) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(mbar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* mbar, unsigned bytes) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(mbar);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* mbar) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const unsigned m = (unsigned)__cvta_generic_to_shared(mbar);
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(d), "l"(src), "r"(bytes), "r"(m) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* mbar, unsigned parity) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(mbar);
  unsigned ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
               : "=r"(ok) : "r"(a), "r"(parity) : "memory");
  return ok != 0;
}
// A tile copy normally lands in microseconds; a wait gives up after this long.  The bound
// is on time, not on polls: try_wait may return at once, and a poll count then would allow
// only milliseconds under load (a CTA that gave up early would leave while its copy is
// still landing in shared memory).
constexpr unsigned long long GC_COPY_WAIT_NS = 2000000000ull;
// Bounded wait: false when the copy did not complete within limit_ns.  The iteration cap
// only guards against a timer that does not advance.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, unsigned parity,
                                          unsigned long long limit_ns = GC_COPY_WAIT_NS) {
  if (mbar_try_wait(mbar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (unsigned i = 1; i < (1u << 31); ++i) {
    if (mbar_try_wait(mbar, parity)) return true;
    if ((i & 255u) == 0 && global_ns() - t0 > limit_ns) return false;
  }
  return false;
}

constexpr int DIS_PLANES = 6;                                  // excess, height, 4 residuals
constexpr unsigned DIS_TILE_BYTES = DIS_PLANES * GC_TILE_PX * 4;  // 24 KiB
// dynamic shared memory: the tile staging buffer + the per-round exchange arrays
constexpr size_t DIS_DYN_SMEM = (size_t)DIS_TILE_BYTES + sizeof(DisSmem);

__device__ __forceinline__ const int32_t* dis_plane(const PoolView& P, int k) {
  return k == 0 ? P.exc : k == 1 ? P.hgt : P.cap[k - 2];
}

// Thread 0: start the bulk copy of tile t's six planes into buffer `buf`.
__device__ __forceinline__ void dis_prefetch(const PoolView& P, int t, int32_t* buf, uint64_t* mbar) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // buffer was last read by threads
  mbar_expect_tx(mbar, DIS_TILE_BYTES);
#pragma unroll
  for (int k = 0; k < DIS_PLANES; ++k)
    bulk_g2s(buf + k * GC_TILE_PX, dis_plane(P, k) + (long long)t * GC_TILE_PX, GC_TILE_PX * 4, mbar);
}

__global__ void __launch_bounds__(DIS_THREADS, 4)
k_discharge(PoolView P, int iters) {
  trace_mark(P, TR_DISCHARGE);
  extern __shared__ __align__(128) int32_t dsm[];
  int32_t* const buf = dsm;                                    // [6][1024] staging
  DisSmem& S = *reinterpret_cast<DisSmem*>(dsm + DIS_PLANES * GC_TILE_PX);
  __shared__ uint64_t mbar;
  __shared__ int s_cur, s_n, s_sent;
  const int tid = threadIdx.x;
  const int r = tid >> 3, q = tid & 7, c0 = q * 4;
  if (tid == 0) {
    s_cur = *((volatile int32_t*)&P.ctl[CTL_PULSE]) & 1;
    s_n = *((volatile int32_t*)&P.qcount[s_cur]);
    mbar_init(&mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const int cur = s_cur, nxt = cur ^ 1;
  // Bookkeeping log: each finished tile leaves (tile, neighbours, flags) here, and the CTA's
  // threads settle up to DIS_LOG tiles at once (its list entry, and the list entries and
  // dirty flags of the neighbours it sent flow to), so the dependent L2 round trips of that
  // bookkeeping are paid once per flush, not once per tile.  Nothing in this launch reads
  // what it writes: the next list, the dirty flags and act_int are read by later kernels.
  __shared__ int s_logt[DIS_LOG], s_logf[DIS_LOG];
  __shared__ int4 s_lognb[DIS_LOG];
  int nlog = 0;   // the same in every thread
  auto flush_log = [&](int cnt) {
    for (int w = tid; w < cnt * 5; w += DIS_THREADS) {
      const int i = w / 5, k = w - i * 5;       // k = 0: the tile; 1..4: up, down, left, right
      const int tt = s_logt[i], f = s_logf[i];
      const int4 nbb = s_lognb[i];
      const int target = k == 0 ? tt : k == 1 ? nbb.x : k == 2 ? nbb.y : k == 3 ? nbb.z : nbb.w;
      if (k == 0 || ((f >> (k - 1)) & 1)) {
        P.touched[target] = 1;
        mark_dirty(P, target);   // its masks are rebuilt by the next flood's first round
        if (k == 0) P.act_int[tt] = (f >> 5) & 1;
        if (k != 0 || ((f >> 4) & 1)) worklist_add(P, nxt, target);
        if (k == 0 && P.ktiles) atomicAdd(&P.ktiles[K_DISCHARGE], 1ull);
      }
    }
  };
  int n = s_n;
  if (n < 0 || n > P.nt) {   // self-check: a list never holds more than every tile once
    if (tid == 0 && blockIdx.x == 0) record_bad(P, 2, n);
    n = 0;
  }
  // list entry li: every position below the checked count was written with a tile id of
  // the pool (by worklist_add or the compaction) before this launch
  auto entry = [&](int li) { return P.queue[cur][li]; };
  const bool erow = (r == 0) || (r == 31);
  const int pix = r * GC_TILE + c0;
  unsigned phase = 0;
  bool failed = false, pending = false;
  if (tid == 0 && (int)blockIdx.x < n) dis_prefetch(P, entry(blockIdx.x), buf, &mbar);
  for (int li = blockIdx.x; li < n; li += gridDim.x) {
    const int t = entry(li);
    const int4 nb = P.nbr[t];
    if (tid < 32) S.hu[tid] = nb.x >= 0 ? P.hgt[(long long)nb.x * GC_TILE_PX + 31 * GC_TILE + tid] : GC_HINF;
    else if (tid < 64) S.hd[tid - 32] = nb.y >= 0 ? P.hgt[(long long)nb.y * GC_TILE_PX + (tid - 32)] : GC_HINF;
    else if (tid < 96) S.hl[tid - 64] = nb.z >= 0 ? P.hgt[(long long)nb.z * GC_TILE_PX + (tid - 64) * GC_TILE + 31] : GC_HINF;
    else if (tid < 128) S.hr[tid - 96] = nb.w >= 0 ? P.hgt[(long long)nb.w * GC_TILE_PX + (tid - 96) * GC_TILE] : GC_HINF;
    else if (tid < 160) S.xu[tid - 128] = 0;
    else if (tid < 192) S.xd[tid - 160] = 0;
    else if (tid < 224) S.xl[tid - 192] = 0;
    else S.xr[tid - 224] = 0;
    if (tid == 0) { P.inq[cur][t] = 0; s_sent = 0; }
    const bool ok = mbar_wait(&mbar, phase);
    if (__syncthreads_or(!ok)) { failed = true; pending = true; break; }  // block-uniform
    phase ^= 1u;
    int e[4], h[4], cu[4], cd[4], cl[4], cr[4];
    {
      int4 v = lds4(buf + 0 * GC_TILE_PX + pix); e[0] = v.x; e[1] = v.y; e[2] = v.z; e[3] = v.w;
      v = lds4(buf + 1 * GC_TILE_PX + pix); h[0] = v.x; h[1] = v.y; h[2] = v.z; h[3] = v.w;
      v = lds4(buf + 2 * GC_TILE_PX + pix); cu[0] = v.x; cu[1] = v.y; cu[2] = v.z; cu[3] = v.w;
      v = lds4(buf + 3 * GC_TILE_PX + pix); cd[0] = v.x; cd[1] = v.y; cd[2] = v.z; cd[3] = v.w;
      v = lds4(buf + 4 * GC_TILE_PX + pix); cl[0] = v.x; cl[1] = v.y; cl[2] = v.z; cl[3] = v.w;
      v = lds4(buf + 5 * GC_TILE_PX + pix); cr[0] = v.x; cr[1] = v.y; cr[2] = v.z; cr[3] = v.w;
    }
    // keep the launch-start values the write-back needs (tile-edge pixels only)
    if (r == 0) {
#pragma unroll
      for (int j = 0; j < 4; ++j) { S.eo_top[c0 + j] = e[j]; S.cu_top[c0 + j] = cu[j]; }
    }
    if (r == 31) {
#pragma unroll
      for (int j = 0; j < 4; ++j) { S.eo_bot[c0 + j] = e[j]; S.cd_bot[c0 + j] = cd[j]; }
    }
    if (q == 0) { S.eo_left[r] = e[0]; S.cl_left[r] = cl[0]; }
    if (q == 7) { S.eo_right[r] = e[3]; S.cr_right[r] = cr[3]; }
    // height cap of tile-edge pixels for this launch (interior: none)
    int hcap[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = c0 + j;
      const bool edge = erow || c == 0 || c == 31;
      hcap[j] = edge ? (h[j] >= GC_HINF - 2 ? GC_HINF : h[j] + 2) : GC_HINF;
    }
    sts4(S.hs + pix, h[0], h[1], h[2], h[3]);
    __syncthreads();   // every thread has its values in registers: the buffer is free
    // prefetch this CTA's next tile into the buffer while this one is worked on
    if (tid == 0 && li + (int)gridDim.x < n) dis_prefetch(P, entry(li + gridDim.x), buf, &mbar);

    for (int it = 0; it < iters; ++it) {
      // neighbour heights (fixed during the push phase)
      int hnu[4], hnd[4], hnl[4], hnr[4];
      if (r > 0) { const int4 v = lds4(S.hs + pix - GC_TILE); hnu[0] = v.x; hnu[1] = v.y; hnu[2] = v.z; hnu[3] = v.w; }
      else { const int4 v = lds4(S.hu + c0); hnu[0] = v.x; hnu[1] = v.y; hnu[2] = v.z; hnu[3] = v.w; }
      if (r < 31) { const int4 v = lds4(S.hs + pix + GC_TILE); hnd[0] = v.x; hnd[1] = v.y; hnd[2] = v.z; hnd[3] = v.w; }
      else { const int4 v = lds4(S.hd + c0); hnd[0] = v.x; hnd[1] = v.y; hnd[2] = v.z; hnd[3] = v.w; }
      hnl[0] = c0 > 0 ? S.hs[pix - 1] : S.hl[r];
      hnl[1] = h[0]; hnl[2] = h[1]; hnl[3] = h[2];
      hnr[0] = h[1]; hnr[1] = h[2]; hnr[2] = h[3];
      hnr[3] = c0 < 28 ? S.hs[pix + 4] : S.hr[r];

      // push phase.  `rem` marks pixels that still hold excess after pushing: every
      // admissible edge of theirs is then saturated, and inflow only adds residual towards
      // higher neighbours, so they relabel without another admissibility test.
      int ou[4], od[4], ol[4], orr[4];
      int changed = 0;
      unsigned rem = 0;
#pragma unroll
      for (int j = 0; j < 4; ++j) ou[j] = od[j] = ol[j] = orr[j] = 0;
      const bool any_act = (e[0] > 0 && h[0] < GC_HINF) || (e[1] > 0 && h[1] < GC_HINF) ||
                           (e[2] > 0 && h[2] < GC_HINF) || (e[3] > 0 && h[3] < GC_HINF);
      if (__any_sync(0xffffffffu, any_act)) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          int ej = e[j];
          if (ej > 0 && h[j] < GC_HINF) {
            const int hm1 = h[j] - 1;
            if (cd[j] > 0 && hnd[j] == hm1) { const int f = imin(ej, cd[j]); ej -= f; cd[j] -= f; od[j] = f; }
            if (ej > 0 && cu[j] > 0 && hnu[j] == hm1) { const int f = imin(ej, cu[j]); ej -= f; cu[j] -= f; ou[j] = f; }
            if (ej > 0 && cr[j] > 0 && hnr[j] == hm1) { const int f = imin(ej, cr[j]); ej -= f; cr[j] -= f; orr[j] = f; }
            if (ej > 0 && cl[j] > 0 && hnl[j] == hm1) { const int f = imin(ej, cl[j]); ej -= f; cl[j] -= f; ol[j] = f; }
            changed |= ej != e[j];
            rem |= (ej > 0 ? 1u : 0u) << j;
            e[j] = ej;
          }
        }
      }
      // flow leaving the tile is delivered at the end of the tile
      if (r == 0) {
#pragma unroll
        for (int j = 0; j < 4; ++j) { S.xu[c0 + j] += ou[j]; ou[j] = 0; }
      }
      if (r == 31) {
#pragma unroll
        for (int j = 0; j < 4; ++j) { S.xd[c0 + j] += od[j]; od[j] = 0; }
      }
      if (q == 0) { S.xl[r] += ol[0]; ol[0] = 0; }
      if (q == 7) { S.xr[r] += orr[3]; orr[3] = 0; }
      sts4(S.fu + pix, ou[0], ou[1], ou[2], ou[3]);
      sts4(S.fd + pix, od[0], od[1], od[2], od[3]);
      S.fl[r * 8 + q] = ol[0];
      S.fr[r * 8 + q] = orr[3];
      __syncthreads();
      // gather inflow; a pixel receiving flow gains the reverse residual
      {
        const int4 a = r < 31 ? lds4(S.fu + pix + GC_TILE) : make_int4(0, 0, 0, 0);
        const int4 bb = r > 0 ? lds4(S.fd + pix - GC_TILE) : make_int4(0, 0, 0, 0);
        const int fb[4] = {a.x, a.y, a.z, a.w}, fa[4] = {bb.x, bb.y, bb.z, bb.w};
        int fromleft[4], fromright[4];
        fromleft[0] = q > 0 ? S.fr[r * 8 + q - 1] : 0;
        fromleft[1] = orr[0]; fromleft[2] = orr[1]; fromleft[3] = orr[2];
        fromright[0] = ol[1]; fromright[1] = ol[2]; fromright[2] = ol[3];
        fromright[3] = q < 7 ? S.fl[r * 8 + q + 1] : 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          e[j] += fb[j] + fa[j] + fromleft[j] + fromright[j];
          cd[j] += fb[j];
          cu[j] += fa[j];
          cl[j] += fromleft[j];
          cr[j] += fromright[j];
        }
      }
      // relabel phase (Jacobi; tile-edge pixels are capped at hcap)
      int nh[4] = {h[0], h[1], h[2], h[3]};
      const bool any_need = (e[0] > 0 && h[0] < hcap[0]) || (e[1] > 0 && h[1] < hcap[1]) ||
                            (e[2] > 0 && h[2] < hcap[2]) || (e[3] > 0 && h[3] < hcap[3]);
      if (__any_sync(0xffffffffu, any_need)) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          if (e[j] > 0 && h[j] < hcap[j]) {
            const int hm1 = h[j] - 1;
            const bool adm = !((rem >> j) & 1u) &&
                             ((cd[j] > 0 && hnd[j] == hm1) || (cu[j] > 0 && hnu[j] == hm1) ||
                              (cr[j] > 0 && hnr[j] == hm1) || (cl[j] > 0 && hnl[j] == hm1));
            if (!adm) {
              int m = GC_HINF;
              if (cd[j] > 0) m = imin(m, hnd[j] + 1);
              if (cu[j] > 0) m = imin(m, hnu[j] + 1);
              if (cr[j] > 0) m = imin(m, hnr[j] + 1);
              if (cl[j] > 0) m = imin(m, hnl[j] + 1);
              nh[j] = imin(imin(m, GC_HINF), hcap[j]);
              changed |= nh[j] != h[j];
            }
          }
        }
      }
      // every read of S.hs in this iteration happened before the flow barrier above, so the
      // new heights can be written now; the next reads follow the barrier below
#pragma unroll
      for (int j = 0; j < 4; ++j) h[j] = nh[j];
      sts4(S.hs + pix, h[0], h[1], h[2], h[3]);
      if (!__syncthreads_or(changed)) break;
    }

    // write back: interior values are owned by this CTA; tile-edge excess and the
    // outward residual of edge pixels also receive atomics from neighbouring tiles, so
    // they are written as deltas against their launch-start values.
    const long long off = (long long)t * GC_TILE_PX + pix;
    if (!erow && q > 0 && q < 7) {
      *(int4*)(P.exc + off) = make_int4(e[0], e[1], e[2], e[3]);
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = c0 + j;
        if (erow || c == 0 || c == 31) {
          const int e0 = r == 0 ? S.eo_top[c] : r == 31 ? S.eo_bot[c] : c == 0 ? S.eo_left[r] : S.eo_right[r];
          if (e[j] != e0) atomicAdd(P.exc + off + j, e[j] - e0);
        } else {
          P.exc[off + j] = e[j];
        }
      }
    }
    *(int4*)(P.hgt + off) = make_int4(h[0], h[1], h[2], h[3]);
    if (r == 0) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int o0 = S.cu_top[c0 + j];
        if (cu[j] != o0) atomicAdd(P.cap[DUP] + off + j, cu[j] - o0);
      }
    } else {
      *(int4*)(P.cap[DUP] + off) = make_int4(cu[0], cu[1], cu[2], cu[3]);
    }
    if (r == 31) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int o0 = S.cd_bot[c0 + j];
        if (cd[j] != o0) atomicAdd(P.cap[DDOWN] + off + j, cd[j] - o0);
      }
    } else {
      *(int4*)(P.cap[DDOWN] + off) = make_int4(cd[0], cd[1], cd[2], cd[3]);
    }
    if (q == 0) {
      const int cl0 = S.cl_left[r];
      if (cl[0] != cl0) atomicAdd(P.cap[DLEFT] + off, cl[0] - cl0);
      P.cap[DLEFT][off + 1] = cl[1]; P.cap[DLEFT][off + 2] = cl[2]; P.cap[DLEFT][off + 3] = cl[3];
    } else {
      *(int4*)(P.cap[DLEFT] + off) = make_int4(cl[0], cl[1], cl[2], cl[3]);
    }
    if (q == 7) {
      const int cr0 = S.cr_right[r];
      if (cr[3] != cr0) atomicAdd(P.cap[DRIGHT] + off + 3, cr[3] - cr0);
      P.cap[DRIGHT][off] = cr[0]; P.cap[DRIGHT][off + 1] = cr[1]; P.cap[DRIGHT][off + 2] = cr[2];
    } else {
      *(int4*)(P.cap[DRIGHT] + off) = make_int4(cr[0], cr[1], cr[2], cr[3]);
    }
    // deliver cross-tile flow: excess of the neighbour pixel and its reverse residual
    int sent_u = 0, sent_d = 0, sent_l = 0, sent_r = 0;
    if (r == 0 && nb.x >= 0) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int x = S.xu[c0 + j];
        if (x) {
          const long long o = (long long)nb.x * GC_TILE_PX + 31 * GC_TILE + c0 + j;
          atomicAdd(P.exc + o, x); atomicAdd(P.cap[DDOWN] + o, x); sent_u = 1;
        }
      }
    }
    if (r == 31 && nb.y >= 0) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int x = S.xd[c0 + j];
        if (x) {
          const long long o = (long long)nb.y * GC_TILE_PX + c0 + j;
          atomicAdd(P.exc + o, x); atomicAdd(P.cap[DUP] + o, x); sent_d = 1;
        }
      }
    }
    if (q == 0 && nb.z >= 0) {
      const int x = S.xl[r];
      if (x) {
        const long long o = (long long)nb.z * GC_TILE_PX + r * GC_TILE + 31;
        atomicAdd(P.exc + o, x); atomicAdd(P.cap[DRIGHT] + o, x); sent_l = 1;
      }
    }
    if (q == 7 && nb.w >= 0) {
      const int x = S.xr[r];
      if (x) {
        const long long o = (long long)nb.w * GC_TILE_PX + r * GC_TILE;
        atomicAdd(P.exc + o, x); atomicAdd(P.cap[DLEFT] + o, x); sent_r = 1;
      }
    }
    int act = 0, act_int = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = c0 + j;
      const int a = e[j] > 0 && h[j] < GC_HINF;
      act |= a;
      act_int |= a && !erow && c > 0 && c < 31;
    }
    const int sent = (sent_u ? 1 : 0) | (sent_d ? 2 : 0) | (sent_l ? 4 : 0) | (sent_r ? 8 : 0);
    if (sent) atomicOr(&s_sent, sent);
    // the block-wide reductions also order every read of this buffer before its reuse
    const int any_act = __syncthreads_or(act);
    act_int = __syncthreads_or(act_int);
    // log the tile's bookkeeping; a full log is settled now (the barrier makes the entries
    // visible; the next write of an entry follows several more barriers)
    if (tid == 0) {
      s_logt[nlog] = t;
      s_lognb[nlog] = nb;
      s_logf[nlog] = (s_sent & 15) | (any_act ? 16 : 0) | (act_int ? 32 : 0);
    }
    if (++nlog == DIS_LOG) { __syncthreads(); flush_log(nlog); nlog = 0; }
  }
  __syncthreads();
  flush_log(nlog);
  if (failed) {
    // a bulk copy did not complete in time: record it, let our copy drain, stop
    if (tid == 0) {
      atomicExch(&P.ctl[CTL_ERR], 3);
      if (pending) mbar_wait(&mbar, phase, 5 * GC_COPY_WAIT_NS);
    }
    __syncthreads();
  }
  // last CTA: the queue just read is consumed; the next launch reads the other one
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    const int d = atomicAdd(&P.ctl[CTL_DDONE], 1);
    if (d == (int)gridDim.x - 1) {
      P.qcount[cur] = 0;
      P.ctl[CTL_PULSE] = P.ctl[CTL_PULSE] + 1;
      P.ctl[CTL_DDONE] = 0;
      __threadfence();
    }
  }
}

// ------------------------------------------------------------------------------------
// Edge relabel + active-tile list.
// ------------------------------------------------------------------------------------
constexpr int EB_THREADS = 512;
constexpr int EB_WARPS = EB_THREADS / 32;
constexpr int EB_TILES = 64;                 // tiles per CTA (4 per warp)

// Relabels up to four tile-edge pixels of one lane (Jacobi: neighbour heights are read
// as they are, a concurrent update only makes them larger, which keeps the labelling
// valid).  Returns whether one of them is active afterwards.
__device__ __forceinline__ int edge_relabel_lane(const PoolView& P, int t, int4 nb, int lane) {
  int rr[4] = {0, 31, lane, lane}, cc[4] = {lane, lane, 0, 31};
  const bool use[4] = {true, true, lane > 0 && lane < 31, lane > 0 && lane < 31};
  const long long base = (long long)t * GC_TILE_PX;
  int e[4], h[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const long long o = base + rr[k] * GC_TILE + cc[k];
    e[k] = use[k] ? P.exc[o] : 0;
    h[k] = use[k] ? P.hgt[o] : GC_HINF;
  }
  int act = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (!(e[k] > 0 && h[k] < GC_HINF)) continue;
    const int r = rr[k], c = cc[k];
    const long long o = base + r * GC_TILE + c;
    const int cu = P.cap[DUP][o], cd = P.cap[DDOWN][o], cl = P.cap[DLEFT][o], cr = P.cap[DRIGHT][o];
    int hu = GC_HINF, hd = GC_HINF, hl = GC_HINF, hr = GC_HINF;
    if (r > 0) hu = P.hgt[o - GC_TILE]; else if (nb.x >= 0) hu = P.hgt[(long long)nb.x * GC_TILE_PX + 31 * GC_TILE + c];
    if (r < 31) hd = P.hgt[o + GC_TILE]; else if (nb.y >= 0) hd = P.hgt[(long long)nb.y * GC_TILE_PX + c];
    if (c > 0) hl = P.hgt[o - 1]; else if (nb.z >= 0) hl = P.hgt[(long long)nb.z * GC_TILE_PX + r * GC_TILE + 31];
    if (c < 31) hr = P.hgt[o + 1]; else if (nb.w >= 0) hr = P.hgt[(long long)nb.w * GC_TILE_PX + r * GC_TILE];
    const int hh = h[k];
    const bool adm = (cu > 0 && hh == hu + 1) || (cd > 0 && hh == hd + 1) || (cl > 0 && hh == hl + 1) ||
                     (cr > 0 && hh == hr + 1);
    if (adm) { act = 1; continue; }
    int m = GC_HINF;
    if (cu > 0) m = imin(m, hu + 1);
    if (cd > 0) m = imin(m, hd + 1);
    if (cl > 0) m = imin(m, hl + 1);
    if (cr > 0) m = imin(m, hr + 1);
    m = imin(m, GC_HINF);
    if (m != hh) P.hgt[o] = m;
    act |= m < GC_HINF;
  }
  return act;
}

// Edge relabel + active-tile list (one launch).  A CTA owns EB_TILES consecutive tiles by
// arrival ticket; each warp takes 4 of them and relabels only the touched ones (one warp
// per tile, 4 edge pixels per lane).  A tile is active when an interior pixel was active
// after its discharge or a tile-edge pixel is active after this relabel.  The active tiles
// are compacted in tile order with a warp-parallel decoupled look-back.
__global__ void __launch_bounds__(EB_THREADS)
k_edge_relabel_build(PoolView P, int32_t* list, int32_t* count, ScanState st) {
  __shared__ int32_t flag[EB_TILES];
  __shared__ int32_t s_chunk;
  __shared__ uint32_t s_tag;
  if (threadIdx.x == 0) {
    s_chunk = atomicAdd(st.ticket, 1);
    s_tag = *((volatile uint32_t*)st.seq);
  }
  __syncthreads();
  const int chunk = s_chunk;
  const int nchunks = (P.nt + EB_TILES - 1) / EB_TILES;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int PER_WARP = EB_TILES / EB_WARPS;
  const int t0 = chunk * EB_TILES + warp * PER_WARP;
  int touched = 0;
  if (lane < PER_WARP && t0 + lane < P.nt) {
    touched = P.touched[t0 + lane];
    P.inq[0][t0 + lane] = 0;  // the worklists are replaced by the rebuilt list
    P.inq[1][t0 + lane] = 0;
  }
  unsigned todo = __ballot_sync(0xffffffffu, touched != 0);
  if (lane < PER_WARP) flag[warp * PER_WARP + lane] = 0;
  __syncwarp();
  while (todo) {
    const int k = __ffs(todo) - 1;
    todo &= todo - 1;
    const int t = t0 + k;
    const int4 nb = P.nbr[t];
    const int a = edge_relabel_lane(P, t, nb, lane);
    const int active = __any_sync(0xffffffffu, a) | P.act_int[t];
    if (lane == 0) {
      flag[warp * PER_WARP + k] = active;
      P.touched[t] = 0;
      if (P.ktiles) atomicAdd(&P.ktiles[K_EDGE_BUILD], 1ull);
    }
  }
  __syncthreads();
  if (warp == 0) {
    const int v0 = flag[2 * lane], v1 = flag[2 * lane + 1];   // two flags per lane
    const int v = v0 + v1;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    const int agg = __shfl_sync(0xffffffffu, x, 31);
    const int excl = lookback_exclusive_warp(st, s_tag, chunk, agg);
    int pos = excl + x - v;
    const int tb = chunk * EB_TILES + 2 * lane;
    if ((unsigned)pos + (unsigned)(v0 + v1) <= (unsigned)P.nt) {
      if (v0) list[pos++] = tb;
      if (v1) list[pos] = tb + 1;
    } else if (v) {
      atomicExch(st.err, 2);   // only after a look-back that gave up
    }
    if (chunk == nchunks - 1 && lane == 0) *count = excl + agg;
    if (lane == 0) scan_finish(st, nchunks);
  }
}

// ------------------------------------------------------------------------------------
// Global relabel: bit-parallel BFS per tile, one warp per tile, lane = row.
// ------------------------------------------------------------------------------------

__device__ __forceinline__ int warp_min(int v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = imin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Multi-source BFS inside a tile on the row masks, level by level (a bucketed BFS with unit
// steps): level 0 holds the sink pixels; a tile-edge pixel with a residual edge into the
// neighbour tile is also seeded at (neighbour height + 1).  Lane c holds the seeds of column c
// in the top row (`top`) and the bottom row (`bot`); lane r holds the seeds of row r at column
// 0 (`sl`) and 31 (`sr`); GC_HINF where there is none.  Level L visits the unvisited pixels
// that are seeds of value L or neighbours, over residual edges, of level L - 1; an empty level
// jumps to the smallest unvisited seed.  Lane r writes the distances of row r into `row`
// (GC_HINF where unreached) and gets the mask of reached pixels.
__device__ __forceinline__ uint32_t tile_bfs_seeded(int* row, uint32_t sink, uint32_t canU,
                                                    uint32_t canD, uint32_t canL, uint32_t canR,
                                                    int lane, int top, int bot, int sl, int sr) {
  const unsigned FULL = 0xffffffffu;
#pragma unroll
  for (int c = 0; c < 32; ++c) row[c] = GC_HINF;
  uint32_t vis = 0, F = 0;
  int L = __any_sync(FULL, sink != 0) ? 0 : warp_min(imin(imin(top, bot), imin(sl, sr)));
  // every step visits a pixel or jumps to an unvisited seed: at most 1024 + 128 steps
  for (int step = 0; step < 2 * GC_TILE_PX && L < GC_HINF; ++step) {
    uint32_t Fu = __shfl_up_sync(FULL, F, 1);
    uint32_t Fd = __shfl_down_sync(FULL, F, 1);
    if (lane == 0) Fu = 0;
    if (lane == 31) Fd = 0;
    const uint32_t bt = __ballot_sync(FULL, top == L);
    const uint32_t bb = __ballot_sync(FULL, bot == L);
    uint32_t S = (L == 0 ? sink : 0u) | (sl == L ? 1u : 0u) | (sr == L ? 0x80000000u : 0u);
    if (lane == 0) S |= bt;
    if (lane == 31) S |= bb;
    const uint32_t N = (((F >> 1) & canR) | ((F << 1) & canL) | (Fu & canU) | (Fd & canD) | S) & ~vis;
    vis |= N;
    F = N;
    for (uint32_t b = N; b; b &= b - 1) row[__ffs(b) - 1] = L;
    if (__any_sync(FULL, F != 0)) {
      ++L;
      continue;
    }
    // the frontier is empty: the next level that still has an unvisited seed
    const uint32_t v0 = __shfl_sync(FULL, vis, 0), v31 = __shfl_sync(FULL, vis, 31);
    int cand = GC_HINF;
    if (top > L && !((v0 >> lane) & 1u)) cand = imin(cand, top);
    if (bot > L && !((v31 >> lane) & 1u)) cand = imin(cand, bot);
    if (sl > L && !(vis & 1u)) cand = imin(cand, sl);
    if (sr > L && !(vis >> 31)) cand = imin(cand, sr);
    L = warp_min(cand);
  }
  return vis;
}

// Frontier rounds.  The first round of a relabel or flood processes the solve's selected
// tiles (grid-stride over the selection); round r > 0 processes the list fq[r & 1] built by
// round r - 1.  A tile whose boundary
// values changed queues its neighbours in fq[(r + 1) & 1], deduplicated by mark[(r + 1) & 1];
// the round that processes a tile clears its mark.  Only the CTAs the list needs take part
// (at least one, so every launched round is finalised), and the last of them consumes the
// list, advances the round number (device memory, ctl[CTL_RND]) and, inside a CUDA graph,
// sets the WHILE condition: another round runs only when the next list is not empty.
__device__ __forceinline__ int frontier_round_number(const PoolView& P, int first) {
  return first ? 0 : *((volatile int32_t*)&P.ctl[CTL_RND]);
}

// Work of this round: *count tiles (the selected tiles for a first round, the frontier list
// otherwise), *nranges the selection's ranges, and the number of CTAs that take part; CTAs
// beyond it return at once.  Called by every thread of the CTA.
__device__ __forceinline__ void frontier_work(const PoolView& P, int first, int in, int per_cta,
                                              int* count, int* participants, int* nranges) {
  __shared__ int s_n, s_nr;
  if (threadIdx.x == 0) {
    int n = first ? *((volatile int32_t*)&P.nsel[1]) : *((volatile int32_t*)&P.fcount[in]);
    int nr = *((volatile int32_t*)&P.nsel[0]);
    if (n < 0 || n > P.nt) {   // self-check: a list holds each tile at most once
      record_bad(P, 6, n);
      n = 0;
    }
    if (nr < 0 || nr > P.nimg) {   // self-check: one range per image at most
      record_bad(P, 9, nr);
      n = nr = 0;
    }
    s_n = n;
    s_nr = nr;
  }
  __syncthreads();
  const int n = s_n;
  *count = n;
  *nranges = s_nr;
  const int need = (n + per_cta - 1) / per_cta;
  *participants = need < 1 ? 1 : (need < (int)gridDim.x ? need : (int)gridDim.x);
}

// Queue tile t for the next round (once).  Within a round the next round's marks only go
// from 0 to 1, so a set mark read with a plain load needs no atomic.
__device__ __forceinline__ void frontier_push(const PoolView& P, int out, int t) {
  if (*((volatile int32_t*)&P.mark[out][t]) != 0) return;
  if (atomicExch(&P.mark[out][t], 1) == 0) {
    const int pos = atomicAdd(&P.fcount[out], 1);
    if (pos < P.nt) P.fq[out][pos] = t;   // the mark deduplicates, so pos < nt always holds
    else record_bad(P, 5, pos);
  }
}

__device__ __forceinline__ void frontier_round_end(const PoolView& P, int first, int in,
                                                   int total_slot, int participants,
                                                   cudaGraphConditionalHandle h) {
  __syncthreads();
  if (threadIdx.x != 0) return;
  __threadfence();
  const int d = atomicAdd(&P.ctl[CTL_DONE], 1);
  if (d != participants - 1) return;
  __threadfence();
  volatile int32_t* ctl = P.ctl;
  const int out = in ^ 1;
  P.rcnt[in] = 0;
  const int next = *((volatile int32_t*)&P.fcount[out]);
  P.fcount[in] = 0;   // this round's list is consumed
  ctl[CTL_LASTCNT] = next;
  ctl[CTL_RND] = first ? 1 : ctl[CTL_RND] + 1;
  const int rounds = first ? 1 : ctl[CTL_ROUNDS] + 1;
  ctl[CTL_ROUNDS] = rounds;
  ctl[total_slot] = ctl[total_slot] + 1;
  ctl[CTL_DONE] = 0;
  bool more = next > 0 && ctl[CTL_ERR] < 3;   // a copy or self-check error ends the loop
  if (more && rounds >= ctl[CTL_MAXROUNDS]) {
    ctl[CTL_ERR] = 1;
    more = false;
  }
  __threadfence();
  if (h) cudaGraphSetConditional(h, more ? 1u : 0u);
}

// Solve prologue: reset the control words and the image stamps; the images of the
// selection take their mode for this solve and restart their flow sums (the others keep
// their results).  One CTA.
__global__ void k_ctl_begin(PoolView P, int max_rounds, int max_cycles, ImageAcc* acc) {
  trace_mark(P, TR_BEGIN);
  for (int i = threadIdx.x; i < CTL_N; i += blockDim.x) P.ctl[i] = 0;
  for (int i = threadIdx.x; i < P.nimg; i += blockDim.x) {
    P.img_live[i] = 0;
    P.img_hit[i] = 0;
    P.img_mode[i] = 0;
  }
  __syncthreads();
  const int nr = *((volatile int32_t*)&P.nsel[0]);
  for (int k = threadIdx.x; k < nr && k < P.nimg; k += blockDim.x) {
    const int img = P.sel[k].w;
    if ((unsigned)img >= (unsigned)P.nimg) continue;
    P.img_mode[img] = P.sel_mode[k];
    acc[img].sumpos_e = 0;   // the floods of this solve accumulate it
  }
  if (threadIdx.x == 0) {
    P.ctl[CTL_MAXROUNDS] = max_rounds;
    P.ctl[CTL_MAXCYCLES] = max_cycles;
    P.rcnt[0] = 0;
    P.rcnt[1] = 0;
    P.fcount[0] = 0;
    P.fcount[1] = 0;
  }
}

// The solve's results written straight into pinned host memory by the kernel that ends a
// graph solve, so the graph needs no copy node after its loops: the control words, then the
// sums of the solve's images at their places in the host mirror (the other images' sums have
// not changed since their own solves).  Threads 0 .. nthreads-1 take part.  The host reads
// the block only after synchronising with the solve's stream, which makes every write of the
// finished kernels visible to it, so no system-scope fence is needed here (one cost about
// 1 % of a 2048^2 step: the labels that follow waited for it).
__device__ __forceinline__ void publish_results(const PoolView& P, const ImageAcc* acc,
                                                int nthreads) {
  if (!P.host_out) return;
  constexpr int AW = (int)(sizeof(ImageAcc) / sizeof(int32_t));
  int nr = *((volatile int32_t*)&P.nsel[0]);
  nr = nr < 0 ? 0 : nr > P.nimg ? P.nimg : nr;
  const volatile int32_t* c = P.ctl;
  const volatile int32_t* a = reinterpret_cast<const volatile int32_t*>(acc);
  for (int i = threadIdx.x; i < CTL_N + AW * nr; i += nthreads) {
    if (i < CTL_N) {
      P.host_out[i] = c[i];
    } else {
      const int img = P.sel[(i - CTL_N) / AW].w, w = (i - CTL_N) % AW;
      if ((unsigned)img < (unsigned)P.nimg) P.host_out[CTL_N + AW * img + w] = a[AW * img + w];
    }
  }
}

// The active-tile list after a global relabel, in one launch: a single-pass scan (chunks by
// arrival ticket, decoupled look-back) of the activity flags of the selected tiles writes the
// ids of the active tiles in order and stamps their images live for the next cycle (stamp =
// cycles + 1 + bump); the last CTA to finish closes the scan and applies the cycle check:
// another cycle runs while tiles are active and the cycle cap is not reached (`count_cycle`
// counts this check as a finished cycle).  Replaces a compaction and a separate stamping
// launch.  filter: 1 only tiles of the images a flood check kept (img_live == the cycle
// stamp; a solved image keeps the activity flags of its last relabel), 2 those and the tiles
// of freshly uploaded images (the first list of a solve).
//
// The grid is a fixed number of CTAs (a few per SM) that take chunk tickets in a loop until
// the selection's chunks run out, so a pool of millions of tiles costs no more launch work
// than one image, and a 2048^2 image (4096 tiles) spreads over four CTAs.  Every ticket
// holder is already running, so a look-back only ever waits for a running CTA.  The image
// of each item comes from the selection (one range per image), and an image's live stamp,
// flood sum and sink-reached stamp are written once per warp that holds one of its active
// tiles rather than once per tile: thousands of stores to one address serialise in L2.
constexpr int ACT_THREADS = 256;
constexpr int ACT_ITEMS = 4;
constexpr int ACT_CHUNK = ACT_THREADS * ACT_ITEMS;

__device__ __forceinline__ void stamp_image(const PoolView& P, ImageAcc* acc, int img, int stamp) {
  P.img_live[img] = stamp;
  // the image's next flood starts afresh: its sum and its sink-reached stamp (the first
  // cycle of a warm solve reuses the stamp of the flood before it)
  acc[img].sumpos_e = 0;
  P.img_hit[img] = 0;
}

__global__ void __launch_bounds__(ACT_THREADS)
k_active_list(PoolView P, ScanState st, int32_t* list, int32_t* count, int bump,
              int count_cycle, int filter, cudaGraphConditionalHandle h, ImageAcc* acc) {
  trace_mark(P, TR_ACTIVE_LIST);
  __shared__ int32_t sm[32];
  __shared__ int32_t s_chunk, s_excl, s_cur, s_n, s_nr;
  __shared__ uint32_t s_tag;
  if (threadIdx.x == 0) {
    s_chunk = atomicAdd(st.ticket, 1);
    s_tag = *((volatile uint32_t*)st.seq);
    s_cur = *((volatile int32_t*)&P.ctl[CTL_CYCLES]) + 1;
    int n = *((volatile int32_t*)&P.nsel[1]), nr = *((volatile int32_t*)&P.nsel[0]);
    if (n < 0 || n > P.nt || nr < 0 || nr > P.nimg) {   // self-check
      record_bad(P, 9, n);
      n = nr = 0;
    }
    s_n = n;
    s_nr = nr;
  }
  __syncthreads();
  const int cur = s_cur, stamp = cur + bump;
  const int n = s_n;
  const int nchunks = (n + ACT_CHUNK - 1) / ACT_CHUNK;
  const int lane = threadIdx.x & 31;
  for (int chunk = s_chunk; chunk < nchunks;) {
    const int base = chunk * ACT_CHUNK + threadIdx.x * ACT_ITEMS;
    SelCursor cursor(P, s_nr, base < n ? base : 0);
    int32_t v[ACT_ITEMS], tl[ACT_ITEMS], im[ACT_ITEMS];
#pragma unroll
    for (int k = 0; k < ACT_ITEMS; ++k) {
      tl[k] = -1;
      im[k] = -1;
      if (base + k < n) {
        tl[k] = cursor.tile(base + k);
        im[k] = cursor.image();
      }
      v[k] = 0;
      if ((unsigned)tl[k] < (unsigned)P.nt && (unsigned)im[k] < (unsigned)P.nimg)
        v[k] = P.tact[tl[k]] != 0;
      else if (tl[k] >= 0)
        record_bad(P, 4, (unsigned)im[k] < (unsigned)P.nimg ? tl[k] : im[k]);
    }
    if (filter) {
#pragma unroll
      for (int k = 0; k < ACT_ITEMS; ++k) {
        if (!v[k]) continue;
        const int il = *((volatile int32_t*)&P.img_live[im[k]]);
        v[k] = il == cur || il == stamp || (filter == 2 && P.img_mode[im[k]] == 1);
      }
    }
    int32_t tsum = 0, first = -1;
#pragma unroll
    for (int k = ACT_ITEMS - 1; k >= 0; --k) {
      tsum += v[k];
      if (v[k]) first = im[k];
    }
    int32_t agg;
    const int32_t tex = block_exclusive_scan(tsum, sm, &agg);
    if (threadIdx.x < 32) {
      const int32_t ex = lookback_exclusive_warp(st, s_tag, chunk, agg);
      if (threadIdx.x == 0) s_excl = ex;
    }
    __syncthreads();
    // one lane per distinct first image in the warp stamps it; the rare later images of a
    // thread (its items straddle two ranges) are stamped by that thread
    const unsigned peers = __match_any_sync(0xffffffffu, first);
    if (first >= 0 && __ffs(peers) - 1 == lane) stamp_image(P, acc, first, stamp);
    int32_t run = s_excl + tex;
    int last = first;
#pragma unroll
    for (int k = 0; k < ACT_ITEMS; ++k) {
      if (v[k]) {
        if ((unsigned)run < (unsigned)P.nt) list[run] = tl[k];
        else atomicExch(st.err, 2);   // only after a look-back that gave up
        if (im[k] != last) {
          stamp_image(P, acc, im[k], stamp);
          last = im[k];
        }
        ++run;
      }
    }
    if (chunk == nchunks - 1 && threadIdx.x == 0) *count = s_excl + agg;
    // the first tickets are 0 .. gridDim.x - 1: when they cover every chunk, none is left
    if ((int)gridDim.x >= nchunks) break;
    __syncthreads();   // every thread has read s_chunk and s_excl
    if (threadIdx.x == 0) s_chunk = atomicAdd(st.ticket, 1);
    __syncthreads();
    chunk = s_chunk;
  }
  if (threadIdx.x != 0) return;
  __threadfence();
  if (atomicAdd(st.done, 1) != (int)gridDim.x - 1) return;
  // last CTA: close the scan (tickets, tag) and apply the cycle check
  __threadfence();
  *st.ticket = 0;
  *st.done = 0;
  uint32_t sq = *st.seq + 1;
  if ((sq & 0x3fffffffu) == 0) sq = 1;
  *st.seq = sq;
  volatile int32_t* ctl = P.ctl;
  if (nchunks == 0) *count = 0;
  const int nact = *((volatile int32_t*)count);
  ctl[CTL_PULSE] = 0;   // the list sits in queue[0]
  ctl[CTL_DDONE] = 0;
  P.qcount[1] = 0;
  const int cycles = ctl[CTL_CYCLES] + (count_cycle ? 1 : 0);
  ctl[CTL_CYCLES] = cycles;
  ctl[CTL_NACT] = ctl[CTL_NACT] + 1;
  // a look-back that gave up (here or in an earlier list of this solve) reaches the host
  // with the control words
  ctl[CTL_SCANERR] = ctl[CTL_SCANERR] | *((volatile int32_t*)st.err);
  bool more = nact > 0 && ctl[CTL_ERR] < 3;
  if (more && cycles >= ctl[CTL_MAXCYCLES]) {
    ctl[CTL_ERR] = 2;
    more = false;
  }
  __threadfence();
  if (h) cudaGraphSetConditional(h, more ? 1u : 0u);
  if (h && !more) publish_results(P, acc, 1);   // the graph solve ends here
}

// k_ctl_begin and the first active-tile list of a solve of fresh images only (no flood
// precedes that list), in one CTA for pools of at most BL_MAX tiles: the reset, a barrier,
// then the list with a block-wide scan instead of a look-back, and the list's cycle check.
// One launch instead of two, and none of the multi-CTA list's tickets and waits.
constexpr int BL_THREADS = 1024;
constexpr int BL_ITEMS = 4;
constexpr int BL_MAX = BL_THREADS * BL_ITEMS;

__global__ void __launch_bounds__(BL_THREADS)
k_begin_list(PoolView P, int max_rounds, int max_cycles, ImageAcc* acc, int32_t* list,
             int32_t* count, cudaGraphConditionalHandle h) {
  trace_mark(P, TR_BEGIN);
  __shared__ int32_t sm[32];
  const int tid = threadIdx.x, lane = tid & 31;
  for (int i = tid; i < CTL_N; i += BL_THREADS) P.ctl[i] = 0;
  for (int i = tid; i < P.nimg; i += BL_THREADS) {
    P.img_live[i] = 0;
    P.img_hit[i] = 0;
    P.img_mode[i] = 0;
  }
  __syncthreads();
  int nr = *((volatile int32_t*)&P.nsel[0]), n = *((volatile int32_t*)&P.nsel[1]);
  if (n < 0 || n > P.nt || n > BL_MAX || nr < 0 || nr > P.nimg) {   // self-check
    if (tid == 0) record_bad(P, 9, n);
    n = nr = 0;
  }
  for (int k = tid; k < nr; k += BL_THREADS) {
    const int img = P.sel[k].w;
    if ((unsigned)img >= (unsigned)P.nimg) continue;
    P.img_mode[img] = P.sel_mode[k];
    acc[img].sumpos_e = 0;   // the floods of this solve accumulate it
  }
  if (tid == 0) {
    P.ctl[CTL_MAXROUNDS] = max_rounds;
    P.ctl[CTL_MAXCYCLES] = max_cycles;
    P.rcnt[0] = 0;
    P.rcnt[1] = 0;
    P.fcount[0] = 0;
    P.fcount[1] = 0;
    trace_record(P, TR_ACTIVE_LIST);
  }
  __syncthreads();   // the modes above are visible to every thread
  // the list: active tiles of the fresh images (cycle stamp 1)
  const int stamp = 1;
  const int base = tid * BL_ITEMS;
  SelCursor cursor(P, nr, base < n ? base : 0);
  int32_t v[BL_ITEMS], tl[BL_ITEMS], im[BL_ITEMS];
#pragma unroll
  for (int k = 0; k < BL_ITEMS; ++k) {
    tl[k] = -1;
    im[k] = -1;
    if (base + k < n) {
      tl[k] = cursor.tile(base + k);
      im[k] = cursor.image();
    }
    v[k] = 0;
    if ((unsigned)tl[k] < (unsigned)P.nt && (unsigned)im[k] < (unsigned)P.nimg)
      v[k] = P.tact[tl[k]] != 0 && P.img_mode[im[k]] == 1;
    else if (tl[k] >= 0)
      record_bad(P, 4, (unsigned)im[k] < (unsigned)P.nimg ? tl[k] : im[k]);
  }
  int32_t tsum = 0, first = -1;
#pragma unroll
  for (int k = BL_ITEMS - 1; k >= 0; --k) {
    tsum += v[k];
    if (v[k]) first = im[k];
  }
  int32_t agg;
  int32_t run = block_exclusive_scan(tsum, sm, &agg);
  const unsigned peers = __match_any_sync(0xffffffffu, first);
  if (first >= 0 && __ffs(peers) - 1 == lane) stamp_image(P, acc, first, stamp);
  int last = first;
#pragma unroll
  for (int k = 0; k < BL_ITEMS; ++k) {
    if (v[k]) {
      if ((unsigned)run < (unsigned)P.nt) list[run] = tl[k];
      if (im[k] != last) {
        stamp_image(P, acc, im[k], stamp);
        last = im[k];
      }
      ++run;
    }
  }
  if (tid != 0) return;
  // the cycle check of k_active_list (count_cycle 0: no cycle has run yet)
  *count = agg;
  volatile int32_t* ctl = P.ctl;
  ctl[CTL_PULSE] = 0;   // the list sits in queue[0]
  ctl[CTL_DDONE] = 0;
  P.qcount[1] = 0;
  ctl[CTL_NACT] = 1;
  bool more = agg > 0 && ctl[CTL_ERR] < 3;
  if (more && ctl[CTL_MAXCYCLES] <= 0) {
    ctl[CTL_ERR] = 2;
    more = false;
  }
  __threadfence();
  if (h) cudaGraphSetConditional(h, more ? 1u : 0u);
  if (h && !more) publish_results(P, acc, 1);   // the graph solve ends here
}

// After the active-tile compaction: another cycle runs while tiles are active and the cycle
// cap is not reached (`count_cycle` counts this check as a finished cycle).
__global__ void k_ctl_cycle(PoolView P, const int32_t* count, int count_cycle,
                            cudaGraphConditionalHandle h) {
  if (threadIdx.x != 0) return;
  volatile int32_t* ctl = P.ctl;
  ctl[CTL_PULSE] = 0;   // the compacted list sits in queue[0]
  ctl[CTL_DDONE] = 0;
  P.qcount[1] = 0;
  int cycles = ctl[CTL_CYCLES] + (count_cycle ? 1 : 0);
  ctl[CTL_CYCLES] = cycles;
  bool more = *((volatile const int32_t*)count) > 0 && ctl[CTL_ERR] < 3;
  if (more && cycles >= ctl[CTL_MAXCYCLES]) {
    ctl[CTL_ERR] = 2;
    more = false;
  }
  __threadfence();
  if (h) cudaGraphSetConditional(h, more ? 1u : 0u);
}

__global__ void __launch_bounds__(WARPS_PER_CTA * 32)
k_bfs_round(PoolView P, int first, cudaGraphConditionalHandle h) {
  trace_mark(P, first ? TR_BFS_FIRST : TR_BFS);
  __shared__ int32_t tr[WARPS_PER_CTA][32 * 33];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int in = frontier_round_number(P, first) & 1, out = in ^ 1;
  int32_t* const markin = P.mark[in];
  int32_t* T = tr[warp];
  int done = 0;
  // first == 2: a global relabel inside the solve loop skips images whose cut was final at
  // the previous check (no active tile); their state no longer changes
  const int live = first == 2 ? *((volatile int32_t*)&P.ctl[CTL_CYCLES]) + 1 : 0;
  int n, parts, nr;
  frontier_work(P, first, in, WARPS_PER_CTA, &n, &parts, &nr);
  if ((int)blockIdx.x >= parts) return;
  const int i0 = blockIdx.x * WARPS_PER_CTA + warp;
  SelCursor cursor(P, first ? nr : 0, i0);
  for (int i = i0; i < n; i += parts * WARPS_PER_CTA) {
    const int t = first ? cursor.tile(i) : P.fq[in][i];
    if (!first) {
      if (lane == 0) markin[t] = 0;
    } else {
      if (first == 2) {
        const int img = P.img_of[t];
        if ((unsigned)img >= (unsigned)P.nimg) {   // self-check
          if (lane == 0) record_bad(P, 4, img);
          continue;
        }
        if (P.img_live[img] != live) continue;
      }
      if (lane == 0) {
        P.inq[0][t] = 0;  // the worklists are rebuilt from the relabelled state
        P.inq[1][t] = 0;
      }
    }
    ++done;
    const int4 nb = P.nbr[t];
    const long long base = (long long)t * GC_TILE_PX;
    // the masks are current: the flood that precedes every global relabel of a solve (or
    // k_masks, before gc_start_bfs) rebuilt every tile that changed since they were written
    const uint32_t* mc = P.mcan + (long long)t * 128;
    const uint32_t canU = mc[lane], canD = mc[32 + lane], canL = mc[64 + lane], canR = mc[96 + lane];
    const uint32_t sink = P.msink[(long long)t * 32 + lane];
    // seeds from the neighbour tiles' heights (frontier rounds only): an edge pixel with a
    // residual edge into the neighbour starts at the neighbour's height + 1
    int top = GC_HINF, bot = GC_HINF, sl = GC_HINF, sr = GC_HINF;
    if (!first) {
      const uint32_t cu0 = __shfl_sync(0xffffffffu, canU, 0);
      const uint32_t cd31 = __shfl_sync(0xffffffffu, canD, 31);
      const int vu = nb.x >= 0 ? P.hgt[(long long)nb.x * GC_TILE_PX + 31 * GC_TILE + lane] : GC_HINF;
      const int vd = nb.y >= 0 ? P.hgt[(long long)nb.y * GC_TILE_PX + lane] : GC_HINF;
      const int vl = nb.z >= 0 ? P.hgt[(long long)nb.z * GC_TILE_PX + lane * GC_TILE + 31] : GC_HINF;
      const int vr = nb.w >= 0 ? P.hgt[(long long)nb.w * GC_TILE_PX + lane * GC_TILE] : GC_HINF;
      if (((cu0 >> lane) & 1u) && vu < GC_HINF) top = vu + 1;
      if (((cd31 >> lane) & 1u) && vd < GC_HINF) bot = vd + 1;
      if ((canL & 1u) && vl < GC_HINF) sl = vl + 1;
      if ((canR >> 31) && vr < GC_HINF) sr = vr + 1;
    }
    const uint32_t fin = tile_bfs_seeded(T + lane * 33, sink, canU, canD, canL, canR, lane, top,
                                         bot, sl, sr);
    __syncwarp();
    int chU = 0, chD = 0, chL = 0, chR = 0;
    for (int rr = 0; rr < 32; ++rr) {
      const int nv = T[rr * 33 + lane];
      int* p = P.hgt + base + rr * GC_TILE + lane;
      if (first) {
        *p = nv;
        const int fv = nv < GC_HINF;
        chU |= (rr == 0) & fv; chD |= (rr == 31) & fv; chL |= (lane == 0) & fv; chR |= (lane == 31) & fv;
      } else {
        const int ov = *p;
        if (nv != ov) *p = nv;
        const int dec = nv < ov;
        chU |= (rr == 0) & dec; chD |= (rr == 31) & dec; chL |= (lane == 0) & dec; chR |= (lane == 31) & dec;
      }
    }
    __syncwarp();
    chU = __any_sync(0xffffffffu, chU); chD = __any_sync(0xffffffffu, chD);
    chL = __any_sync(0xffffffffu, chL); chR = __any_sync(0xffffffffu, chR);
    const uint32_t pos = P.mexc[(long long)t * 32 + lane];
    const int act = __any_sync(0xffffffffu, (pos & fin) != 0);
    if (lane == 0) P.tact[t] = act;
    // the neighbours to queue, one lane each (their atomics run in parallel)
    if (lane < 4) {
      const int go = lane == 0 ? chU : lane == 1 ? chD : lane == 2 ? chL : chR;
      const int nt = lane == 0 ? nb.x : lane == 1 ? nb.y : lane == 2 ? nb.z : nb.w;
      if (go && nt >= 0) frontier_push(P, out, nt);
    }
  }
  if (lane == 0 && done) {
    atomicAdd(&P.rcnt[in], done);
    if (P.ktiles) atomicAdd(&P.ktiles[first ? K_BFS_FIRST : K_BFS], (unsigned long long)done);
  }
  frontier_round_end(P, first, in, CTL_BFS_TOTAL, parts, h);
}

// After a flood: an image whose flood reached no sink pixel is solved (its flood is the
// canonical cut, its sums are final) and leaves the live set; the others go on to a global
// relabel.  all != 0: the images that continue from a previous flow (img_mode == 2; the
// first check of a solve); else the images live in this cycle.  Sets the condition of the
// IF node around the relabel (hbfs) and, when no image is left, ends the solve loop (hmain,
// 0 outside the loop) and, with `publish`, writes the results to the host (the graph solve
// ends here); the last cycle of a solve is counted here.  Every thread of one CTA calls it: k_flood_check,
// or the last CTA of the flood's last round, which reads what the round's other CTAs wrote
// (their fence before the round's count orders it), hence the volatile loads.
__device__ void flood_check_cta(const PoolView& P, int all, cudaGraphConditionalHandle hbfs,
                                cudaGraphConditionalHandle hmain, int publish,
                                const ImageAcc* acc) {
  __shared__ int s_left, s_n;
  if (threadIdx.x == 0) {
    s_left = 0;
    trace_record(P, TR_CHECK);
  }
  __syncthreads();
  volatile int32_t* ctl = P.ctl;
  const int stamp = ctl[CTL_CYCLES] + 1;
  int left = 0;
  for (int i = threadIdx.x; i < P.nimg; i += blockDim.x) {
    const bool part = all ? *((volatile int32_t*)&P.img_mode[i]) == 2
                          : *((volatile int32_t*)&P.img_live[i]) == stamp;
    if (!part) continue;
    if (*((volatile int32_t*)&P.img_hit[i]) == stamp) {
      P.img_live[i] = stamp;
      ++left;
    } else {
      P.img_live[i] = 0;   // solved: no later stamp equals 0
    }
  }
  if (left) atomicAdd(&s_left, left);
  __syncthreads();
  if (threadIdx.x == 0) {
    int n = s_left;
    if (ctl[CTL_ERR] != 0) n = 0;   // a cap or a self-check ends the loops
    ctl[CTL_LEFT] = n;
    ctl[CTL_NCHECK] = ctl[CTL_NCHECK] + 1;
    if (n == 0 && !all) ctl[CTL_CYCLES] = ctl[CTL_CYCLES] + 1;
    __threadfence();
    if (hbfs) cudaGraphSetConditional(hbfs, n > 0 ? 1u : 0u);
    if (hmain && n == 0) cudaGraphSetConditional(hmain, 0u);
    if (n == 0) trace_record(P, TR_END);
    s_n = n;
  }
  __syncthreads();
  if (s_n == 0 && publish) publish_results(P, acc, blockDim.x);   // the graph solve ends here
}

// End of a flood round: frontier_round_end's bookkeeping by the round's last CTA; when the
// flood is over (no frontier left, or a cap), that CTA runs the flood check too (check >= 0
// is its `all`), so the solve graph needs no separate check launch.  Every thread calls it.
__device__ __forceinline__ void flood_round_end(const PoolView& P, int first, int in, int parts,
                                                cudaGraphConditionalHandle h, int check,
                                                cudaGraphConditionalHandle hbfs,
                                                cudaGraphConditionalHandle hmain, int publish,
                                                const ImageAcc* acc) {
  __shared__ int s_last, s_more;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&P.ctl[CTL_DONE], 1) == parts - 1;
    if (s_last) {
      __threadfence();
      volatile int32_t* ctl = P.ctl;
      const int out = in ^ 1;
      P.rcnt[in] = 0;
      const int next = *((volatile int32_t*)&P.fcount[out]);
      P.fcount[in] = 0;   // this round's list is consumed
      ctl[CTL_LASTCNT] = next;
      ctl[CTL_RND] = first ? 1 : ctl[CTL_RND] + 1;
      const int rounds = first ? 1 : ctl[CTL_ROUNDS] + 1;
      ctl[CTL_ROUNDS] = rounds;
      ctl[CTL_FLOOD_TOTAL] = ctl[CTL_FLOOD_TOTAL] + 1;
      ctl[CTL_DONE] = 0;
      bool more = next > 0 && ctl[CTL_ERR] < 3;   // a copy or self-check error ends the loop
      if (more && rounds >= ctl[CTL_MAXROUNDS]) {
        ctl[CTL_ERR] = 1;
        more = false;
      }
      __threadfence();
      if (h) cudaGraphSetConditional(h, more ? 1u : 0u);
      s_more = more;
    }
  }
  __syncthreads();
  if (!s_last || check < 0 || s_more) return;
  flood_check_cta(P, check, hbfs, hmain, publish, acc);
}

// ------------------------------------------------------------------------------------
// Canonical cut: flood from excess pixels over residual edges (forward direction).
// The first flood round also sums max(excess, 0) per image for the flow value.
//
// The flood also decides termination: an excess pixel can reach a sink pixel exactly when
// the flood from the excess pixels reaches one, so an image whose flood reaches no sink
// pixel is solved (its flood is the canonical cut) and one whose flood does needs another
// global relabel and push cycle.  Every round stamps img_hit[img] with the cycle stamp
// (ctl[CTL_CYCLES] + 1) when a tile's reached set meets its sink pixels.
//
// mode: 0 frontier round; first rounds over the selected tiles: 1 all of them, 2 those of the
// images live in this cycle (img_live == stamp), 3 those of the images that continue from a
// previous flow (img_mode == 2).  abort_hit: frontier rounds skip the tiles of images already
// stamped (their flood is redone in a later cycle).
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(WARPS_PER_CTA * 32)
k_flood_round(PoolView P, int mode, int abort_hit, cudaGraphConditionalHandle h, ImageAcc* acc,
              int check, cudaGraphConditionalHandle hbfs, cudaGraphConditionalHandle hmain,
              int publish) {
  trace_mark(P, mode ? TR_FLOOD_FIRST : TR_FLOOD);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int first = mode != 0;
  const int in = frontier_round_number(P, first) & 1, out = in ^ 1;
  const int stamp = *((volatile int32_t*)&P.ctl[CTL_CYCLES]) + 1;
  int32_t* const markin = P.mark[in];
  int done = 0;
  int n, parts, nr;
  frontier_work(P, first, in, WARPS_PER_CTA, &n, &parts, &nr);
  if ((int)blockIdx.x >= parts) return;
  const int i0 = blockIdx.x * WARPS_PER_CTA + warp;
  SelCursor cursor(P, first ? nr : 0, i0);
  int wimg = -1;                 // first round: the image whose tile sums this warp holds
  unsigned long long wsum = 0;
  for (int i = i0; i < n; i += parts * WARPS_PER_CTA) {
    const int t = first ? cursor.tile(i) : P.fq[in][i];
    if (!first && lane == 0) markin[t] = 0;
    const int img = P.img_of[t];
    if ((unsigned)img >= (unsigned)P.nimg) {   // self-check
      if (lane == 0) record_bad(P, 4, img);
      continue;
    }
    if (mode == 2 && P.img_live[img] != stamp) continue;
    if (mode == 3 && P.img_mode[img] != 2) continue;
    if (mode == 0 && abort_hit && *((volatile int32_t*)&P.img_hit[img]) == stamp) continue;
    ++done;
    const int4 nb = P.nbr[t];
    uint32_t canU, canD, canL, canR, sink, R, R0;
    long long ps = 0;
    if (first && P.mdirty[t] != 0) {
      // the tile changed since its masks were written (a discharge or an edit): rebuild them
      // here, before anything reads them (every tile of an image this round covers is done
      // in this round, so the frontier rounds and the global relabel after it see them)
      const RowMasks m = warp_rebuild_masks(P, t, lane, &ps);
      canU = m.up; canD = m.down; canL = m.left; canR = m.right;
      sink = m.sink;
      R = m.exc;
    } else {
      const uint32_t* mc = P.mcan + (long long)t * 128;
      canU = mc[lane]; canD = mc[32 + lane]; canL = mc[64 + lane]; canR = mc[96 + lane];
      sink = P.msink[(long long)t * 32 + lane];
      if (first) {
        R = P.mexc[(long long)t * 32 + lane];
        ps = P.tpos[t];
      }
    }
    if (first) {
      R0 = 0;
      // Σ max(excess, 0) of the tile, taken with its masks; summed per warp and per CTA
      // before the add to the image's word
      if (lane == 0 && ps) {
        if (img != wimg) {
          if (wsum) atomicAdd(&acc[wimg].sumpos_e, wsum);
          wimg = img;
          wsum = 0;
        }
        wsum += (unsigned long long)ps;
      }
    } else {
      R = R0 = P.mreach[(long long)t * 32 + lane];
      if (lane == 0 && nb.x >= 0)
        R |= P.mreach[(long long)nb.x * 32 + 31] & P.mcan[(long long)nb.x * 128 + 32 + 31];
      if (lane == 31 && nb.y >= 0)
        R |= P.mreach[(long long)nb.y * 32] & P.mcan[(long long)nb.y * 128 + 0];
      if (nb.z >= 0 && ((P.mreach[(long long)nb.z * 32 + lane] & P.mcan[(long long)nb.z * 128 + 96 + lane]) >> 31))
        R |= 1u;
      if (nb.w >= 0 && ((P.mreach[(long long)nb.w * 32 + lane] & P.mcan[(long long)nb.w * 128 + 64 + lane]) & 1u))
        R |= 0x80000000u;
    }
    for (int guard = 0; guard < GC_TILE_PX + 1; ++guard) {
      uint32_t dn = __shfl_up_sync(0xffffffffu, R & canD, 1);   // row r-1 flows down into r
      uint32_t up = __shfl_down_sync(0xffffffffu, R & canU, 1); // row r+1 flows up into r
      if (lane == 0) dn = 0;
      if (lane == 31) up = 0;
      const uint32_t N = R | ((R & canR) << 1) | ((R & canL) >> 1) | dn | up;
      if (!__any_sync(0xffffffffu, N != R)) break;
      R = N;
    }
    P.mreach[(long long)t * 32 + lane] = R;
    if (__any_sync(0xffffffffu, (R & sink) != 0) && lane == 0 &&
        *((volatile int32_t*)&P.img_hit[img]) != stamp)
      P.img_hit[img] = stamp;
    const uint32_t nw = first ? R : (R & ~R0);
    const int sU = __any_sync(0xffffffffu, lane == 0 && (nw & canU));
    const int sD = __any_sync(0xffffffffu, lane == 31 && (nw & canD));
    const int sL = __any_sync(0xffffffffu, (nw & canL & 1u) != 0);
    const int sR = __any_sync(0xffffffffu, ((nw & canR) >> 31) != 0);
    if (lane < 4) {   // the neighbours to queue, one lane each
      const int go = lane == 0 ? sU : lane == 1 ? sD : lane == 2 ? sL : sR;
      const int nt = lane == 0 ? nb.x : lane == 1 ? nb.y : lane == 2 ? nb.z : nb.w;
      if (go && nt >= 0) frontier_push(P, out, nt);
    }
  }
  if (lane == 0 && done) {
    atomicAdd(&P.rcnt[in], done);
    if (P.ktiles) atomicAdd(&P.ktiles[first ? K_FLOOD_FIRST : K_FLOOD], (unsigned long long)done);
  }
  if (first) {   // the CTA's warps that summed the same image add once
    __shared__ int s_img[WARPS_PER_CTA];
    __shared__ unsigned long long s_sum[WARPS_PER_CTA];
    if (lane == 0) {
      s_img[warp] = wsum ? wimg : -1;
      s_sum[warp] = wsum;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int a = 0; a < WARPS_PER_CTA; ++a) {
        if (s_img[a] < 0) continue;
        unsigned long long v = s_sum[a];
        for (int b = a + 1; b < WARPS_PER_CTA; ++b)
          if (s_img[b] == s_img[a]) { v += s_sum[b]; s_img[b] = -1; }
        atomicAdd(&acc[s_img[a]].sumpos_e, v);
      }
    }
  }
  flood_round_end(P, first, in, parts, h, check, hbfs, hmain, publish, acc);
}

// After a flood (host-driven loops; the solve graph runs the check at the end of its last
// flood round instead): see flood_check_cta.  One CTA.
__global__ void k_flood_check(PoolView P, int all, cudaGraphConditionalHandle hbfs,
                              cudaGraphConditionalHandle hmain) {
  flood_check_cta(P, all, hbfs, hmain, 0, nullptr);
}

// Neighbour tile ids and image index of one image's tiles (row-major from im.tile0), for an
// image placed in a session pool.
__global__ void k_image_tiles(PoolView P, ImageDesc im, int img) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= im.tw * im.th) return;
  const int tx = k % im.tw, ty = k / im.tw, t = im.tile0 + k;
  P.nbr[t] = make_int4(ty > 0 ? t - im.tw : -1, ty < im.th - 1 ? t + im.tw : -1,
                       tx > 0 ? t - 1 : -1, tx < im.tw - 1 ? t + 1 : -1);
  P.img_of[t] = img;
}

// The labels kernels inside a solve graph that ends with the labels of its one image:
// `first`: the launch that follows the first cycle's flood writes only when that cycle's
// check left no image (the solve ended there; otherwise the launch at the end of the relabel
// IF node writes them).  `slot`: the output buffer is read from this device word, which the
// host sets when the caller's buffer changes, so the graph never changes.  Every thread
// reads words that earlier launches (or copies) wrote.
__device__ __forceinline__ bool labels_skip(const PoolView& P, int first) {
  return first && *((volatile int32_t*)&P.ctl[CTL_LEFT]) != 0;
}
__device__ __forceinline__ uint8_t* labels_dest(uint8_t* out, const unsigned long long* slot) {
  return slot ? reinterpret_cast<uint8_t*>(*((const volatile unsigned long long*)slot)) : out;
}

// Labels of one image, row-major, padding excluded.  One thread writes the 32 pixels of
// one tile row (one mask word); consecutive threads take consecutive tiles of an image row.
__global__ void k_labels_out(PoolView P, ImageDesc im, uint8_t* __restrict__ out_arg, int first,
                             const unsigned long long* slot) {
  if (labels_skip(P, first)) return;
  trace_mark(P, TR_LABELS);
  uint8_t* const out = labels_dest(out_arg, slot);
  const long long n = (long long)im.H * im.tw;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i / im.tw), tx = (int)(i % im.tw);
    const int t = im.tile0 + (y >> 5) * im.tw + tx;
    const uint32_t m = P.mreach[(long long)t * 32 + (y & 31)];
    const int x0 = tx * GC_TILE;
    uint8_t* row = out + (long long)y * im.W + x0;
    if (x0 + GC_TILE <= im.W && (((uintptr_t)row) & 3) == 0) {
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t b = (m >> (4 * k)) & 0xfu;
        const uint32_t w = (b & 1u) | ((b & 2u) << 7) | ((b & 4u) << 14) | ((b & 8u) << 21);
        reinterpret_cast<uint32_t*>(row)[k] = w;
      }
    } else {
      for (int c = 0; c < GC_TILE && x0 + c < im.W; ++c) row[c] = (uint8_t)((m >> c) & 1u);
    }
  }
}

// Bit-packed labels: thread (y, tx) writes the up to four bytes of tile column tx in row y
// (row stride (W + 7) / 8 bytes, little bit order).  Pixels of a ragged tile beyond the
// image have no capacities and no excess, so their reach bits are 0.
__global__ void k_labels_packed(PoolView P, ImageDesc im, uint8_t* __restrict__ out_arg,
                                int first, const unsigned long long* slot) {
  if (labels_skip(P, first)) return;
  trace_mark(P, TR_LABELS);
  uint8_t* const out = labels_dest(out_arg, slot);
  const long long n = (long long)im.H * im.tw;
  const int stride = (im.W + 7) >> 3;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i / im.tw), tx = (int)(i % im.tw);
    const int t = im.tile0 + (y >> 5) * im.tw + tx;
    const uint32_t m = P.mreach[(long long)t * 32 + (y & 31)];
    uint8_t* row = out + (long long)y * stride + 4 * tx;
    const int nb = stride - 4 * tx < 4 ? stride - 4 * tx : 4;
    if (nb == 4 && (((uintptr_t)row) & 3) == 0) {
      *reinterpret_cast<uint32_t*>(row) = m;
    } else {
      for (int k = 0; k < nb; ++k) row[k] = (uint8_t)(m >> (8 * k));
    }
  }
}

// One plane of one image back to row-major.
__global__ void k_state_out(ImageDesc im, const int32_t* __restrict__ plane, int32_t* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)im.W * im.H) return;
  const int y = (int)(i / im.W), x = (int)(i % im.W);
  const int t = im.tile0 + (y >> 5) * im.tw + (x >> 5);
  out[i] = plane[(long long)t * GC_TILE_PX + (y & 31) * GC_TILE + (x & 31)];
}

// T-link edits: excess moves by (new - old) t-link; the running sum of max(t, 0) follows.
__device__ __forceinline__ void apply_tlink(const PoolView& P, const ImageDesc& im, int img,
                                            int x, int y, int32_t v, int32_t* tl, ImageAcc* acc) {
  const int t = im.tile0 + (y >> 5) * im.tw + (x >> 5);
  const long long o = (long long)t * GC_TILE_PX + (y & 31) * GC_TILE + (x & 31);
  const int32_t old = tl[o];
  if (old == v) return;
  tl[o] = v;
  atomicAdd(P.exc + o, v - old);
  mark_dirty(P, t);
  const long long dpos = (long long)(v > 0 ? v : 0) - (long long)(old > 0 ? old : 0);
  if (dpos) atomicAdd(&acc[img].sumpos_t, (unsigned long long)dpos);
}

__global__ void k_edit(PoolView P, ImageDesc im, int img, const int32_t* __restrict__ idx,
                       const int32_t* __restrict__ val, int n, int32_t* tl, ImageAcc* acc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = idx[i];
  if (p < 0 || p >= im.W * im.H) return;
  apply_tlink(P, im, img, p % im.W, p / im.W, val[i], tl, acc);
}

// Stroke: pixels within `radius` of the polyline get t-link `value`.  Exact integer test:
// with a = p - A, b = B - A, L = b.b, s = a.b: inside iff |p - A|^2 <= r^2 (s <= 0),
// |p - B|^2 <= r^2 (s >= L), else |a|^2 L - s^2 <= r^2 L.
__device__ __forceinline__ bool in_stroke(int px, int py, const int32_t* pts, int npts, int r) {
  const long long r2 = (long long)r * r;
  for (int k = 0; k < (npts > 1 ? npts - 1 : 1); ++k) {
    const long long ax = pts[2 * k], ay = pts[2 * k + 1];
    const long long bx = npts > 1 ? pts[2 * k + 2] : ax, by = npts > 1 ? pts[2 * k + 3] : ay;
    const long long dx = px - ax, dy = py - ay, ux = bx - ax, uy = by - ay;
    const long long L = ux * ux + uy * uy, s = dx * ux + dy * uy;
    if (L == 0 || s <= 0) { if (dx * dx + dy * dy <= r2) return true; continue; }
    if (s >= L) { const long long ex = px - bx, ey = py - by; if (ex * ex + ey * ey <= r2) return true; continue; }
    if ((dx * dx + dy * dy) * L - s * s <= r2 * L) return true;
  }
  return false;
}

__global__ void k_stroke(PoolView P, ImageDesc im, int img, const int32_t* __restrict__ pts,
                         int npts, int radius, int32_t value, int x0, int y0, int bw, int bh,
                         int32_t* tl, ImageAcc* acc) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)bw * bh) return;
  const int x = x0 + (int)(i % bw), y = y0 + (int)(i / bw);
  if (x < 0 || y < 0 || x >= im.W || y >= im.H) return;
  if (!in_stroke(x, y, pts, npts, radius)) return;
  apply_tlink(P, im, img, x, y, value, tl, acc);
}

// Reference brush (gc_edit_brush): the pixel set of Brush.points (brush.pyx:138-161), the
// line pixels of each segment (skimage.draw.line: Bresenham, the minor axis stepping while
// the error term d = 2 dr - dc + ... is >= 0) widened by the disc of skimage.draw.circle, whose
// points satisfy (dy / R)^2 + (dx / R)^2 < 1 in float64.  The disc is centred on every line
// pixel (the reference adds circle(R, R, R), a disc shifted by +R) and pixels outside the
// image are skipped (the reference's y * W + x wraps them).
//
// Along the major axis (n steps, minor-axis travel m) Bresenham's i-th pixel has minor
// offset floor((2 m i + n) / (2 n)): the loop steps the minor axis once for every time the
// error term 2 m (i + 1) - n - 2 n k reaches 0, which is rounding m i / n to the nearest
// integer with halves up.  Each thread tests one pixel of the bounding box against the
// line pixels within R - 1 of it along the major axis, so every pixel is written once.
constexpr int GC_BRUSH_MAX_RADIUS = 1024;

// skimage's disc test for the offset (dy, dx): two quotients, two squares and a sum, each
// rounded on its own as numpy evaluates ((y - cy) / ry) ** 2 + ((x - cx) / rx) ** 2 < 1.
__device__ __forceinline__ bool brush_disk(int dy, int dx, int R) {
  const double a = __ddiv_rn((double)dy, (double)R), b = __ddiv_rn((double)dx, (double)R);
  return __dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)) < 1.0;
}

__device__ __forceinline__ bool in_brush(int px, int py, const int32_t* pts, int npts, int R,
                                         const int32_t* half) {
  const int nseg = npts > 1 ? npts - 1 : 1;
  for (int k = 0; k < nseg; ++k) {
    const int x0 = pts[2 * k], y0 = pts[2 * k + 1];
    const int x1 = npts > 1 ? pts[2 * k + 2] : x0, y1 = npts > 1 ? pts[2 * k + 3] : y0;
    const int dr = abs(y1 - y0), dc = abs(x1 - x0);
    const int sr = (y1 - y0) > 0 ? 1 : -1, sc = (x1 - x0) > 0 ? 1 : -1;
    const bool steep = dr > dc;
    const int n = steep ? dr : dc, m = steep ? dc : dr;       // major steps, minor travel
    const int a0 = steep ? y0 : x0, b0 = steep ? x0 : y0;     // major / minor start
    const int sa = steep ? sr : sc, sb = steep ? sc : sr;
    const int pa = steep ? py : px;
    const int t = sa * (pa - a0);                             // pixel's major-axis step
    const int ilo = max(t - (R - 1), 0), ihi = min(t + (R - 1), n);
    for (int i = ilo; i <= ihi; ++i) {
      const int bi = n > 0 ? b0 + sb * (int)((2LL * m * i + n) / (2LL * n)) : b0;
      const int ai = a0 + sa * i;
      const int dy = py - (steep ? ai : bi), dx = px - (steep ? bi : ai);
      if (dy < 1 - R || dy > R - 1) continue;
      const int w = half[dy + R - 1];
      if (dx >= -w && dx <= w) return true;
    }
  }
  return false;
}

__global__ void k_brush(PoolView P, ImageDesc im, int img, const int32_t* __restrict__ pts,
                        int npts, int R, int32_t value, int x0, int y0, int bw, int bh,
                        int32_t* tl, ImageAcc* acc) {
  // half[dy + R - 1] = the largest dx >= 0 with the offset (dy, dx) inside the disc (the
  // test is monotone in |dx|; dx = 0 is inside for |dy| <= R - 1)
  __shared__ int32_t half[2 * GC_BRUSH_MAX_RADIUS - 1];
  for (int j = threadIdx.x; j < 2 * R - 1; j += blockDim.x) {
    const int dy = j - (R - 1);
    int lo = 0, hi = R - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (brush_disk(dy, mid, R)) lo = mid; else hi = mid - 1;
    }
    half[j] = lo;
  }
  __syncthreads();
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)bw * bh) return;
  const int x = x0 + (int)(i % bw), y = y0 + (int)(i / bw);
  if (x < 0 || y < 0 || x >= im.W || y >= im.H) return;
  if (!in_brush(x, y, pts, npts, R, half)) return;
  apply_tlink(P, im, img, x, y, value, tl, acc);
}

// ------------------------------------------------------------------------------------
// Launchers
// ------------------------------------------------------------------------------------
static inline int ok() { return cudaGetLastError() == cudaSuccess ? GC_OK : GC_ERR_CUDA; }

int launch_upload(const PoolView& P, const ImageDesc& im, int img, const int32_t* up,
                  const int32_t* down, const int32_t* left, const int32_t* right,
                  const int32_t* excess, int32_t* tl, ImageAcc* acc, cudaStream_t s) {
  auto a16 = [](const int32_t* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  const bool vec = im.W % 4 == 0 && a16(up) && a16(down) && a16(left) && a16(right) && a16(excess);
  const PlaneSource src{up, down, left, right, excess, vec};
  k_upload<<<im.tw * im.th, DIS_THREADS, 0, s>>>(P, im, img, src, tl, acc);
  return ok();
}

int launch_upload_rgba(const PoolView& P, const ImageDesc& im, int img, const uint32_t* rgba,
                       const int32_t* excess, const int32_t* tab, int lambda, int32_t* tl,
                       ImageAcc* acc, cudaStream_t s) {
  const RgbaSource src{rgba, excess, tab, lambda};
  k_upload<<<im.tw * im.th, DIS_THREADS, 0, s>>>(P, im, img, src, tl, acc);
  return ok();
}

int launch_nlink_table(const unsigned long long* sum, long long npairs, int32_t* tab,
                       cudaStream_t s) {
  k_nlink_table<<<1, 64, 0, s>>>(sum, npairs, tab);
  return ok();
}

// Sum over all 4-neighbour pairs of |I_i - I_j|^2 (R, G, B), exact in 64 bits: the mean the
// n-link scale beta comes from.
__global__ void __launch_bounds__(256) k_dsum(const uint32_t* __restrict__ rgba, int W, int H,
                                              unsigned long long* sum) {
  __shared__ unsigned long long part[8];
  unsigned long long acc = 0;
  const long long n = (long long)W * H;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % W);
    const uint32_t c = rgba[i];
    if (i >= W) acc += (unsigned)rgb_dist2(c, rgba[i - W]);
    if (x > 0) acc += (unsigned)rgb_dist2(c, rgba[i - 1]);
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long tsum = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) tsum += part[k];
    if (tsum) atomicAdd(sum, tsum);
  }
}

int launch_dsum(const uint32_t* rgba, int W, int H, unsigned long long* sum, int sms,
                cudaStream_t s) {
  const long long n = (long long)W * H;
  long long blocks = (n + 255) / 256;
  if (blocks > 8LL * sms) blocks = 8LL * sms;
  k_dsum<<<(unsigned)(blocks > 0 ? blocks : 1), 256, 0, s>>>(rgba, W, H, sum);
  return ok();
}

int launch_masks(const PoolView& P, int grid, cudaStream_t s) {
  k_masks<<<grid, WARPS_PER_CTA * 32, 0, s>>>(P);
  return ok();
}

int launch_discharge(const PoolView& P, int iters, int grid, cudaStream_t s) {
  k_discharge<<<grid, DIS_THREADS, DIS_DYN_SMEM, s>>>(P, iters);
  return ok();
}

int launch_edge_relabel_build(const PoolView& P, int32_t* list, int32_t* count,
                              const ScanState& st, cudaStream_t s) {
  const int nch = (P.nt + EB_TILES - 1) / EB_TILES;
  if (nch > st.max_chunks) return GC_ERR_INVALID;
  k_edge_relabel_build<<<nch, EB_THREADS, 0, s>>>(P, list, count, st);
  return ok();
}

int launch_bfs_round(const PoolView& P, int first, cudaGraphConditionalHandle h, int grid,
                     cudaStream_t s) {
  k_bfs_round<<<grid, WARPS_PER_CTA * 32, 0, s>>>(P, first, h);
  return ok();
}

int launch_flood_round(const PoolView& P, int mode, int abort_hit, cudaGraphConditionalHandle h,
                       ImageAcc* acc, int grid, cudaStream_t s, int check,
                       cudaGraphConditionalHandle hbfs, cudaGraphConditionalHandle hmain,
                       int publish) {
  k_flood_round<<<grid, WARPS_PER_CTA * 32, 0, s>>>(P, mode, abort_hit, h, acc, check, hbfs, hmain,
                                                    publish);
  return ok();
}

int launch_flood_check(const PoolView& P, int all, cudaGraphConditionalHandle hbfs,
                       cudaGraphConditionalHandle hmain, cudaStream_t s) {
  k_flood_check<<<1, 256, 0, s>>>(P, all, hbfs, hmain);
  return ok();
}

__global__ void k_acc_reset(ImageAcc* acc, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) acc[i].sumpos_e = 0;
}

int launch_acc_reset(ImageAcc* acc, int n, cudaStream_t s) {
  k_acc_reset<<<(n + 255) / 256, 256, 0, s>>>(acc, n);
  return ok();
}

int launch_ctl_begin(const PoolView& P, int max_rounds, int max_cycles, ImageAcc* acc,
                     cudaStream_t s) {
  k_ctl_begin<<<1, 256, 0, s>>>(P, max_rounds, max_cycles, acc);
  return ok();
}

int launch_active_list(const PoolView& P, const ScanState& st, int32_t* list, int32_t* count,
                       int bump, int count_cycle, int filter, cudaGraphConditionalHandle h,
                       ImageAcc* acc, int grid, cudaStream_t s) {
  const int nch = (P.nt + ACT_CHUNK - 1) / ACT_CHUNK;   // enough for any selection
  if (nch > st.max_chunks) return GC_ERR_INVALID;
  grid = grid < nch ? grid : nch;
  k_active_list<<<grid > 0 ? grid : 1, ACT_THREADS, 0, s>>>(P, st, list, count, bump, count_cycle,
                                                            filter, h, acc);
  return ok();
}

int begin_list_max_tiles() { return BL_MAX; }

int launch_begin_list(const PoolView& P, int max_rounds, int max_cycles, ImageAcc* acc,
                      int32_t* list, int32_t* count, cudaGraphConditionalHandle h, cudaStream_t s) {
  if (P.nt > BL_MAX) return GC_ERR_INVALID;
  k_begin_list<<<1, BL_THREADS, 0, s>>>(P, max_rounds, max_cycles, acc, list, count, h);
  return ok();
}

int launch_ctl_cycle(const PoolView& P, const int32_t* count, int count_cycle,
                     cudaGraphConditionalHandle h, cudaStream_t s) {
  k_ctl_cycle<<<1, 32, 0, s>>>(P, count, count_cycle, h);
  return ok();
}

int launch_image_tiles(const PoolView& P, const ImageDesc& im, int img, cudaStream_t s) {
  const int n = im.tw * im.th;
  if (n <= 0) return GC_OK;
  k_image_tiles<<<(n + 255) / 256, 256, 0, s>>>(P, im, img);
  return ok();
}

// one thread per tile row of the image; grid_cap > 0 caps the CTAs (they stride over rows)
static unsigned labels_grid(const ImageDesc& im, int grid_cap) {
  const long long need = ((long long)im.H * im.tw + 255) / 256;
  const long long g = grid_cap > 0 && need > grid_cap ? grid_cap : need;
  return (unsigned)(g < 1 ? 1 : g);
}

int launch_labels_out(const PoolView& P, const ImageDesc& im, uint8_t* out, cudaStream_t s,
                      int first, const unsigned long long* slot, int grid_cap) {
  k_labels_out<<<labels_grid(im, grid_cap), 256, 0, s>>>(P, im, out, first, slot);
  return ok();
}

int launch_labels_packed(const PoolView& P, const ImageDesc& im, uint8_t* out, cudaStream_t s,
                         int first, const unsigned long long* slot, int grid_cap) {
  k_labels_packed<<<labels_grid(im, grid_cap), 256, 0, s>>>(P, im, out, first, slot);
  return ok();
}

int launch_state_out(const PoolView& P, const ImageDesc& im, const int32_t* plane,
                     int32_t* out, cudaStream_t s) {
  (void)P;
  const long long n = (long long)im.W * im.H;
  k_state_out<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(im, plane, out);
  return ok();
}

int launch_edit(const PoolView& P, const ImageDesc& im, int img, const int32_t* idx,
                const int32_t* val, int n, int32_t* tl, ImageAcc* acc, cudaStream_t s) {
  if (n <= 0) return GC_OK;
  k_edit<<<(n + 255) / 256, 256, 0, s>>>(P, im, img, idx, val, n, tl, acc);
  return ok();
}

int launch_stroke(const PoolView& P, const ImageDesc& im, int img, const int32_t* pts_dev,
                  const int32_t* pts_host, int npts, int radius, int32_t value, int32_t* tl,
                  ImageAcc* acc, cudaStream_t s) {
  int xmin = pts_host[0], xmax = pts_host[0], ymin = pts_host[1], ymax = pts_host[1];
  for (int k = 1; k < npts; ++k) {
    xmin = xmin < pts_host[2 * k] ? xmin : pts_host[2 * k];
    xmax = xmax > pts_host[2 * k] ? xmax : pts_host[2 * k];
    ymin = ymin < pts_host[2 * k + 1] ? ymin : pts_host[2 * k + 1];
    ymax = ymax > pts_host[2 * k + 1] ? ymax : pts_host[2 * k + 1];
  }
  int x0 = xmin - radius, y0 = ymin - radius, x1 = xmax + radius, y1 = ymax + radius;
  x0 = x0 < 0 ? 0 : x0; y0 = y0 < 0 ? 0 : y0;
  x1 = x1 > im.W - 1 ? im.W - 1 : x1; y1 = y1 > im.H - 1 ? im.H - 1 : y1;
  if (x1 < x0 || y1 < y0) return GC_OK;
  const int bw = x1 - x0 + 1, bh = y1 - y0 + 1;
  const long long n = (long long)bw * bh;
  k_stroke<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(P, im, img, pts_dev, npts, radius, value,
                                                     x0, y0, bw, bh, tl, acc);
  return ok();
}

int launch_brush(const PoolView& P, const ImageDesc& im, int img, const int32_t* pts_dev,
                 const int32_t* pts_host, int npts, int radius, int32_t value, int32_t* tl,
                 ImageAcc* acc, cudaStream_t s) {
  const int R = radius < 1 ? 1 : radius;
  if (R > GC_BRUSH_MAX_RADIUS) return GC_ERR_INVALID;
  int xmin = pts_host[0], xmax = pts_host[0], ymin = pts_host[1], ymax = pts_host[1];
  for (int k = 1; k < npts; ++k) {
    xmin = xmin < pts_host[2 * k] ? xmin : pts_host[2 * k];
    xmax = xmax > pts_host[2 * k] ? xmax : pts_host[2 * k];
    ymin = ymin < pts_host[2 * k + 1] ? ymin : pts_host[2 * k + 1];
    ymax = ymax > pts_host[2 * k + 1] ? ymax : pts_host[2 * k + 1];
  }
  long long x0 = (long long)xmin - (R - 1), y0 = (long long)ymin - (R - 1);
  long long x1 = (long long)xmax + (R - 1), y1 = (long long)ymax + (R - 1);
  x0 = x0 < 0 ? 0 : x0; y0 = y0 < 0 ? 0 : y0;
  x1 = x1 > im.W - 1 ? im.W - 1 : x1; y1 = y1 > im.H - 1 ? im.H - 1 : y1;
  if (x1 < x0 || y1 < y0) return GC_OK;
  const int bw = (int)(x1 - x0 + 1), bh = (int)(y1 - y0 + 1);
  const long long n = (long long)bw * bh;
  k_brush<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(P, im, img, pts_dev, npts, R, value,
                                                     (int)x0, (int)y0, bw, bh, tl, acc);
  return ok();
}

// Loads every kernel of the library on the current device.  With lazy module loading (the
// CUDA default) a kernel is loaded at its first launch or graph instantiation; doing it
// here, once per device under a lock, keeps that loading away from threads that solve on
// several streams at once.
void preload_kernels() {
  static std::mutex mu;
  static std::unordered_map<int, bool> done;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  std::lock_guard<std::mutex> lock(mu);
  if (done[dev]) return;
  cudaFuncAttributes a;
  const void* kernels[] = {
      (const void*)k_upload<PlaneSource>, (const void*)k_upload<RgbaSource>, (const void*)k_dsum,
      (const void*)k_nlink_table,
      (const void*)k_masks, (const void*)k_discharge, (const void*)k_edge_relabel_build,
      (const void*)k_bfs_round, (const void*)k_flood_round, (const void*)k_ctl_begin,
      (const void*)k_active_list, (const void*)k_begin_list, (const void*)k_ctl_cycle,
      (const void*)k_flood_check,
      (const void*)k_image_tiles,
      (const void*)k_acc_reset, (const void*)k_labels_out, (const void*)k_labels_packed,
      (const void*)k_state_out, (const void*)k_edit, (const void*)k_stroke,
      (const void*)k_brush};
  for (const void* k : kernels) cudaFuncGetAttributes(&a, k);
  preload_scan_kernels();
  cudaGetLastError();
  done[dev] = true;
}

namespace {
// Launch geometry per device, set up once: the dynamic shared memory opt-in of k_discharge
// changes the function's state, so it is not repeated while other threads launch or
// instantiate graphs that contain the kernel.
struct Geometry { int dis = 0, warps = 0; };
std::mutex g_geom_mu;
std::unordered_map<int, Geometry> g_geom;

Geometry device_geometry(int device) {
  std::lock_guard<std::mutex> lock(g_geom_mu);
  auto it = g_geom.find(device);
  if (it != g_geom.end()) return it->second;
  preload_kernels();
  int per_dis = 0, per_bfs = 0, sms = 0;
  cudaFuncSetAttribute(k_discharge, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)DIS_DYN_SMEM);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_dis, k_discharge, DIS_THREADS, DIS_DYN_SMEM);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_bfs, k_bfs_round, WARPS_PER_CTA * 32, 0);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  sms = sms > 0 ? sms : 1;
  Geometry g{(per_dis > 0 ? per_dis : 1) * sms, (per_bfs > 0 ? per_bfs : 1) * sms};
  g_geom.emplace(device, g);
  return g;
}
}  // namespace

int occupancy_discharge(int device) { return device_geometry(device).dis; }
int occupancy_warps(int device) { return device_geometry(device).warps; }

}  // namespace gcut
