// Shared definitions for the sm_100a tiled push-relabel graph cut.
//
// Data layout in HBM (tile-major "tile pool"):
//   A pool holds NT tiles of 32x32 pixels, possibly from several images.  Every per-pixel
//   plane is stored tile after tile: plane[t * 1024 + r * 32 + c] is pixel (r, c) of tile t,
//   so one tile of one plane is a contiguous 4 KiB block and a warp reading a tile row reads
//   one 128-byte line.  Planes: excess (signed t-link + net inflow), height, and the four
//   residual capacities cap_up/down/left/right (edge from the pixel to that neighbour).
//   Per tile: its four neighbour tile ids (-1 outside the image), 32-bit row masks used by
//   the bit-parallel BFS (residual edge present per direction, sink pixels, excess pixels,
//   reachable pixels) and small int flags.
//
// All arithmetic is int32 (int64 for the flow sums); heights use HINF for "cannot reach a
// sink pixel".
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define GC_TILE 32
#define GC_TILE_PX 1024
#define GC_HINF 0x3fffffff

namespace gcut {

enum { DUP = 0, DDOWN = 1, DLEFT = 2, DRIGHT = 3 };

// Device view of a tile pool.  All pointers are device pointers.
struct PoolView {
  int nt;                 // tiles in the pool
  int32_t* exc;           // [nt][1024]
  int32_t* hgt;           // [nt][1024]
  int32_t* cap[4];        // [nt][1024] each: up, down, left, right
  int4* nbr;              // [nt] neighbour tile ids (up, down, left, right), -1 if none
  uint32_t* mcan;         // [nt][4][32] residual-edge row masks (up, down, left, right)
  uint32_t* msink;        // [nt][32]   excess < 0
  uint32_t* mexc;         // [nt][32]   excess > 0
  uint32_t* mreach;       // [nt][32]   reachable from an excess pixel (canonical cut)
  int32_t* touched;       // [nt] tile was discharged or received cross-tile flow
  int32_t* act_int;       // [nt] tile has an active interior pixel after its discharge
  int32_t* mark[2];       // [nt] BFS / flood-fill frontier marks, alternating by round
  int32_t* rcnt;          // [2] tiles processed by the current / next frontier round
  int32_t* ctl;           // [CTL_N] device-side loop control (see CtlSlot)
  int32_t* queue[2];      // [nt] active-tile worklists, alternating by pulse
  int32_t* qcount;        // [2] worklist lengths
  int32_t* inq[2];        // [nt] tile is in queue[k] (deduplication)
  int32_t* fq[2];         // [nt] frontier lists of the BFS / flood rounds (dedup by mark[k])
  int32_t* fcount;        // [2] frontier list lengths
  int32_t* tact;          // [nt] tile has an active pixel (excess > 0, height < HINF)
  int32_t* img_of;        // [nt] image index of the tile
  int32_t* mdirty;        // [nt] the tile's planes changed after its masks were written
  long long* tpos;        // [nt] sum of max(excess, 0) over the tile (with the masks)
  int nimg;               // images in the pool
  int32_t* img_live;      // [nimg] cycle stamp of images that still have active tiles
  int32_t* img_hit;       // [nimg] cycle stamp: the image's flood reached a sink pixel
  int32_t* img_mode;      // [nimg] the image's part in this solve: 0 none, 1 fresh upload
                          // (trivial labelling), 2 continues from its previous flow
  // The solve's selection: the tile ranges of the images it solves (first rounds and
  // active-tile lists walk these instead of the whole pool)
  int4* sel;              // [nimg] first tile, tiles, first selected index, image
  int32_t* sel_mode;      // [nimg] img_mode of the range's image
  int32_t* nsel;          // [2] ranges, selected tiles in all
  unsigned long long* ktiles;  // [K_COUNT] tiles processed per kernel kind (profiling)
  // device-side trace of the solve: trace_ctl[0] on, trace_ctl[1] entries written; entry i
  // is (start time in ns of %globaltimer, kind) in trace[2i], trace[2i + 1].  trace_ctl is
  // null while tracing is off, so the kernels skip the mark without a memory access.
  unsigned long long* trace;
  int32_t* trace_ctl;
  // pinned host memory (as the device sees it) that the kernel ending a graph solve writes
  // the control words and the per-image sums to; null: the graph copies them instead
  int32_t* host_out;
};

// Device-side loop control words.  The last CTA of every frontier round advances the round
// parity and decides whether another round follows; in a CUDA graph it also sets the
// condition of the enclosing WHILE node, so no host round trip is needed per round.
enum CtlSlot {
  CTL_RND = 0,        // frontier round number (its parity selects the mark buffer)
  CTL_DONE = 1,       // CTAs finished in the current round
  CTL_LASTCNT = 2,    // tiles processed by the last finished round
  CTL_ROUNDS = 3,     // rounds of the current frontier loop
  CTL_BFS_TOTAL = 4,  // BFS rounds of the solve
  CTL_FLOOD_TOTAL = 5,
  CTL_CYCLES = 6,     // global-relabel cycles of the solve
  CTL_ERR = 7,        // 1: round cap, 2: cycle cap, 3: copy wait gave up, 4: self-check
  CTL_MAXROUNDS = 8,
  CTL_MAXCYCLES = 9,
  CTL_PULSE = 10,     // discharge launches since the last list rebuild (parity = worklist)
  CTL_DDONE = 11,     // CTAs finished in the current discharge launch
  CTL_BAD = 12,       // first out-of-range worklist value seen by a self-check
  CTL_BADWHERE = 13,  // 1: worklist append, 2: worklist length, 3: list length, 4: image id
                      // (or tile) of the selection, 5: frontier append, 6: frontier length,
                      // 9: selection size
  CTL_RESERVED = 14,
  CTL_NCHECK = 15,    // flood checks run (k_flood_check launches)
  CTL_NACT = 16,      // active-list rebuilds run (k_active_list launches)
  CTL_LEFT = 17,      // images still running after the last flood check
  CTL_SCANERR = 18,   // the scan state's error word, as the last active list saw it
  CTL_N = 64          // the control words fill 256 bytes; the per-image sums follow them
};

// Walks consecutive selected indices: the tile of index i, with the range found once by a
// binary search over the ranges' first indices and then followed range by range.
struct SelCursor {
  const int4* sel;
  int nr, k;
  int4 cur;
  __device__ __forceinline__ SelCursor(const PoolView& P, int nranges, int i) : sel(P.sel), nr(nranges) {
    int lo = 0, hi = nr - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (sel[mid].z <= i) lo = mid; else hi = mid - 1;
    }
    k = lo;
    cur = nr > 0 ? sel[k] : make_int4(0, 0, 0, 0);
  }
  // tile of selected index i (i >= the previous index asked for)
  __device__ __forceinline__ int tile(int i) {
    while (i >= cur.z + cur.y && k + 1 < nr) cur = sel[++k];
    return cur.x + (i - cur.z);
  }
  __device__ __forceinline__ int image() const { return cur.w; }
};

// A self-check found a worklist value outside the pool: keep the first one, flag the solve
// (the loops stop at the next check and the host returns GC_ERR_INTERNAL).
__device__ __forceinline__ void record_bad(const PoolView& P, int where, int value) {
  if (atomicCAS(&P.ctl[CTL_BADWHERE], 0, where) == 0) P.ctl[CTL_BAD] = value;
  atomicCAS(&P.ctl[CTL_ERR], 0, 4);
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Kinds of the device-side trace (gc_set_trace); the values are part of the C ABI.
enum TraceKind { TR_BEGIN = 0, TR_ACTIVE_LIST, TR_DISCHARGE, TR_MASKS, TR_FLOOD_FIRST, TR_FLOOD,
                 TR_CHECK, TR_BFS_FIRST, TR_BFS, TR_UPLOAD, TR_LABELS, TR_END };
#ifndef GC_TRACE_MAX
#define GC_TRACE_MAX 2048
#endif

// Records an event in the solve's trace when tracing is on (one calling thread).
__device__ __forceinline__ void trace_record(const PoolView& P, int kind) {
  if (!P.trace_ctl) return;
  if (*((volatile int32_t*)&P.trace_ctl[0]) == 0) return;
  const int i = atomicAdd(&P.trace_ctl[1], 1);
  if (i < GC_TRACE_MAX) {
    P.trace[2 * i] = global_ns();
    P.trace[2 * i + 1] = (unsigned long long)kind;
  }
}

// Records the start of a kernel in the solve's trace (CTA 0, thread 0, when tracing is on).
__device__ __forceinline__ void trace_mark(const PoolView& P, int kind) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  trace_record(P, kind);
}

// Kernel kinds for profiling (launch counts, event time, tiles processed).
enum KernelKind { K_UPLOAD = 0, K_DISCHARGE, K_EDGE_BUILD, K_BFS_FIRST, K_BFS, K_FLOOD_FIRST,
                  K_FLOOD, K_COMPACT, K_LABELS, K_MASKS, K_COUNT };

// Decoupled look-back bookkeeping (single-pass scan).  status[] words are tagged with the
// launch sequence number, so no reset is needed between launches.
struct ScanState {
  unsigned long long* status;  // [max chunks]
  int32_t* ticket;             // dynamic chunk ids (reset by the last CTA)
  int32_t* done;               // finished CTAs (reset by the last CTA)
  uint32_t* seq;               // launch sequence tag (bumped by the last CTA)
  int32_t* err;                // set when a look-back wait gives up (sticky until read)
  int max_chunks;
  int spin_limit;              // polls before a look-back wait gives up; 0: GC_SPIN_LIMIT
};

enum ScanStateFlag : unsigned { SS_NONE = 0, SS_AGG = 1, SS_PREFIX = 2 };

__device__ __forceinline__ unsigned long long ss_pack(uint32_t tag, unsigned st, int32_t v) {
  return ((unsigned long long)(tag & 0x3fffffffu) << 34) | ((unsigned long long)st << 32) |
         (unsigned long long)(uint32_t)v;
}

// Spin limit for look-back waits: after this many polls the wait gives up, records an
// error and continues, so a scheduling anomaly can never hang the GPU.
#define GC_SPIN_LIMIT (1 << 22)

__device__ __forceinline__ int spin_limit_of(const ScanState& st) {
  return st.spin_limit > 0 ? st.spin_limit : GC_SPIN_LIMIT;
}

// Called by one thread (thread 0) of the CTA owning chunk `chunk` after it knows its own
// aggregate.  Publishes the aggregate, walks back over predecessors and returns the
// exclusive prefix of the chunk.  Chunks are numbered by arrival ticket, so every
// predecessor belongs to a CTA that is already running.
__device__ __forceinline__ int32_t lookback_exclusive(const ScanState& st, uint32_t tag,
                                                      int chunk, int32_t aggregate) {
  volatile unsigned long long* status = st.status;
  if (chunk == 0) {
    __threadfence();
    status[0] = ss_pack(tag, SS_PREFIX, aggregate);
    return 0;
  }
  status[chunk] = ss_pack(tag, SS_AGG, aggregate);
  __threadfence();
  int32_t excl = 0;
  int j = chunk - 1;
  int spins = 0;
  const int limit = spin_limit_of(st);
  while (j >= 0) {
    unsigned long long s = status[j];
    uint32_t stag = (uint32_t)(s >> 34);
    unsigned sst = (unsigned)((s >> 32) & 3u);
    if (stag != (tag & 0x3fffffffu) || sst == SS_NONE) {
      if (++spins > limit) {
        atomicExch(st.err, 1);
        break;
      }
      __nanosleep(32);
      continue;
    }
    excl += (int32_t)(uint32_t)(s & 0xffffffffull);
    if (sst == SS_PREFIX) break;
    --j;
  }
  __threadfence();
  status[chunk] = ss_pack(tag, SS_PREFIX, excl + aggregate);
  return excl;
}

// Warp-parallel variant, executed by all 32 lanes of one warp: each step inspects the
// status words of 32 predecessors at once.  Returns the exclusive prefix to every lane.
__device__ __forceinline__ int32_t lookback_exclusive_warp(const ScanState& st, uint32_t tag,
                                                           int chunk, int32_t aggregate) {
  const int lane = threadIdx.x & 31;
  volatile unsigned long long* status = st.status;
  const uint32_t tg = tag & 0x3fffffffu;
  if (chunk == 0) {
    if (lane == 0) { __threadfence(); status[0] = ss_pack(tag, SS_PREFIX, aggregate); }
    return 0;
  }
  if (lane == 0) { status[chunk] = ss_pack(tag, SS_AGG, aggregate); __threadfence(); }
  __syncwarp();
  int32_t excl = 0;
  int j = chunk - 1;
  int spins = 0;
  const int limit = spin_limit_of(st);
  bool gave_up = false;
  while (j >= 0) {
    const int idx = j - lane;
    unsigned long long s = 0;
    unsigned sst = SS_PREFIX;
    int32_t v = 0;
    bool ready = true;
    if (idx >= 0) {
      s = status[idx];
      sst = (unsigned)((s >> 32) & 3u);
      ready = (uint32_t)(s >> 34) == tg && sst != SS_NONE;
      v = (int32_t)(uint32_t)(s & 0xffffffffull);
    }
    if (!__all_sync(0xffffffffu, ready)) {
      if (++spins > limit) { gave_up = true; break; }
      __nanosleep(32);
      continue;
    }
    const unsigned pm = __ballot_sync(0xffffffffu, idx >= 0 && sst == SS_PREFIX);
    const int stop = pm ? __ffs(pm) - 1 : 31;      // nearest predecessor with a prefix
    int32_t w = (lane <= stop && idx >= 0) ? v : 0;
#pragma unroll
    for (int o = 16; o; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
    excl += w;
    if (pm || j - 31 < 0) break;
    j -= 32;
  }
  if (lane == 0) {
    if (gave_up) atomicExch(st.err, 1);
    __threadfence();
    status[chunk] = ss_pack(tag, SS_PREFIX, excl + aggregate);
  }
  return excl;
}

// Last CTA to finish resets the tickets and bumps the tag for the next launch; returns
// true in that CTA (every other CTA's writes are visible to it).
__device__ __forceinline__ bool scan_finish(const ScanState& st, int nchunks) {
  __threadfence();
  int d = atomicAdd(st.done, 1);
  if (d == nchunks - 1) {
    __threadfence();
    *st.ticket = 0;
    *st.done = 0;
    uint32_t s = *st.seq + 1;
    if ((s & 0x3fffffffu) == 0) s = 1;
    *st.seq = s;
    __threadfence();
    return true;
  }
  return false;
}

// Block-wide exclusive scan of one int per thread (blockDim.x multiple of 32, <= 1024).
// Returns the exclusive prefix; *total gets the block sum.  `sm` needs 32 ints.
__device__ __forceinline__ int32_t block_exclusive_scan(int32_t v, int32_t* sm, int32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sm[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int32_t w = lane < nw ? sm[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    sm[lane] = w;  // inclusive warp prefix
  }
  __syncthreads();
  int32_t base = warp ? sm[warp - 1] : 0;
  *total = sm[nw - 1];
  __syncthreads();
  return base + x - v;
}

}  // namespace gcut
