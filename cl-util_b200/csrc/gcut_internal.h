// Internal interfaces between the translation units of libgcut.so.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/gcut.h"
#include "gcut_common.cuh"

static_assert(gcut::K_COUNT == GC_NKERN, "kernel kinds");

namespace gcut {

enum ScanMode {
  GC_SCAN_MODE_SCAN = 0,     // exclusive scan of values
  GC_SCAN_MODE_COMPACT = 1,  // indices of non-zero values
  GC_SCAN_MODE_FLAG = 2,     // indices where op1(in, a1)
  GC_SCAN_MODE_LOGICAL = 3,  // indices where op1(in, a1) AND/OR op2(in2, a2)
};

int scan_chunks(int n);
// Records the message returned by gc_last_error() for the calling thread; returns code.
int set_last_error(int code, const char* msg);
int launch_scan(int mode, const int32_t* in, const int32_t* in2, int32_t* clear,
                int32_t* scan_out, int32_t* list_out, int32_t* total_out, int n, int op1,
                int32_t a1, int op2, int32_t a2, int logical, const ScanState& st,
                cudaStream_t s);
// One warp waits on a look-back predecessor that never publishes, until st.spin_limit
// polls run out (sets *st.err); needs st.max_chunks >= 2.
int launch_lookback_selftest(const ScanState& st, cudaStream_t s);
int launch_increment_logical(const int32_t* in1, const int32_t* in2, int32_t* out, int n,
                             int op1, int op2, int32_t a1, int32_t a2, int logical,
                             int32_t iteration, cudaStream_t s);
int launch_fill(int32_t* p, int n, int32_t v, cudaStream_t s);
int launch_tiles_view(const int32_t* tiles, int tiles_w, int tiles_h, int tile_w, int tile_h,
                      int32_t iteration, int width, int height, uint32_t* out, cudaStream_t s);

// One image inside a tile pool.
struct ImageDesc {
  int W, H;      // pixel size
  int tw, th;    // tile grid
  int tile0;     // first tile id; tiles are row-major from there
};

// Per-image accumulators on the device.
struct ImageAcc {
  unsigned long long sumpos_t;   // sum max(t-link, 0)  (two's complement int64)
  unsigned long long sumpos_e;   // sum max(excess, 0) at the end of a solve
  int32_t bad_caps;              // negative capacities seen at upload
  int32_t pad;
};

// Solver kernels (gcut_solver.cu).
struct Launch {
  int grid_discharge;   // persistent CTAs for the discharge kernel
  int grid_warps;       // CTAs (4 warps each) for the per-tile warp kernels
};

int launch_upload(const PoolView& P, const ImageDesc& im, int img, const int32_t* up,
                  const int32_t* down, const int32_t* left, const int32_t* right,
                  const int32_t* excess, int32_t* tl, ImageAcc* acc, cudaStream_t s);
// reads the worklist queue[ctl[CTL_PULSE] & 1], builds the other one
int launch_masks(const PoolView& P, int grid, cudaStream_t s);

// n-link table of gc_upload_rgba: weight(d) = floor(50 * exp(-beta * d) + 0.5) for d = |dI|^2
// equals the number of entries t[k] >= d (t[k] = largest d with weight >= k + 1).
constexpr int GC_NLINK_LEVELS = 50;
// tab: the 50 device thresholds (exp weighting), or null for the reference's weighting
// floor(lambda / (0.1 sqrt(d) + 0.05) + 0.5) (gc_upload_rgba_lambda)
int launch_upload_rgba(const PoolView& P, const ImageDesc& im, int img, const uint32_t* rgba,
                       const int32_t* excess, const int32_t* tab, int lambda, int32_t* tl,
                       ImageAcc* acc, cudaStream_t s);
// tab[0..50) from the |dI|^2 sum (device) and the number of 4-neighbour pairs
int launch_nlink_table(const unsigned long long* sum, long long npairs, int32_t* tab,
                       cudaStream_t s);
int launch_dsum(const uint32_t* rgba, int W, int H, unsigned long long* sum, int sms,
                cudaStream_t s);
int launch_discharge(const PoolView& P, int iters, int grid, cudaStream_t s);
int launch_edge_relabel_build(const PoolView& P, int32_t* list, int32_t* count,
                              const ScanState& st, cudaStream_t s);
// h: condition of the enclosing WHILE node of a CUDA graph (0 outside graphs).
// first: 0 frontier round, 1 first round over every tile, 2 first round over the tiles of
// images that still had active tiles at the previous check.
int launch_bfs_round(const PoolView& P, int first, cudaGraphConditionalHandle h, int grid,
                     cudaStream_t s);
// mode: 0 frontier round, 1 first round over every tile, 2 first round over the tiles of the
// images live in this cycle; abort_hit: frontier rounds skip images that reached a sink
// check >= 0: the round that ends the flood also runs the flood check (its `all`), with the
// IF / WHILE handles of launch_flood_check; publish: a check that finds no image left writes
// the results to the handle's pinned host block (the graph solve ends there)
int launch_flood_round(const PoolView& P, int mode, int abort_hit, cudaGraphConditionalHandle h,
                       ImageAcc* acc, int grid, cudaStream_t s, int check = -1,
                       cudaGraphConditionalHandle hbfs = 0, cudaGraphConditionalHandle hmain = 0,
                       int publish = 0);
// retires the images whose flood reached no sink; all: every image takes part
int launch_flood_check(const PoolView& P, int all, cudaGraphConditionalHandle hbfs,
                       cudaGraphConditionalHandle hmain, cudaStream_t s);
int launch_ctl_begin(const PoolView& P, int max_rounds, int max_cycles, ImageAcc* acc,
                     cudaStream_t s);
// over the solve's selected tiles; filter 1: only tiles of the images a flood check kept
// (img_live == the cycle stamp), 2: those and the tiles of freshly uploaded images; grid:
// most CTAs (a few per SM), which loop over the selection's chunks
int launch_active_list(const PoolView& P, const ScanState& st, int32_t* list, int32_t* count,
                       int bump, int count_cycle, int filter, cudaGraphConditionalHandle h,
                       ImageAcc* acc, int grid, cudaStream_t s);
// launch_ctl_begin followed by the first launch_active_list (filter 2, no flood before it) in
// one single-CTA launch, for pools of at most begin_list_max_tiles() tiles
int begin_list_max_tiles();
int launch_begin_list(const PoolView& P, int max_rounds, int max_cycles, ImageAcc* acc,
                      int32_t* list, int32_t* count, cudaGraphConditionalHandle h, cudaStream_t s);
int launch_acc_reset(ImageAcc* acc, int n, cudaStream_t s);
int launch_ctl_cycle(const PoolView& P, const int32_t* count, int count_cycle,
                     cudaGraphConditionalHandle h, cudaStream_t s);
// neighbour ids and image index of the tiles of image img (a session-pool slot)
int launch_image_tiles(const PoolView& P, const ImageDesc& im, int img, cudaStream_t s);
// Inside a solve graph that ends with the labels: first = 1 for the launch after the first
// cycle's flood (it writes only when that cycle ended the solve); slot: the device word that
// holds the output buffer (out is then ignored); grid_cap > 0 caps the CTAs.
int launch_labels_out(const PoolView& P, const ImageDesc& im, uint8_t* out, cudaStream_t s,
                      int first = 0, const unsigned long long* slot = nullptr, int grid_cap = 0);
int launch_labels_packed(const PoolView& P, const ImageDesc& im, uint8_t* out, cudaStream_t s,
                         int first = 0, const unsigned long long* slot = nullptr,
                         int grid_cap = 0);
int launch_state_out(const PoolView& P, const ImageDesc& im, const int32_t* plane,
                     int32_t* out, cudaStream_t s);
int launch_edit(const PoolView& P, const ImageDesc& im, int img, const int32_t* idx,
                const int32_t* val, int n, int32_t* tl, ImageAcc* acc, cudaStream_t s);
// pts_dev / pts_host: the same (x, y) pairs on the device and on the host (for the bounds).
int launch_stroke(const PoolView& P, const ImageDesc& im, int img, const int32_t* pts_dev,
                  const int32_t* pts_host, int npts, int radius, int32_t value, int32_t* tl,
                  ImageAcc* acc, cudaStream_t s);
// The reference brush's pixel set (gc_edit_brush); radius <= 0 counts as 1; GC_ERR_INVALID
// above 1024.
int launch_brush(const PoolView& P, const ImageDesc& im, int img, const int32_t* pts_dev,
                 const int32_t* pts_host, int npts, int radius, int32_t value, int32_t* tl,
                 ImageAcc* acc, cudaStream_t s);
// Loads every kernel of the library on the current device (once per device; called by the
// first handle creation and the first stand-alone primitive on a device).
void preload_kernels();
void preload_scan_kernels();
// gc_view_colorize; ramp9: range lo, hi, hue lo, hi, saturation lo, hi, value lo, hi, opacity
int launch_view_colorize(const int32_t* values, int values_w, int values_h, int cell_w,
                         int cell_h, int width, int height, const float* ramp9,
                         const uint32_t* base, uint32_t* out, cudaStream_t s);
int occupancy_discharge(int device);
int occupancy_warps(int device);

}  // namespace gcut
