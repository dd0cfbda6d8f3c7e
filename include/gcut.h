/* gcut.h - C ABI of the sm_100a tiled push-relabel graph cut (libgcut.so).
 *
 * Drop-in boundary for the path GraphCut.pyx -> graphcut.cl of rheiland/cl-util, with the
 * IncrementalTileList / StreamCompact / PrefixSum layer beneath it.  Plain C types only:
 * device buffers are passed as pointers, streams as `void*` (a cudaStream_t, NULL for the
 * legacy default stream).  Every function returns a status code (GC_OK == 0); no C++
 * exception crosses the boundary.  gc_last_error() describes the last failure of the
 * calling thread.
 *
 * Graph convention (all int32, row-major [height][width], pitch = width):
 *   up[y][x]    residual capacity of the edge (x,y) -> (x,y-1)
 *   down[y][x]  ... (x,y) -> (x,y+1)
 *   left[y][x]  ... (x,y) -> (x-1,y)
 *   right[y][x] ... (x,y) -> (x+1,y)
 *   excess[y][x] signed t-link: > 0 source capacity, < 0 sink capacity.
 * Capacities pointing out of the image are ignored (treated as 0), as the reference zeroes
 * them (graphcut.cl:1107-1108, 1125-1127).  Capacities must be >= 0; every value must
 * satisfy |excess| + 4 * max(cap(u->v) + cap(v->u)) < 2^31.
 *
 * Result: the max-flow value (int64) and the canonical minimum cut, i.e. the set of pixels
 * reachable from the source in the final residual graph (label 1), which is unique for a
 * given graph.  The reference exposes neither directly: GraphCut.cut mutates dExcess and
 * leaves BFS distances in dHeight (GraphCut.pyx:348-418).
 */
#ifndef GCUT_H
#define GCUT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define GC_OK 0
#define GC_ERR_INVALID 1        /* bad argument (sizes, null pointers, negative capacity) */
#define GC_ERR_OOM 2            /* device allocation failed */
#define GC_ERR_NOT_CONVERGED 3  /* iteration cap reached before the cut was final */
#define GC_ERR_CUDA 4           /* a CUDA call failed */
#define GC_ERR_INTERNAL 5       /* a bounded device-side wait gave up */
#define GC_ERR_STATE 6          /* call out of order (e.g. labels before a solve) */

/* Stamp predicates of IncrementalTileList (IncrementalTileList.pyx:26-35). */
#define GC_OPERATOR_EQUAL 0
#define GC_OPERATOR_GT 1
#define GC_OPERATOR_LT 2
#define GC_OPERATOR_GTE 3
#define GC_OPERATOR_LTE 4
#define GC_LOGICAL_AND 0
#define GC_LOGICAL_OR 1

typedef struct gc_opts {
  int device;              /* CUDA device ordinal */
  int discharge_iters;     /* push + interior-relabel iterations inside a tile per launch */
  int pulses_per_relabel;  /* discharge launches between global relabels, >= 1 (reference:
                              bfs=5 push iterations, GraphCut.pyx:27) */
  int initial_relabel;     /* 1: exact global relabel before the first push; 0: start from
                              heights 0 (sink pixels) / 1 (others) */
  int max_cycles;          /* cap on global-relabel cycles; exceeded -> GC_ERR_NOT_CONVERGED */
  int max_bfs_rounds;      /* cap on tile rounds of one BFS / flood fill */
  int use_graph;           /* 1: the solve is one CUDA-graph launch whose loops are WHILE nodes
                              decided on the device (one host wait per solve); 0: the host
                              drives the loops (used when profiling is on) */
} gc_opts;

typedef struct gc_stats {
  int64_t cycles;          /* global-relabel cycles of the last solve */
  int64_t pulses;          /* discharge launches */
  int64_t bfs_rounds;      /* tile rounds over all global relabels */
  int64_t flood_rounds;    /* tile rounds of the canonical-cut flood fill */
  int64_t launches;        /* kernels launched by the last solve */
  int64_t tiles_discharged;/* sum over pulses of the active-list length (host-visible
                              only when stats collection is on) */
} gc_stats;

typedef struct gc_handle gc_handle;

/* Fills opts with defaults. */
int gc_opts_default(gc_opts* opts);

/* One solver for one width x height grid (any size >= 1; padded internally to 32).
   Replaces GraphCut.__init__ (GraphCut.pyx:80-154). */
int gc_create(int width, int height, const gc_opts* opts, gc_handle** out);
int gc_destroy(gc_handle* h);

/* Bytes of device memory a width x height handle keeps (its arena: tile planes, masks,
   flags, label staging).  Host-only computation, no device needed. */
int gc_arena_bytes(int width, int height, int64_t* bytes);
/* gc_create inside caller-owned device memory: `arena` (256-byte aligned, at least
   gc_arena_bytes bytes, on opts->device) holds every device buffer of the handle, so
   creating and destroying handles allocates and frees no device memory (gc_upload_host
   alone allocates its staging on first use).  A server that sub-allocates one HBM region
   between sessions uses this to keep cudaMalloc / cudaFree, which synchronise the device,
   off its request path.  gc_destroy waits for the work of the handle's last call (on that
   call's stream), after which the caller may reuse the memory.  No counterpart in the
   reference (GraphCut.__init__ allocates its buffers, GraphCut.pyx:117-154). */
int gc_create_in(int width, int height, const gc_opts* opts, void* arena, int64_t bytes,
                 gc_handle** out);
int gc_size(const gc_handle* h, int* width, int* height);

/* Capacity upload from DEVICE buffers (row-major, see above).  Replaces init_gc +
   load_tiles (graphcut.cl:63-112, 1033-1132), which built n-links from an image.
   Resets the residual graph to these capacities. */
int gc_upload(gc_handle* h, const int32_t* up, const int32_t* down, const int32_t* left,
              const int32_t* right, const int32_t* excess, void* stream);
/* Same from HOST buffers (copied through a pinned staging buffer owned by the handle).
   Synchronous with respect to the host buffers. */
int gc_upload_host(gc_handle* h, const int32_t* up, const int32_t* down, const int32_t* left,
                   const int32_t* right, const int32_t* excess, void* stream);

/* Capacities built on the device from an image, as the reference builds its n-links in
   load_tiles from the RGBA image it was given (graphcut.cl:1033-1132, GraphCut.pyx:80-116):
   the n-link between 4-neighbours i, j is floor(50 * exp(-beta * |I_i - I_j|^2) + 0.5) with
   |.|^2 over R, G, B and beta = 1 / (2 * mean |dI|^2) over all 4-neighbour pairs (0 for a
   uniform image); t-links are the int32 excess plane (positive: source).  rgba: DEVICE
   uint32 [height][width], R in bits 0-7, G 8-15, B 16-23 (alpha ignored), i.e. RGBA bytes
   viewed as uint32 (test_GraphCut.py:21); excess: DEVICE int32 [height][width].  Replaces
   the 20 bytes per pixel of gc_upload with 8.  The scale beta is computed on the device
   (no host wait): the call only enqueues work on the stream. */
int gc_upload_rgba(gc_handle* h, const uint32_t* rgba, const int32_t* excess, void* stream);
/* Same with HOST arrays (copied through a device staging buffer; synchronous). */
int gc_upload_rgba_host(gc_handle* h, const uint32_t* rgba, const int32_t* excess,
                        void* stream);
/* Capacities from an image with the reference's own n-link rule: GraphCut(context, devices,
   dImg, lamda) (GraphCut.pyx:80-116) weighs the edge between 4-neighbours i, j as
   LAMBDA / (BETA * sqrt(|I_i - I_j|^2) + EPSILON) with BETA = 0.1, EPSILON = 0.05 and
   LAMBDA = lamda (60 by default) in float (weight(), graphcut.cl:1018-1031; load_tiles
   :1033-1132).  Here the capacity is that value rounded to the nearest integer (halves up),
   computed exactly: floor(x + 0.5) >= k  <=>  b = 40 lambda - 2k + 1 >= 0 and
   4 (2k - 1)^2 d <= b^2, for d = |I_i - I_j|^2.  It differs from the reference's float32
   value by at most 0.5 plus float rounding.  The reference's load_tiles bugs (assigning
   instead of adding the last row/column, zeroing the right boundary in the last tile only)
   are not reproduced: every pair gets the weight both ways and capacities out of the image
   are 0.  1 <= lambda <= GC_NLINK_MAX_LAMBDA.  Layouts as gc_upload_rgba; no host wait. */
#define GC_NLINK_MAX_LAMBDA 1000
int gc_upload_rgba_lambda(gc_handle* h, const uint32_t* rgba, const int32_t* excess,
                          int32_t lambda, void* stream);
/* Same with HOST arrays (synchronous). */
int gc_upload_rgba_lambda_host(gc_handle* h, const uint32_t* rgba, const int32_t* excess,
                               int32_t lambda, void* stream);

/* One Gaussian component of a colour model, in the form its log-density is evaluated in:
   log(w N(x | mean, S)) = c - 0.5 * |Li (x - mean)|^2 for the pixel colour x = (R, G, B),
   with Li the inverse of the lower Cholesky factor of S (lower triangle, row-major: Li00,
   Li10, Li11, Li20, Li21, Li22) and c = log w - 0.5 * (3 log 2pi + log det S).  A diagonal
   model (the reference's, GMM.calcA_cpu GMM.pyx:375-395) has Li = diag(1 / sqrt(S_ii)). */
typedef struct gc_gauss {
  double c;
  double mean[3];
  double li[6];
} gc_gauss;
#define GC_GMM_MAX_COMPONENTS 8 /* MAX_NCOMPONENT of gmm.cl:4-5 */

/* T-links from a foreground and a background colour model, on the device.  The reference
   scores every pixel under each mixture (GMM.score, GMM.pyx:130-163; score_buf and
   score_img2d, gmm.cl:373-491: s = -log sum_k exp(e_k)) and gives the solver
   excess = scoreBg - scoreFg (test_GraphCut.py:44-47).  Here both scores, the difference
   and the int32 rounding are one pass:
     excess = clamp(floor(scale * (s_bg - s_fg) + 0.5), -clamp, clamp)
   with s = -(m + log(sum_k exp(e_k - m))), m = max_k e_k, the sum over k = 0, 1, ... in
   turn, and for each component d_j = x_j - mean_j, y0 = Li00 d0, y1 = Li10 d0 + Li11 d1,
   y2 = (Li20 d0 + Li21 d1) + Li22 d2, e = c - 0.5 * ((y0 y0 + y1 y1) + y2 y2): float64,
   every add and multiply rounded on its own (no fused multiply-add), in that order.
   - rgba: DEVICE uint32, row y at rgba + y * pitch (pitch >= width, in pixels), R in bits
     0-7, G 8-15, B 16-23; excess: DEVICE int32 [height][width] (row-major, dense).
   - 1 <= n_fg, n_bg <= GC_GMM_MAX_COMPONENTS; every parameter finite with |c| <= 2^64,
     |mean| <= 2^32, |li| <= 2^32; |scale| <= 2^32; 0 <= clamp <= 2^30.  Otherwise
     GC_ERR_INVALID.  width or height 0 is a no-op.
   - The result equals a float64 host evaluation of the same expression except where the
     host's and the device's exp / log differ in the last bit and that moves
     scale * (s_bg - s_fg) + 0.5 across an integer (then the two differ by 1).
   - Pass excess to gc_upload_rgba with the same image to build the whole graph on the
     device from 4 bytes per pixel. */
int gc_tlinks_gmm(const uint32_t* rgba, int width, int height, int pitch, const gc_gauss* fg,
                  int n_fg, const gc_gauss* bg, int n_bg, double scale, int32_t clamp,
                  int32_t* excess, void* stream);

/* Result of gc_gmm_fit (written to DEVICE memory). */
typedef struct gc_gmm_fit_result {
  double weights[GC_GMM_MAX_COMPONENTS];
  double means[GC_GMM_MAX_COMPONENTS][3];
  double covars[GC_GMM_MAX_COMPONENTS][6]; /* lower triangle: S00, S10, S11, S20, S21, S22 */
  double log_likelihood;  /* sum over the samples of log p(x) under the returned model */
  int32_t iterations;     /* EM iterations run */
  int32_t converged;      /* 1: the likelihood test stopped the loop before max_iterations */
  int32_t status;         /* 0; 1: a covariance stopped being positive definite */
  int32_t n_components;
  /* the returned model in the form gc_tlinks_gmm takes (all zero when status is 1); leave
     out components of weight 0, whose c is -infinity */
  gc_gauss components[GC_GMM_MAX_COMPONENTS];
} gc_gmm_fit_result;

/* Colour-model fit on the device: GMM.fit (GMM.pyx:165-372; initA, em1, em2, eval and
   check_converge, gmm.cl:33-372), in float64.
   - samples: DEVICE uint32 [n] RGBA words (R in bits 0-7, G 8-15, B 16-23), n >= n_components.
   - Start (initA): weights 1/K; mean_k = the colour of sample k * (n - 1) / (K - 1) (integer
     division; sample 0 when K = 1); covariance init_covar * I.
   - Iteration: responsibilities r_k(x) = w_k N(x | mean_k, S_k) / p(x) under the current
     model; N_k = sum r_k; w_k = N_k / sum_j N_j; mean_k = sum r_k x / N_k;
     S_k = sum r_k x x^T / N_k - mean_k mean_k^T + min_covar * I, off-diagonal terms set to 0
     unless full_covariance.  A component whose N_k is 0 keeps its mean and covariance with
     weight 0.
   - Stop: L_i, the log-likelihood of the samples under the model of iteration i, is
     evaluated after each iteration; for i > 1 the loop stops when |L_i - L_{i-1}| < tolerance
     (the reference uses 0.01), else after max_iterations.
   - 1 <= n_components <= GC_GMM_MAX_COMPONENTS, 1 <= max_iterations <= 100000, tolerance,
     min_covar >= 0 and init_covar > 0 finite; otherwise GC_ERR_INVALID.
   - One launch of one thread-block cluster whose blocks add their sums through distributed
     shared memory in a fixed order, so results are deterministic; they equal a float64 host
     evaluation of the same steps up to rounding.  *result is complete when the stream
     reaches the end of the call; result->status 1 means the fit stopped early. */
int gc_gmm_fit(const uint32_t* samples, int n, int n_components, int max_iterations,
               double tolerance, double min_covar, double init_covar, int full_covariance,
               gc_gmm_fit_result* result, void* stream);

/* Max-flow to the final cut.  Replaces GraphCut.cut (GraphCut.pyx:348-418); warm-starts
   from the current residual graph when called again after gc_edit_tlinks.  Blocks the
   calling host thread until the solve is done (one wait for the solve's CUDA graph; the
   host-driven path of gc_set_profile / gc_set_collect_stats reads the loop counters between
   launches). */
int gc_solve(gc_handle* h, void* stream);

/* gc_solve, then the canonical labels into the DEVICE buffer `labels` (packed != 0: the
   bit-packed rows of gc_labels_packed, else one byte per pixel as gc_labels), with one host
   wait for both: the labels kernel is queued behind the solve on `stream` instead of after
   the host has seen the solve finish.  On an error return the buffer's content is
   unspecified. */
int gc_solve_labels(gc_handle* h, uint8_t* labels, int packed, void* stream);

/* Manual stepping, mirroring the reference methods a caller can drive one at a time (the
   GUI buttons of test_GraphCut.py:81-83).  gc_push = one discharge launch over the active
   tiles (GraphCut.push, GraphCut.pyx:242-323, all four directions plus the in-tile local
   relabel); gc_relabel = relabel of active tile-edge pixels and the active-tile list
   rebuild (GraphCut.relabel, GraphCut.pyx:224-240); gc_start_bfs = exact global relabel
   and the active-tile list from it (GraphCut.startBfs, GraphCut.pyx:187-222);
   gc_is_completed = 1 when no pixel with excess > 0 can reach a sink pixel, valid right
   after gc_start_bfs (GraphCut.isCompleted, GraphCut.pyx:328-346); it also computes the
   canonical cut and the flow when it returns 1. */
int gc_push(gc_handle* h, void* stream);
int gc_relabel(gc_handle* h, void* stream);
int gc_start_bfs(gc_handle* h, void* stream);
int gc_is_completed(gc_handle* h, int* completed, void* stream);

/* Flow value of the last solve (int64). */
int gc_flow(gc_handle* h, int64_t* flow);
/* Canonical labels (1 = source side) into a DEVICE buffer [height][width] uint8. */
int gc_labels(gc_handle* h, uint8_t* labels, void* stream);
/* Same into a HOST buffer (synchronous). */
int gc_labels_host(gc_handle* h, uint8_t* labels, void* stream);
/* Canonical labels bit-packed, one row of (width + 7) / 8 bytes per image row, pixel x in
   bit x % 8 of byte x / 8 (numpy.packbits(labels, axis=1, bitorder="little")); unused
   bits of a row's last byte are 0.  The serving loop returns these: 8x fewer bytes to
   read back than gc_labels.  No counterpart in the reference (its cut stays on the
   device as a float mask).  DEVICE buffer of height * ((width + 7) / 8) bytes. */
int gc_labels_packed(gc_handle* h, uint8_t* bits, void* stream);
/* Same into a HOST buffer (synchronous). */
int gc_labels_packed_host(gc_handle* h, uint8_t* bits, void* stream);

/* Sets the signed t-link of n pixels (flat indices y*width+x, DEVICE arrays) to value[i];
   the excess changes by value - previous t-link, which warm-starts the next gc_solve from
   the previous flow.  Indices must be distinct within one call. */
int gc_edit_tlinks(gc_handle* h, const int32_t* idx, const int32_t* value, int n, void* stream);
/* Stroke edit: every pixel within `radius` of the polyline (xs[i], ys[i]), i < npts (host
   arrays, integer pixel centres) gets t-link `value`.  Rasterised on the device. */
int gc_edit_stroke(gc_handle* h, const int32_t* xs, const int32_t* ys, int npts, int radius,
                   int32_t value, void* stream);

/* Brush edit with the reference's own pixel set (Brush.points, brush.pyx:138-161): for one
   point, the disc skimage.draw.circle(y, x, radius) around it; for a polyline, the Bresenham
   pixels of every segment (skimage.draw.line) each widened by that disc, whose offsets
   (dy, dx) satisfy (dy / radius)^2 + (dx / radius)^2 < 1 in float64.  Every covered pixel
   gets t-link `value` (the reference paints label 7 there, brush.cl:1-13).  radius <= 0
   counts as 1, as Brush.setRadius does; radius <= 1024, 1 <= npts <= 1024 (host arrays).
   Two reference bugs are not reproduced: the reference widens segments by
   circle(radius, radius, radius), a disc shifted by +radius in x and y, where this centres
   it on the line; and it flattens pixels outside the image into y * width + x (wrapping
   into other rows), where this skips them. */
int gc_edit_brush(gc_handle* h, const int32_t* xs, const int32_t* ys, int npts, int radius,
                  int32_t value, void* stream);

/* Residual state back to row-major DEVICE buffers (any pointer may be NULL): excess,
   height, residual capacities.  Inspection and tests. */
int gc_download_state(gc_handle* h, int32_t* excess, int32_t* height, int32_t* up,
                      int32_t* down, int32_t* left, int32_t* right, void* stream);
int gc_get_stats(const gc_handle* h, gc_stats* stats);
/* Per-pulse host readback of the active-tile count (diagnostics; slows the solve). */
int gc_set_collect_stats(gc_handle* h, int on);

/* Per-kernel profile of the last solve (and the upload / labels calls around it):
   launches, summed CUDA-event time of each launch on the caller's stream, and tiles
   processed (device counters).  Kinds 0..GC_NKERN-1, named by gc_kernel_name. */
#define GC_NKERN 10
typedef struct gc_kernel_prof {
  int64_t launches;
  double ms;
  int64_t tiles;
} gc_kernel_prof;
int gc_set_profile(gc_handle* h, int on);
int gc_get_profile(const gc_handle* h, gc_kernel_prof* out, int n);
const char* gc_kernel_name(int kind);

/* Device-side trace of the solves, for looking inside a CUDA-graph solve (whose kernels a
   host profiler does not list): while on, the first thread of every solver kernel appends
   (start time in ns of the GPU's global timer, kind) to a buffer of GC_TRACE_MAX entries in
   the handle's memory; the difference of consecutive start times is a kernel's duration
   including its launch.  Kinds: 0 solve start, 1 active-tile list, 2 discharge, 3 mask
   rebuild, 4 flood first round, 5 flood round, 6 flood check, 7 BFS first round, 8 BFS
   round, 9 upload, 10 labels, 11 solve end.  gc_set_trace turns it on or off and empties
   the buffer; gc_get_trace copies up to max_entries entries (two uint64 each) and sets *n
   to the number written since (it may exceed the buffer).  Both synchronise `stream`.
   The kernels take the trace as an argument, so an untraced solve pays nothing for it;
   switching it on or off therefore rebuilds the solve's CUDA graph at the next solve (one
   graph instantiation; calling gc_set_trace again with the same state only empties the
   buffer).  No counterpart in the reference (its host loop timed kernels with OpenCL
   events). */
#define GC_TRACE_MAX 2048
int gc_set_trace(gc_handle* h, int on, void* stream);
int gc_get_trace(gc_handle* h, uint64_t* entries, int max_entries, int* n, void* stream);

/* Message of the last error on this thread ("" if none). */
const char* gc_last_error(void);

/* ---- data-parallel primitives beneath IncrementalTileList ---------------------------
   All pointers are DEVICE pointers; n items; one launch each.

   Each primitive runs on a look-back state (the single-pass scan's tickets, per-chunk status
   words, launch tag and error word).  The reference gives every tile list its own
   StreamCompact and PrefixSum (IncrementalTileList.pyx:74, StreamCompact.pyx:39,
   PrefixSum.pyx:46); the counterpart here is one gc_scan_state per such object.  Calls on
   one state must not overlap on the GPU (one stream per state, or host ordering); calls on
   different states never interfere.  A NULL state selects one state shared by every caller
   on the current device: calls on it from different streams must not overlap either.

   Errors found on the device (a bounded look-back wait that gave up, an out-of-range
   scatter index) set the state's error word, which stays set until reported:
   - compactions (gc_compact, gc_tiles_build, gc_tiles_build_logical) then write length -1;
   - the next call on the state returns GC_ERR_INTERNAL once the word has reached the host
     (it is copied back after every launch, on the caller's stream);
   - gc_scan_state_error reads it synchronously. */
typedef struct gc_scan_state gc_scan_state;
/* A state for launches of up to max_items items on `device`.  No counterpart in the
   reference (the objects above own their buffers). */
int gc_scan_state_create(int device, int max_items, gc_scan_state** out);
/* Waits for the state's last launch, then frees it. */
int gc_scan_state_destroy(gc_scan_state* state);
/* *err = the state's error word (0 none, 1 a look-back wait gave up, 2 a scatter index was
   out of range), then clears it.  Synchronises `stream`. */
int gc_scan_state_error(gc_scan_state* state, int* err, void* stream);
/* Diagnostic of the bounded wait: one warp waits, with a limit of `spins` polls, for a
   look-back predecessor that never publishes, gives up, and records error 1.  With err
   non-NULL, *err gets the error word as gc_scan_state_error reads it (1 when the wait ran
   out as designed); with err NULL the word is left on the state and reported like any
   device error (the next call on the state returns GC_ERR_INTERNAL).  The state stays
   usable. */
int gc_scan_state_selftest(gc_scan_state* state, int spins, int* err, void* stream);

/* PrefixSum.scan (PrefixSum.pyx:83-129, prefixsum.cl): exclusive scan of in[0..n) into
   out (may alias in) and the sum into *total (int32 wrap-around). */
int gc_scan_exclusive(gc_scan_state* state, const int32_t* in, int32_t* out, int32_t* total,
                      int n, void* stream);
/* StreamCompact.compact (StreamCompact.pyx:66-82, streamcompact.cl): indices i with
   flags[i] != 0, increasing, into list; their number into *length.  list must not alias
   flags. */
int gc_compact(gc_scan_state* state, const int32_t* flags, int32_t* list, int32_t* length,
               int n, void* stream);
/* IncrementalTileList.build(operator, operand) (IncrementalTileList.pyx:119-136,
   incremental_tile_list.cl:40-64 + compaction). */
int gc_tiles_build(gc_scan_state* state, const int32_t* tiles, int op, int32_t operand,
                   int32_t* list, int32_t* length, int n, void* stream);
/* Same compaction as gc_compact for callers that cannot allocate device memory.  No
   counterpart in the reference.  gc_compact keeps its look-back scratch in a gc_scan_state,
   whose device memory comes from cudaMalloc (in gc_scan_state_create, or on the first call
   on a device for the shared NULL state); code that must keep a fixed device-memory
   footprint (for example a serving process with a pre-divided budget on a shared GPU) or
   that cannot risk the implicit synchronisation of cudaMalloc/cudaFree while other work
   runs, calls this variant instead.  Its scratch is a fixed 8208-byte array compiled into
   the library, present on every GPU that loads the library until the process exits; it
   calls no cudaMalloc, cudaFree or allocating library routine.
   - n must not exceed GC_COMPACT_NOALLOC_MAX_N (4194304 items); larger n returns
     GC_ERR_INVALID.
   - The first call on each device looks up the array's device address and loads the
     library's kernels (with that device current); make that first call before any stream
     capture.
   - All calls share the one array and each call clears the part it uses, so calls whose
     work overlaps on the GPU (different streams, or different host threads) race and must
     be serialised by the caller.
   - A look-back wait that gives up is reported in the result: *length is -1. */
#define GC_COMPACT_NOALLOC_MAX_N 4194304
int gc_compact_noalloc(const int32_t* flags, int32_t* list, int32_t* length, int n, void* stream);
/* IncrementalTileList.buildLogical (IncrementalTileList.pyx:157-176,
   incremental_tile_list.cl:66-108 + compaction). */
int gc_tiles_build_logical(gc_scan_state* state, const int32_t* tiles, const int32_t* tiles2,
                           int op1, int32_t a1, int op2, int32_t a2, int logical, int32_t* list,
                           int32_t* length, int n, void* stream);
/* IncrementalTileList.incorporate (IncrementalTileList.pyx:138-155,
   incremental_tile_list.cl:110-154): tiles[i] = iteration where the predicate holds. */
int gc_tiles_incorporate(int32_t* tiles, const int32_t* tiles2, int op1, int32_t a1, int op2,
                         int32_t a2, int logical, int32_t iteration, int n, void* stream);
/* IncrementalTileList.reset (IncrementalTileList.pyx:178-189, init_incremental
   incremental_tile_list.cl:26-38): tiles[i] = value. */
int gc_tiles_fill(int32_t* tiles, int32_t value, int n, void* stream);
/* IncrementalTileList.execute (IncrementalTileList.pyx:191-208; filter,
   incremental_tile_list.cl:156-175), the tile-list display layer without a graphics stack:
   out[y * width + x] = 0xFF0000FF (opaque red, R in the low byte) where
   tiles[(y / tile_h) * tiles_w + x / tile_w] == iteration, else 0xFF000000.  tiles: DEVICE
   int32 [tiles_h][tiles_w]; out: DEVICE uint32 [height][width].  Pixels outside the
   tiles_w x tiles_h tile grid are black (the reference reads past its tile array there). */
int gc_tiles_view(const int32_t* tiles, int tiles_w, int tiles_h, int tile_w, int tile_h,
                  int32_t iteration, int width, int height, uint32_t* out, void* stream);
/* The reference's display filters without a graphics stack (graphcut_filter.cl:5-155:
   colorizef, HSVtoRGB, and the tranpose / tilelist / tilelist_growcut kernels that paint a
   plane or a tile map over the displayed image).  Pixel (x, y) of the width x height output
   takes v = values[(y / cell_h) * values_w + x / cell_w] (1 x 1 cells: a pixel plane such as
   GraphCut's heights; the tile size: a tile map), converted to float.
   - ramp (HOST, 9 floats, all finite): range lo, hi; hue lo, hi; saturation lo, hi; value lo,
     hi; opacity.
   - Colour: black for v < lo, white for v > hi; inside the range, hue, saturation and value
     run linearly from their lo to their hi ends (t = (v - lo) / (hi - lo), 0 when hi == lo),
     then HSV -> RGB by the hue sectors of the reference's HSVtoRGB (its sector 4 repeats
     sector 5's (v, p, q), and so does this one). Its alpha is 0, as the reference's. The
     reference's double literals (1.0, 0.000001) are taken as float here.
   - out = base + (colour - base) * opacity per channel, channels read as byte / 255; float32
     arithmetic, rounded to the nearest byte, ties to even. base may be NULL (all zero).
   - Pixels outside the values_w x values_h cell grid keep the base.
   values, base, out: DEVICE; base and out are RGBA words, R in the low byte. */
int gc_view_colorize(const int32_t* values, int values_w, int values_h, int cell_w, int cell_h,
                     int width, int height, const float* ramp, const uint32_t* base,
                     uint32_t* out, void* stream);

/* ---- batched solver: many independent grids in one tile pool ------------------------ */
typedef struct gcb_handle gcb_handle;
int gcb_create(int n, const int* widths, const int* heights, const gc_opts* opts,
               gcb_handle** out);
int gcb_destroy(gcb_handle* b);
/* Upload grid i from DEVICE buffers (layout as gc_upload). */
int gcb_upload(gcb_handle* b, int i, const int32_t* up, const int32_t* down,
               const int32_t* left, const int32_t* right, const int32_t* excess, void* stream);
/* Solves every grid of the pool together (one tile queue over all grids). */
int gcb_solve(gcb_handle* b, void* stream);
int gcb_flow(gcb_handle* b, int i, int64_t* flow);
int gcb_labels(gcb_handle* b, int i, uint8_t* labels, void* stream);
int gcb_get_stats(const gcb_handle* b, gc_stats* stats);
int gcb_set_profile(gcb_handle* b, int on);
int gcb_get_profile(const gcb_handle* b, gc_kernel_prof* out, int n);
int gcb_set_trace(gcb_handle* b, int on, void* stream);
int gcb_get_trace(gcb_handle* b, uint64_t* entries, int max_entries, int* n, void* stream);

/* ---- session pools: many resident images, solved together a few at a time ------------
   A pool of max_tiles 32x32 tiles and max_sessions image slots in one arena.  An image
   (a serving session) opens on a slot with a caller-chosen range of tiles, keeps its
   residual graph there between requests, and any set of slots is solved together by one
   launch of the pool's CUDA graph; the other slots keep their state and results.  The graph
   is built on the pool's first solves (one for solves of fresh uploads only, one when some
   slot continues from a previous flow), so requests never wait for a graph construction.
   No counterpart in the reference (one GraphCut object per image, GraphCut.pyx:80-154).
   One caller thread and one stream per pool at a time. */
typedef struct gcp_handle gcp_handle;
/* Device bytes of a pool (host-only computation). */
int gcp_arena_bytes(int max_tiles, int max_sessions, int64_t* bytes);
int gcp_create(int max_tiles, int max_sessions, const gc_opts* opts, gcp_handle** out);
/* In caller-owned device memory (256-byte aligned, at least gcp_arena_bytes bytes). */
int gcp_create_in(int max_tiles, int max_sessions, const gc_opts* opts, void* arena,
                  int64_t bytes, gcp_handle** out);
int gcp_destroy(gcp_handle* p);
/* Opens slot `slot` for a width x height image on tiles [tile0, tile0 + ceil(W/32) *
   ceil(H/32)) of the pool, which must not overlap another open slot's. */
int gcp_open(gcp_handle* p, int slot, int width, int height, int tile0, void* stream);
/* Closes a slot; its tiles may be given to another slot. */
int gcp_close(gcp_handle* p, int slot);
/* Uploads and edits of one slot, as gc_upload / gc_upload_rgba / gc_edit_stroke /
   gc_edit_brush do for a handle. */
int gcp_upload(gcp_handle* p, int slot, const int32_t* up, const int32_t* down,
               const int32_t* left, const int32_t* right, const int32_t* excess, void* stream);
int gcp_upload_rgba(gcp_handle* p, int slot, const uint32_t* rgba, const int32_t* excess,
                    void* stream);
int gcp_edit_stroke(gcp_handle* p, int slot, const int32_t* xs, const int32_t* ys, int npts,
                    int radius, int32_t value, void* stream);
int gcp_edit_brush(gcp_handle* p, int slot, const int32_t* xs, const int32_t* ys, int npts,
                   int radius, int32_t value, void* stream);
/* Solves the n listed slots (distinct, open, uploaded) together: one graph launch; a slot
   uploaded since its last solve starts fresh, an edited or solved one warm-starts from its
   previous flow.  Blocks the calling thread until the solve is done. */
int gcp_solve(gcp_handle* p, const int* slots, int n, void* stream);
/* gcp_solve, then every listed slot's labels into the DEVICE buffer labels[k] (packed as in
   gc_solve_labels), with one host wait for the solve and all the labels. */
int gcp_solve_labels(gcp_handle* p, const int* slots, int n, uint8_t* const* labels, int packed,
                     void* stream);
int gcp_flow(gcp_handle* p, int slot, int64_t* flow);
/* Canonical labels of a slot's last solve into DEVICE buffers (as gc_labels /
   gc_labels_packed). */
int gcp_labels(gcp_handle* p, int slot, uint8_t* labels, void* stream);
int gcp_labels_packed(gcp_handle* p, int slot, uint8_t* bits, void* stream);
int gcp_get_stats(const gcp_handle* p, gc_stats* stats);
int gcp_set_trace(gcp_handle* p, int on, void* stream);
int gcp_get_trace(gcp_handle* p, uint64_t* entries, int max_entries, int* n, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GCUT_H */
