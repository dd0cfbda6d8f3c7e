/* The reference's own graph-cut kernels, run on the host.  TEST INFRASTRUCTURE ONLY: the
 * parity tests and the script that writes the reference-kernel golden fixtures use it to
 * check the oracle; nothing in the product links or loads it.
 *
 * The reference's graph-cut kernels (graphcut.cl) are compiled unchanged from where they
 * lie (the Makefile passes the path as REF_GRAPHCUT_CL; the build output goes to
 * oracle/_ref/ only), with the options GraphCut.__init__ gives them (GraphCut.pyx:85-96).
 * refcl_clc.h supplies the OpenCL C built-ins, refcl_runtime.h the work-group runtime
 * (fibers switched at barrier()), and this file the host side: GraphCut.cut / push /
 * relabel / startBfs / isCompleted (GraphCut.pyx:155-418) and IncrementalTileList.reset /
 * increment / build / incorporate (IncrementalTileList.pyx:101-189), each launch with the
 * reference's own global and local sizes and argument lists.
 *
 * The tile lists' kernels (init_incremental, flag, increment_logical) are the reference's
 * too: the Makefile compiles incremental_tile_list.cl (REF_TILELIST_CL) from a copy without
 * its last kernel, `filter` (the display view, :156-175), whose OpenCL vector literals C
 * cannot parse.
 *
 * The tile lists compact with the reference's StreamCompact / PrefixSum kernels under their
 * host code (refcl_prefixsum.h).  Two things differ from the reference, both on the input
 * side:
 *   - load_tiles (graphcut.cl:1033-1132) derives float capacities from an RGBA image.
 *     Here the capacities are given as integer planes, and loading a tile adds them to the
 *     tile's residual planes: up/down as they are, left/right in the kernels' tile-transposed
 *     layout (plane row ty*32 + x', column tx*32 + y' holds pixel (tx*32 + x', ty*32 + y')).
 *     load_tiles itself adds for every edge except two that it assigns (:1104, :1130); the
 *     image-edge capacities it zeroes are zero in the given planes already.
 *   - dHeight, which the reference never clears, starts at zero; every device buffer starts
 *     at zero, inside zero-filled guard bands (the kernels read up to one image row before
 *     the first tile row and after the last).  The harness reports a guard band that no
 *     longer holds zero, and a barrier() reached by a kernel run without fibers.
 *
 * The integer planes are exact in the kernels' float32 buffers while every capacity and
 * excess stays below 2^24 in magnitude; refcl_cut refuses larger inputs and reports any
 * final value that is not a whole number.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "refcl_clc.h"

/* ---------------------------------------------------------------------------------------
 * The reference kernels.  GraphCut.__init__ (GraphCut.pyx:85-96) builds graphcut.cl with
 * MAX_HEIGHT = W * H, LAMBDA, EPSILON, TILESW and TILESH; the image size itself is fixed
 * in the source (graphcut.cl:15-16: 800 x 608).  REFCL_W / REFCL_H name the size the
 * kernels were built for: 800 x 608 for the source as it is, or the size the Makefile
 * wrote into a generated copy whose two #define lines it rewrote (nothing else changes).
 *
 * bfs_intratile keeps its loop flag in local memory (_l_didChange, graphcut.cl:925-990):
 * every work-item tests it, resets it and, when its pixels changed, sets it, with no barrier
 * between the test and the reset or between the reset and the set.  The lanes of a GPU warp
 * make each of these accesses together, so all reset before any sets.  Compiled here, the
 * flag's name stands for a call into the harness, and under the default (lockstep)
 * schedule every access to it is a scheduling point: the work-items of the group make each
 * access in turn before any makes the next -- all test, then all reset, then those that
 * changed set it.  Under the serial schedule (a CPU OpenCL runtime's order: each work-item
 * runs on until a barrier) later work-items see the flag another has reset, or reset it
 * after another set it, and the in-tile BFS ends early.  Nothing else in the kernels is
 * shared between work-items without a barrier between a write and a read.
 * ------------------------------------------------------------------------------------- */
#ifndef REFCL_W
#define REFCL_W 800
#define REFCL_H 608
#endif
#define MAX_HEIGHT (REFCL_W * REFCL_H)
#define LAMBDA 60
#define EPSILON 0.05
#define TILESW (REFCL_W / 32)
#define TILESH (REFCL_H / 32)
#define _l_didChange refcl_loop_flag()
#include REF_GRAPHCUT_CL
#undef _l_didChange

/* IncrementalTileList's kernels (IncrementalTileList.pyx:82-87 builds them with the tile
 * grid's sizes, which only the omitted `filter` kernel reads). */
#include REF_TILELIST_CL

/* StreamCompact / PrefixSum's kernels, under which IncrementalTileList.build compacts
 * (IncrementalTileList.pyx:119-136).  prefixsum.cl's helpers are C99 `inline` functions
 * without an external definition; here they become file-local. */
#define inline static inline
#include REF_PREFIXSUM_CL
#undef inline
#include REF_STREAMCOMPACT_CL

#include "refcl_runtime.h"
#include "refcl_prefixsum.h"

/* bfs_intratile's loop flag: local-memory slot 1 of its launch (intratile_gaps). */
static int* loop_flag_access(void) {
  if (R.fibers && R.lockstep) refcl_swap(&R.cur->sp, R.sched_sp);
  return (int*)R.loc[1];
}

/* ---------------------------------------------------------------------------------------
 * Kernel arguments (one set per kernel; every work-item gets the same) and the per-kernel
 * entry the runtime calls for each work-item.
 * ------------------------------------------------------------------------------------- */
#define L(T, k) ((T*)R.loc[k])
static struct {
  float *up, *down, *left, *right, *excess, *border;
  int *height, *height2;
  uint *can_up, *can_down, *can_left, *can_right;
  int* list;
  int* tiles;
  int* tiles2;
  int* flags;
  int* is_completed;
  int iteration, direction, length, op1, op2, a1, a2, logical;
  int2 dim;
} A;

static void k_init_gc(void) {
  init_gc(A.up, A.down, A.left, A.right, A.excess, L(int, 0), A.tiles, A.iteration);
}
static void k_init_bfs(void) {
  init_bfs(A.list, A.excess, L(float, 0), A.height, L(int, 1), A.down, A.up, A.right, A.left,
           A.can_down, A.can_up, A.can_right, A.can_left, L(uchar, 2), L(uchar, 3),
           L(uchar, 4), L(uchar, 5), A.tiles, A.iteration);
}
static void k_bfs_intratile(void) {
  bfs_intratile(A.list, A.height, L(int, 0), A.can_down, A.can_up, A.can_right, A.can_left,
                loop_flag_access, A.tiles, A.iteration);
}
static void k_bfs_intertile(void) {
  bfs_intertile(A.list, L(int, 0), A.height, A.can_down, A.can_up, A.can_right, A.can_left,
                A.iteration, A.tiles);
}
static void k_relabel(void) {
  relabel(A.down, A.right, A.up, A.left, A.excess, A.height, A.height2);
}
static void k_push_down(void) {
  push_down(A.list, A.down, A.up, A.height, A.excess, A.border, L(int, 0), A.tiles,
            A.iteration);
}
static void k_push_up(void) {
  push_up(A.list, A.down, A.up, A.height, A.excess, A.border, L(int, 0), A.tiles, A.iteration);
}
static void k_push_right(void) {
  push_right(A.list, A.excess, L(float, 0), A.height, L(int, 1), A.right, A.left, A.border,
             L(int, 2), A.tiles, A.iteration);
}
static void k_push_left(void) {
  push_left(A.list, A.excess, L(float, 0), A.height, L(int, 1), A.right, A.left, A.border,
            L(int, 2), A.tiles, A.iteration);
}
static void k_add_border(void) { add_border(A.list, A.border, A.excess, A.direction); }
static void k_check_completion(void) {
  check_completion(A.list, A.excess, A.height, L(int, 0), A.is_completed);
}
static void k_init_incremental(void) { init_incremental(A.tiles, A.dim, A.iteration); }
static void k_flag(void) { flag(A.tiles, A.flags, A.length, A.op1, A.a1); }
static void k_increment_logical(void) {
  increment_logical(A.tiles, A.tiles2, A.tiles, A.length, A.op1, A.op2, A.a1, A.a2, A.logical,
                    A.iteration);
}

static int round_up(int v, int m) { return (v + m - 1) / m * m; }

/* ---------------------------------------------------------------------------------------
 * Device buffers: zero-filled, inside zero-filled guard bands.
 * ------------------------------------------------------------------------------------- */
_Static_assert(IMAGEW == REFCL_W && IMAGEH == REFCL_H, "kernels built for another size");
_Static_assert(REFCL_W % 32 == 0 && REFCL_H % 32 == 0, "whole 32 x 32 tiles");
enum { WW = REFCL_W, HH = REFCL_H, TW = TILESW, TH = TILESH, NT = TILESW * TILESH, GUARD = 8 * WW };
enum { NPIX = WW * HH, NWAVE = WW * (HH / 32) };

typedef struct {
  char* base;
  size_t elem, n;
} Buf;

static Buf g_bufs[32];
static int g_nbufs;

static void* buf_new(size_t n, size_t elem) {
  if (g_nbufs >= (int)(sizeof(g_bufs) / sizeof(g_bufs[0]))) return NULL;
  Buf* b = &g_bufs[g_nbufs++];
  b->elem = elem;
  b->n = n;
  b->base = calloc(n + 2 * GUARD, elem);
  return b->base ? b->base + GUARD * elem : NULL;
}

static long long guards_dirty(void) {
  long long bad = 0;
  for (int k = 0; k < g_nbufs; ++k) {
    const Buf* b = &g_bufs[k];
    const char* lo = b->base;
    const char* hi = b->base + (GUARD + b->n) * b->elem;
    for (size_t i = 0; i < GUARD * b->elem; ++i) bad += (lo[i] != 0) + (hi[i] != 0);
  }
  return bad;
}

static void bufs_free(void) {
  for (int k = 0; k < g_nbufs; ++k) free(g_bufs[k].base);
  g_nbufs = 0;
}

/* ---------------------------------------------------------------------------------------
 * IncrementalTileList (IncrementalTileList.pyx:60-189), tile grid 25 x 19.
 * ------------------------------------------------------------------------------------- */
typedef struct {
  int *tiles, *flags, *list;
  int length, iteration;
  PrefixSum ps;  /* its StreamCompact's scan (IncrementalTileList.pyx:64-65) */
  int* d_length;
} TileList;

enum { OP_EQUAL = 0, OP_GT = 1, OP_LT = 2, OP_GTE = 3, OP_LTE = 4, LOGIC_AND = 0 };

static int tl_init(TileList* t) {
  t->tiles = buf_new(NT, sizeof(int));
  t->flags = buf_new(NT, sizeof(int));
  t->list = buf_new(NT, sizeof(int));
  t->d_length = gbuf_new(1, 1);
  if (!t->tiles || !t->flags || !t->list || !t->d_length) return 1;
  if (ps_init(&t->ps, NT)) return 1;
  /* reset(): iteration = init_iteration + 1, every stamp = init_iteration = -1 */
  t->iteration = 0;
  t->length = 0;
  A.tiles = t->tiles;
  A.dim.x = TW;
  A.dim.y = TH;
  A.iteration = -1;
  set_local(0, NULL);
  return launch(k_init_incremental, round_up(TW, 16), round_up(TH, 16), 16, 16, 0);
}

static int tl_increment(TileList* t) { return ++t->iteration; }

/* build(operator, operand): the flag kernel, then StreamCompact.compact */
static int tl_build(TileList* t, int op, int operand) {
  A.tiles = t->tiles;
  A.flags = t->flags;
  A.length = NT;
  A.op1 = op;
  A.a1 = operand;
  set_local(0, NULL);
  int rc = launch(k_flag, round_up(NT, 256), 1, 256, 1, 0);
  if (rc) return rc;
  rc = sc_compact(&t->ps, t->flags, t->list, t->d_length, NT);
  t->length = *t->d_length;
  return rc;
}

static int tl_incorporate(TileList* t, const int* tiles2, int op1, int a1, int op2, int a2,
                          int logical) {
  A.tiles = t->tiles;
  A.tiles2 = (int*)tiles2;
  A.length = NT;
  A.op1 = op1;
  A.op2 = op2;
  A.a1 = a1;
  A.a2 = a2;
  A.logical = logical;
  A.iteration = t->iteration;
  set_local(0, NULL);
  return launch(k_increment_logical, round_up(NT, 256), 1, 256, 1, 0);
}

/* ---------------------------------------------------------------------------------------
 * GraphCut (GraphCut.pyx).
 * ------------------------------------------------------------------------------------- */
typedef struct {
  float *up, *down, *left, *right, *excess, *border;
  int *height, *height2;
  uint *can_up, *can_down, *can_left, *can_right;
  int is_completed;
  TileList load, bfs, edges, brd;
  const int32_t* src[4]; /* up, down, left, right: integer capacities, row-major */
  long long iterations, relabels, bfs_rounds;
  int err;
} GC;

static void bind_planes(const GC* g) {
  A.up = g->up;
  A.down = g->down;
  A.left = g->left;
  A.right = g->right;
  A.excess = g->excess;
  A.border = g->border;
  A.height = g->height;
  A.height2 = g->height2;
  A.can_up = g->can_up;
  A.can_down = g->can_down;
  A.can_left = g->can_left;
  A.can_right = g->can_right;
}

/* Index of pixel (x, y)'s left/right capacity in the kernels' tile-transposed planes. */
static long tpos(int x, int y) {
  return (long)((y / 32) * 32 + x % 32) * WW + (x / 32) * 32 + y % 32;
}

/* In place of load_tiles (graphcut.cl:1033-1132): add the given capacities of the listed
 * tiles to their residual planes. */
static void load_listed(GC* g) {
  for (int k = 0; k < g->load.length; ++k) {
    const int t = g->load.list[k], tx = t % TW, ty = t / TW;
    for (int y = ty * 32; y < ty * 32 + 32; ++y)
      for (int x = tx * 32; x < tx * 32 + 32; ++x) {
        const long i = (long)y * WW + x;
        g->up[i] += (float)g->src[0][i];
        g->down[i] += (float)g->src[1][i];
        g->left[tpos(x, y)] += (float)g->src[2][i];
        g->right[tpos(x, y)] += (float)g->src[3][i];
      }
  }
}

static void chk(GC* g, int rc) {
  if (rc && !g->err) g->err = rc;
}

/* intratile_gaps (GraphCut.pyx:155-170) */
static void intratile_gaps(GC* g) {
  bind_planes(g);
  A.list = g->bfs.list;
  A.tiles = g->edges.tiles;
  A.iteration = tl_increment(&g->edges);
  const size_t loc[2] = {4 * (32 + 2) * (8 * 4 + 2), 4};
  set_local(2, loc);
  chk(g, launch(k_bfs_intratile, 32 * g->bfs.length, 8, 32, 4, 1));
}

/* intertile_gaps (GraphCut.pyx:172-185) */
static void intertile_gaps(GC* g) {
  bind_planes(g);
  A.list = g->edges.list;
  A.iteration = tl_increment(&g->bfs);
  A.tiles = g->bfs.tiles;
  const size_t loc[1] = {4 * 3};
  set_local(1, loc);
  chk(g, launch(k_bfs_intertile, 32 * g->edges.length, 1, 32, 1, 1));
}

/* startBfs (GraphCut.pyx:187-222) */
static void start_bfs(GC* g) {
  bind_planes(g);
  A.list = g->load.list;
  A.tiles = g->bfs.tiles;
  A.iteration = tl_increment(&g->bfs);
  const size_t loc[6] = {4 * 32 * 32, 4 * 6, 32 * 4, 32 * 4, 32 * 4, 32 * 4};
  set_local(6, loc);
  chk(g, launch(k_init_bfs, 32 * g->load.length, 4, 32, 4, 1));
  for (;;) {
    chk(g, tl_build(&g->bfs, OP_EQUAL, g->bfs.iteration));
    if (g->bfs.length > 0) {
      g->bfs_rounds++;
      intratile_gaps(g);
    } else {
      break;
    }
    chk(g, tl_build(&g->edges, OP_EQUAL, g->edges.iteration));
    if (g->edges.length > 0)
      intertile_gaps(g);
    else
      break;
  }
}

/* relabel (GraphCut.pyx:224-241): the Jacobi pass, then the two height buffers swap */
static void relabel_pass(GC* g) {
  bind_planes(g);
  set_local(0, NULL);
  chk(g, launch(k_relabel, round_up(WW, 16), round_up(HH, 16), 16, 16, 0));
  int* t = g->height;
  g->height = g->height2;
  g->height2 = t;
}

static void add_border_pass(GC* g, int direction) {
  chk(g, tl_build(&g->brd, OP_EQUAL, g->brd.iteration));
  if (!g->brd.length) return;
  bind_planes(g);
  A.list = g->brd.list;
  A.direction = direction;
  set_local(0, NULL);
  chk(g, launch(k_add_border, 32 * g->brd.length, 1, 32, 1, 0));
}

/* push (GraphCut.pyx:243-326): down, up, right, left, each followed by add_border */
static void push(GC* g) {
  const size_t loc_ud[1] = {4};
  const size_t loc_lr[3] = {4 * 32 * 33, 4 * 32 * 33, 4};
  void (*const body[4])(void) = {k_push_down, k_push_up, k_push_right, k_push_left};
  for (int d = 0; d < 4; ++d) {
    bind_planes(g);
    A.list = g->load.list;
    A.tiles = g->brd.tiles;
    A.iteration = tl_increment(&g->brd);
    if (d < 2)
      set_local(1, loc_ud);
    else
      set_local(3, loc_lr);
    chk(g, launch(body[d], 32 * g->load.length, 4, 32, 4, 1));
    add_border_pass(g, d);
  }
}

/* isCompleted (GraphCut.pyx:328-346) */
static int is_completed(GC* g) {
  g->is_completed = 1;
  bind_planes(g);
  A.list = g->load.list;
  A.is_completed = &g->is_completed;
  const size_t loc[1] = {4};
  set_local(1, loc);
  chk(g, launch(k_check_completion, 32 * g->load.length, 4, 32, 4, 1));
  return g->is_completed != 0;
}

/* cut (GraphCut.pyx:348-418), with an iteration cap (the reference loops until done) */
static int cut(GC* g, int bfs_period, long long max_iters) {
  const int load_iteration = g->load.iteration;
  bind_planes(g);
  A.tiles = g->load.tiles;
  A.iteration = tl_increment(&g->load);
  const size_t loc[1] = {4};
  set_local(1, loc);
  chk(g, launch(k_init_gc, WW, HH / 8, 32, 4, 1));
  chk(g, tl_build(&g->load, OP_EQUAL, g->load.iteration));
  load_listed(g);
  start_bfs(g);
  for (long long iteration = 1;; ++iteration) {
    if (g->err) return g->err;
    if (iteration > max_iters) return 3;
    push(g);
    g->iterations++;
    if (iteration % bfs_period == 0) {
      tl_increment(&g->load);
      chk(g, tl_incorporate(&g->load, g->brd.tiles, OP_LTE, load_iteration, OP_GTE,
                            g->brd.iteration - bfs_period * 4, LOGIC_AND));
      chk(g, tl_build(&g->load, OP_EQUAL, g->load.iteration));
      if (g->load.length > 0) load_listed(g);
      chk(g, tl_build(&g->load, OP_GT, load_iteration));
      start_bfs(g);
      if (is_completed(g)) return g->err;
    } else {
      relabel_pass(g);
      g->relabels++;
    }
  }
}

/* ---------------------------------------------------------------------------------------
 * C entry point.
 *
 * up/down/left/right/excess: int32 row-major [H][W] planes, where W x H is the size the
 * kernels were built for (refcl_width / refcl_height).  up/down/left/right hold the
 * capacity of the edge from a pixel to that neighbour; excess is the signed t-link
 * (positive = source capacity).
 * Out: the final residual planes and excess in the same layout (tiles never loaded get
 * their given capacities added, so the planes are the true residual graph), the final
 * heights, and stats[8] = {push iterations, relabel passes, BFS rounds, launches, guard
 * bytes found non-zero, barrier() calls without fibers, barrier releases with work-items
 * that had ended before it, final values that are not whole numbers}.  schedule: 0 =
 * the work-items of a group access bfs_intratile's loop flag in lockstep (a warp's order),
 * 1 = strictly one after another (a CPU OpenCL runtime's order).
 * Returns 0 when cut() finished, 1 for a bad argument, 2 for out of memory, 3 when
 * max_iters push iterations did not finish.  The harness keeps its state in file-scope
 * variables: one call at a time per process.
 * ------------------------------------------------------------------------------------- */
int refcl_width(void) { return WW; }
int refcl_height(void) { return HH; }

int refcl_cut(const int32_t* up, const int32_t* down, const int32_t* left,
              const int32_t* right, const int32_t* excess, int bfs_period, long long max_iters,
              int32_t* r_up, int32_t* r_down, int32_t* r_left, int32_t* r_right,
              int32_t* r_excess, int32_t* r_height, int schedule, long long* stats) {
  if (!up || !down || !left || !right || !excess || bfs_period <= 0 || schedule < 0 ||
      schedule > 1)
    return 1;
  const int32_t lim = 1 << 24;
  for (long i = 0; i < NPIX; ++i)
    if (up[i] < 0 || down[i] < 0 || left[i] < 0 || right[i] < 0 || up[i] >= lim ||
        down[i] >= lim || left[i] >= lim || right[i] >= lim || excess[i] >= lim ||
        excess[i] <= -lim)
      return 1;
  memset(&R, 0, sizeof(R));
  memset(&A, 0, sizeof(A));
  memset(&S, 0, sizeof(S));
  R.lockstep = schedule == 0;
  GC g;
  memset(&g, 0, sizeof(g));
  int rc = 0;
  R.stacks = malloc((size_t)MAX_ITEMS * STACK_BYTES);
  g.up = buf_new(NPIX, 4);
  g.down = buf_new(NPIX, 4);
  g.left = buf_new(NPIX, 4);
  g.right = buf_new(NPIX, 4);
  g.excess = buf_new(NPIX, 4);
  g.height = buf_new(NPIX, 4);
  g.height2 = buf_new(NPIX, 4);
  g.border = buf_new(NWAVE, 4);
  g.can_up = buf_new(NWAVE, 4);
  g.can_down = buf_new(NWAVE, 4);
  g.can_left = buf_new(NWAVE, 4);
  g.can_right = buf_new(NWAVE, 4);
  if (!R.stacks || !g.up || !g.down || !g.left || !g.right || !g.excess || !g.height ||
      !g.height2 || !g.border || !g.can_up || !g.can_down || !g.can_left || !g.can_right) {
    rc = 2;
    goto done;
  }
  if (tl_init(&g.load) || tl_init(&g.bfs) || tl_init(&g.edges) || tl_init(&g.brd)) {
    rc = 2;
    goto done;
  }
  g.src[0] = up;
  g.src[1] = down;
  g.src[2] = left;
  g.src[3] = right;
  for (long i = 0; i < NPIX; ++i) g.excess[i] = (float)excess[i];
  rc = cut(&g, bfs_period, max_iters);

  {
    /* tiles never loaded hold only the reverse flow pushed into them */
    uint8_t loaded[NT];
    for (int t = 0; t < NT; ++t) loaded[t] = g.load.tiles[t] > 0;
    long long frac = 0;
    for (int y = 0; y < HH; ++y)
      for (int x = 0; x < WW; ++x) {
        const long i = (long)y * WW + x, j = tpos(x, y);
        const int t = (y / 32) * TW + x / 32;
        float v[6] = {g.up[i], g.down[i], g.left[j], g.right[j], g.excess[i], 0.f};
        if (!loaded[t])
          for (int d = 0; d < 4; ++d) v[d] += (float)g.src[d][i];
        int32_t* out[5] = {r_up, r_down, r_left, r_right, r_excess};
        for (int d = 0; d < 5; ++d) {
          if ((float)(int32_t)v[d] != v[d]) frac++;
          if (out[d]) out[d][i] = (int32_t)v[d];
        }
        if (r_height) r_height[i] = g.height[i];
      }
    if (stats) {
      stats[0] = g.iterations;
      stats[1] = g.relabels;
      stats[2] = g.bfs_rounds;
      stats[3] = R.launches;
      stats[4] = guards_dirty() + gbufs_dirty();
      stats[5] = R.bad_barrier;
      stats[6] = R.divergent;
      stats[7] = frac;
    }
  }
done:
  for (int k = 0; k < MAX_LOCAL; ++k) {
    free(R.loc[k]);
    R.loc[k] = NULL;
  }
  free(R.stacks);
  bufs_free();
  gbufs_free();
  return rc;
}
