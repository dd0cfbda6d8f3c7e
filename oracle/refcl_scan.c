/* The reference's own scan and compaction kernels, run on the host.  TEST INFRASTRUCTURE
 * ONLY: the parity tests use it to check the reference's PrefixSum / StreamCompact against
 * exact answers; nothing in the product links or loads it.
 *
 * prefixsum.cl and streamcompact.cl are compiled unchanged from where they lie (the
 * Makefile passes their paths as REF_PREFIXSUM_CL / REF_STREAMCOMPACT_CL; the library goes
 * to oracle/_ref/ only), under the work-group runtime of refcl_runtime.h.  The host side
 * restates PrefixSum.__init__ / scan (PrefixSum.pyx:40-129: 256 work-items per group, 512
 * elements per group, one buffer of partial sums per level, the level picked as
 * int(log(length) / log(512)) - 1, recursion on the partial sums) and StreamCompact.compact
 * (StreamCompact.pyx:66-82: copy the flags into the list, scan the list in place, then the
 * compact kernel with the list as both prefix sums and output).
 *
 * Every buffer sits inside zero-filled guard bands (for a partial-sum buffer, as long as
 * the largest partial-sum array any level can write), and each call reports how many guard
 * bytes it found written: the reference's kernels or its host code writing past a buffer
 * show up there instead of corrupting other memory.
 */
#include <math.h>

#include "refcl_clc.h"

/* prefixsum.cl defines its helpers as C99 `inline` functions without an external
 * definition; here they become file-local. */
#define inline static inline
#include REF_PREFIXSUM_CL
#undef inline
#include REF_STREAMCOMPACT_CL

#include "refcl_runtime.h"

enum { LEN_WORKGROUP = 256, ELEMENTS_PER_WORKGROUP = 512, MAX_LEVELS = 8 };

/* ---------------------------------------------------------------------------------------
 * Buffers of n ints between two guard bands of `guard` ints each.
 * ------------------------------------------------------------------------------------- */
typedef struct {
  char* base;
  size_t bytes, guard;
} GBuf;

static GBuf g_scan_bufs[MAX_LEVELS + 4];
static int g_scan_nbufs;

static int* gbuf_new(size_t n, size_t guard) {
  if (g_scan_nbufs >= (int)(sizeof(g_scan_bufs) / sizeof(g_scan_bufs[0]))) return NULL;
  GBuf* b = &g_scan_bufs[g_scan_nbufs++];
  b->bytes = (n ? n : 1) * sizeof(int);
  b->guard = (guard ? guard : 1) * sizeof(int);
  b->base = calloc(1, b->bytes + 2 * b->guard);
  return b->base ? (int*)(b->base + b->guard) : NULL;
}

static long long gbufs_dirty(void) {
  long long bad = 0;
  for (int k = 0; k < g_scan_nbufs; ++k) {
    const GBuf* b = &g_scan_bufs[k];
    for (size_t i = 0; i < b->guard; ++i)
      bad += (b->base[i] != 0) + (b->base[b->guard + b->bytes + i] != 0);
  }
  return bad;
}

static void gbufs_free(void) {
  for (int k = 0; k < g_scan_nbufs; ++k) free(g_scan_bufs[k].base);
  g_scan_nbufs = 0;
}

/* ---------------------------------------------------------------------------------------
 * Kernel arguments and entries.
 * ------------------------------------------------------------------------------------- */
static struct {
  int *data, *part, *total, *flags, *list;
  int n;
} S;

static void k_pad(void) { scan_pad_to_pow2(S.data, (int*)R.loc[0], S.n, S.total); }
static void k_sub(void) { scan_subarrays(S.data, (int*)R.loc[0], S.part, S.n); }
static void k_inc(void) { scan_inc_subarrays(S.data, (int*)R.loc[0], S.part, S.n); }
static void k_compact(void) { compact(S.flags, S.list, S.list, S.n); }

/* ---------------------------------------------------------------------------------------
 * PrefixSum (PrefixSum.pyx:40-129).
 * ------------------------------------------------------------------------------------- */
typedef struct {
  int capacity;
  int* parts[MAX_LEVELS];
  int nparts;
} PrefixSum;

static int ps_init(PrefixSum* ps, int capacity) {
  /* capacity rounded up to whole groups; one partial-sum buffer per level */
  ps->capacity = (capacity + ELEMENTS_PER_WORKGROUP - 1) / ELEMENTS_PER_WORKGROUP *
                 ELEMENTS_PER_WORKGROUP;
  ps->nparts = 0;
  const size_t widest = (size_t)(ps->capacity / ELEMENTS_PER_WORKGROUP) + 1;
  for (int len = ps->capacity / ELEMENTS_PER_WORKGROUP; len > 0; len /= ELEMENTS_PER_WORKGROUP) {
    if (ps->nparts >= MAX_LEVELS) return 1;
    if (!(ps->parts[ps->nparts++] = gbuf_new((size_t)len, widest))) return 2;
  }
  return 0;
}

static int ps_scan(PrefixSum* ps, int* data, int* total, int length) {
  const int k = (length + ELEMENTS_PER_WORKGROUP - 1) / ELEMENTS_PER_WORKGROUP;
  const size_t loc[1] = {ELEMENTS_PER_WORKGROUP * sizeof(int)};
  set_local(1, loc);
  if (k == 1) {
    S.data = data;
    S.n = length;
    S.total = total;
    return launch(k_pad, k * LEN_WORKGROUP, 1, LEN_WORKGROUP, 1, 1);
  }
  if (length > ps->capacity) return 1;
  const int i = (int)(log((double)length) / log((double)ELEMENTS_PER_WORKGROUP)) - 1;
  if (i < 0 || i >= ps->nparts) return 4; /* the reference indexes a missing level */
  int* part = ps->parts[i];
  S.data = data;
  S.part = part;
  S.n = length;
  int rc = launch(k_sub, k * LEN_WORKGROUP, 1, LEN_WORKGROUP, 1, 1);
  if (rc) return rc;
  rc = ps_scan(ps, part, total, k);
  if (rc) return rc;
  set_local(1, loc);
  S.data = data;
  S.part = part;
  S.n = length;
  return launch(k_inc, k * LEN_WORKGROUP, 1, LEN_WORKGROUP, 1, 0);
}

static void run_begin(void) {
  memset(&R, 0, sizeof(R));
  memset(&S, 0, sizeof(S));
  R.lockstep = 0;
}

static void run_end(void) {
  for (int k = 0; k < MAX_LOCAL; ++k) {
    free(R.loc[k]);
    R.loc[k] = NULL;
  }
  free(R.stacks);
  R.stacks = NULL;
  gbufs_free();
}

/* ---------------------------------------------------------------------------------------
 * C entry points.  stats[3] = {launches, guard bytes found written, barrier() calls
 * without fibers}.  Return 0, 1 for a bad argument, 2 for out of memory, 4 when the
 * reference's host code would index a partial-sum level that does not exist.  The
 * reference cannot scan an empty array (log(0)), so length must be >= 1.  File-scope
 * state: one call at a time per process.
 * ------------------------------------------------------------------------------------- */

/* PrefixSum(capacity).scan(data, total, length): out[i] = exclusive scan of in[0, length),
 * *total = the sum. */
int refcl_scan(const int32_t* in, int length, int capacity, int32_t* out, int32_t* total,
               long long* stats) {
  if (!in || !out || !total || length < 1 || capacity < length) return 1;
  run_begin();
  int rc = 0;
  PrefixSum ps;
  R.stacks = malloc((size_t)MAX_ITEMS * STACK_BYTES);
  int* data = gbuf_new((size_t)length, (size_t)length);
  int* tot = gbuf_new(1, 1);
  if (!R.stacks || !data || !tot) {
    rc = 2;
    goto done;
  }
  if ((rc = ps_init(&ps, capacity)) != 0) goto done;
  memcpy(data, in, sizeof(int) * (size_t)length);
  rc = ps_scan(&ps, data, tot, length);
  memcpy(out, data, sizeof(int) * (size_t)length);
  *total = *tot;
  if (stats) {
    stats[0] = R.launches;
    stats[1] = gbufs_dirty();
    stats[2] = R.bad_barrier;
  }
done:
  run_end();
  return rc;
}

/* StreamCompact(capacity).compact(flags, list, length_out, length): the list of flagged
 * indices and its length. */
int refcl_compact(const int32_t* flags, int length, int capacity, int32_t* list,
                  int32_t* length_out, long long* stats) {
  if (!flags || !list || !length_out || length < 1 || capacity < length) return 1;
  run_begin();
  int rc = 0;
  PrefixSum ps;
  R.stacks = malloc((size_t)MAX_ITEMS * STACK_BYTES);
  int* d_flags = gbuf_new((size_t)length, (size_t)length);
  int* d_list = gbuf_new((size_t)length, (size_t)length);
  int* d_len = gbuf_new(1, 1);
  if (!R.stacks || !d_flags || !d_list || !d_len) {
    rc = 2;
    goto done;
  }
  if ((rc = ps_init(&ps, capacity)) != 0) goto done;
  memcpy(d_flags, flags, sizeof(int) * (size_t)length);
  memcpy(d_list, flags, sizeof(int) * (size_t)length); /* enqueue_copy(dList, dFlags) */
  if ((rc = ps_scan(&ps, d_list, d_len, length)) != 0) goto done;
  S.flags = d_flags;
  S.list = d_list;
  S.n = length;
  set_local(0, NULL);
  rc = launch(k_compact, (length + LEN_WORKGROUP - 1) / LEN_WORKGROUP * LEN_WORKGROUP, 1,
              LEN_WORKGROUP, 1, 0);
  memcpy(list, d_list, sizeof(int) * (size_t)length);
  *length_out = *d_len;
  if (stats) {
    stats[0] = R.launches;
    stats[1] = gbufs_dirty();
    stats[2] = R.bad_barrier;
  }
done:
  run_end();
  return rc;
}
