/* PrefixSum / StreamCompact host code (PrefixSum.pyx:40-129, StreamCompact.pyx:66-82)
 * restated over the reference's prefixsum.cl / streamcompact.cl kernels.  TEST
 * INFRASTRUCTURE ONLY: included, after the kernels and refcl_runtime.h, by refcl_scan.c and
 * refcl_host.c (whose tile lists compact with it, as IncrementalTileList.build does).
 *
 * Its buffers sit between zero-filled guard bands (for a partial-sum buffer, as long as the
 * largest partial-sum array any level can write); gbufs_dirty() counts guard bytes found
 * written, so a write past a buffer shows up instead of corrupting other memory.
 */
#ifndef REFCL_PREFIXSUM_H
#define REFCL_PREFIXSUM_H

#include <math.h>

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

/* StreamCompact.compact (StreamCompact.pyx:66-82): copy the flags into the list, scan the
 * list in place (the sum goes to *length_out), then the compact kernel with the list as
 * both prefix sums and output. */
static int sc_compact(PrefixSum* ps, int* flags, int* list, int* length_out, int length) {
  memcpy(list, flags, sizeof(int) * (size_t)length);
  int rc = ps_scan(ps, list, length_out, length);
  if (rc) return rc;
  S.flags = flags;
  S.list = list;
  S.n = length;
  set_local(0, NULL);
  return launch(k_compact, (length + LEN_WORKGROUP - 1) / LEN_WORKGROUP * LEN_WORKGROUP, 1,
                LEN_WORKGROUP, 1, 0);
}

#endif
