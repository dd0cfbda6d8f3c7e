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
 * Every buffer sits inside zero-filled guard bands (refcl_prefixsum.h), and each call
 * reports how many guard bytes it found written: the reference's kernels or its host code
 * writing past a buffer show up there instead of corrupting other memory.
 */
#include "refcl_clc.h"

/* prefixsum.cl defines its helpers as C99 `inline` functions without an external
 * definition; here they become file-local. */
#define inline static inline
#include REF_PREFIXSUM_CL
#undef inline
#include REF_STREAMCOMPACT_CL

#include "refcl_runtime.h"

#include "refcl_prefixsum.h"

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
  rc = sc_compact(&ps, d_flags, d_list, d_len, length);
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
