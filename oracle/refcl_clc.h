/* OpenCL C built-ins for compiling the reference's own kernel sources (graphcut.cl,
 * incremental_tile_list.cl) unchanged as C on the host.  TEST INFRASTRUCTURE ONLY: it
 * serves the reference-kernel harness (refcl_host.c), which checks the oracle; nothing in
 * the product includes it.
 *
 * Execution model (refcl_host.c implements it): the work-items of a work-group run as
 * cooperative fibers on one host thread, in local-id order (x fastest).  barrier() hands
 * control to the next work-item, so every work-item runs up to the barrier before any
 * runs past it -- the way a CPU OpenCL runtime executes a work-group.  Work-groups run one
 * after another in group-id order, so no two work-groups race on global memory.
 *
 * Address-space qualifiers vanish (one flat host address space); min/max follow the
 * OpenCL C definitions (min(x, y) = y < x ? y : x); <tgmath.h> makes sqrt of a float a
 * float sqrt, as in OpenCL C.  Compile with -ffp-contract=off so that float expressions
 * round operation by operation, as OpenCL C requires without -cl-mad-enable.
 */
#ifndef REFCL_CLC_H
#define REFCL_CLC_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>
#include <tgmath.h>

#define __kernel static
#define __global
#define __local
#define __private
#define __constant const
#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2

typedef unsigned char uchar;
typedef unsigned short ushort;
typedef unsigned int uint;
typedef struct {
  int x, y;
} int2;

#define min(a, b) ((b) < (a) ? (b) : (a))
#define max(a, b) ((a) < (b) ? (b) : (a))

size_t get_global_id(uint dim);
size_t get_local_id(uint dim);
size_t get_group_id(uint dim);
size_t get_local_size(uint dim);
size_t get_global_size(uint dim);
size_t get_num_groups(uint dim);
void barrier(int fence);

#endif
