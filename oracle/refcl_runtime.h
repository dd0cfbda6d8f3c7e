/* Work-group runtime for running the reference's OpenCL kernels on the host.  TEST
 * INFRASTRUCTURE ONLY: included by refcl_host.c (graphcut.cl) and refcl_scan.c
 * (prefixsum.cl, streamcompact.cl), each built into its own library under oracle/_ref/.
 * Every definition is file-local except the OpenCL built-ins refcl_clc.h declares.
 */
#ifndef REFCL_RUNTIME_H
#define REFCL_RUNTIME_H

#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "refcl_clc.h"

/* ---------------------------------------------------------------------------------------
 * Work-group runtime.  A work-item switches back to the scheduler at a barrier, at a
 * lockstep point the including file defines (refcl_host.c: each access to
 * bfs_intratile's loop flag) and when it ends.  The scheduler resumes, in local-id order,
 * every work-item not waiting at a barrier, pass after pass; when every work-item still
 * running waits at the barrier, it releases them all.  Work-items that ended before a
 * barrier are not waited for (a GPU drops exited threads from a barrier the same way); the
 * harness counts such releases.
 * ------------------------------------------------------------------------------------- */
enum { MAX_ITEMS = 256, STACK_BYTES = 64 * 1024, MAX_LOCAL = 8 };
enum { ST_RUN = 0, ST_BARRIER = 1, ST_DONE = 2 };

typedef struct {
  void* sp;
  int lid[2];
  int state;
} Item;

static struct {
  int lsz[2], ngrp[2], grp[2];
  Item* cur;
  void* sched_sp;
  void (*body)(void);
  int fibers, lockstep;
  Item items[MAX_ITEMS];
  char* stacks;
  void* loc[MAX_LOCAL];
  size_t locsz[MAX_LOCAL];
  int nloc;
  long long launches, divergent, bad_barrier;
} R;

/* Stack switch (x86-64 System V): save the callee-saved registers on the current stack,
 * store the stack pointer in *save, load `to` and restore the registers saved there. */
__asm__(
    ".text\n"
    ".p2align 4\n"
    ".globl refcl_swap\n"
    ".hidden refcl_swap\n"
    ".type refcl_swap, @function\n"
    "refcl_swap:\n"
    "  pushq %rbp\n"
    "  pushq %rbx\n"
    "  pushq %r12\n"
    "  pushq %r13\n"
    "  pushq %r14\n"
    "  pushq %r15\n"
    "  movq %rsp, (%rdi)\n"
    "  movq %rsi, %rsp\n"
    "  popq %r15\n"
    "  popq %r14\n"
    "  popq %r13\n"
    "  popq %r12\n"
    "  popq %rbx\n"
    "  popq %rbp\n"
    "  ret\n"
    ".size refcl_swap, .-refcl_swap\n");
void refcl_swap(void** save, void* to);

static void fiber_entry(void) {
  R.body();
  R.cur->state = ST_DONE;
  refcl_swap(&R.cur->sp, R.sched_sp);
  abort(); /* a finished work-item is never resumed */
}

/* A fresh fiber's stack: six zero registers for refcl_swap to pop, then fiber_entry as the
 * return address, placed so that fiber_entry starts with the stack aligned as after a call. */
static void* fiber_stack(int i) {
  uintptr_t top = ((uintptr_t)(R.stacks + (size_t)(i + 1) * STACK_BYTES)) & ~(uintptr_t)15;
  uintptr_t* sp = (uintptr_t*)top;
  *--sp = 0;
  *--sp = (uintptr_t)fiber_entry;
  for (int k = 0; k < 6; ++k) *--sp = 0;
  return sp;
}

size_t get_local_id(uint d) { return d < 2 ? (size_t)R.cur->lid[d] : 0; }
size_t get_group_id(uint d) { return d < 2 ? (size_t)R.grp[d] : 0; }
size_t get_local_size(uint d) { return d < 2 ? (size_t)R.lsz[d] : 1; }
size_t get_num_groups(uint d) { return d < 2 ? (size_t)R.ngrp[d] : 1; }
size_t get_global_size(uint d) { return d < 2 ? (size_t)R.ngrp[d] * R.lsz[d] : 1; }
size_t get_global_id(uint d) {
  return d < 2 ? (size_t)R.grp[d] * R.lsz[d] + (size_t)R.cur->lid[d] : 0;
}

void barrier(int fence) {
  (void)fence;
  if (!R.fibers) {
    R.bad_barrier++;
    return;
  }
  R.cur->state = ST_BARRIER;
  refcl_swap(&R.cur->sp, R.sched_sp);
}

static void set_local(int n, const size_t* bytes) {
  for (int k = 0; k < n; ++k) {
    free(R.loc[k]);
    R.loc[k] = calloc(1, bytes[k] ? bytes[k] : 1);
    R.locsz[k] = bytes[k];
  }
  R.nloc = n;
}

/* One NDRange launch: global size g0 x g1, work-group size l0 x l1.  Kernels that reach a
 * barrier run as fibers; the others run each work-item as a plain call.  Local memory is
 * cleared before every work-group. */
static int launch(void (*body)(void), int g0, int g1, int l0, int l1, int fibers) {
  if (g0 < 0 || g1 < 0 || l0 <= 0 || l1 <= 0 || g0 % l0 || g1 % l1 || l0 * l1 > MAX_ITEMS)
    return 1;
  R.launches++;
  if (g0 == 0 || g1 == 0) return 0;
  R.lsz[0] = l0;
  R.lsz[1] = l1;
  R.ngrp[0] = g0 / l0;
  R.ngrp[1] = g1 / l1;
  R.body = body;
  R.fibers = fibers;
  const int n = l0 * l1;
  for (int gy = 0; gy < R.ngrp[1]; ++gy)
    for (int gx = 0; gx < R.ngrp[0]; ++gx) {
      R.grp[0] = gx;
      R.grp[1] = gy;
      for (int k = 0; k < R.nloc; ++k) memset(R.loc[k], 0, R.locsz[k]);
      if (!fibers) {
        Item it = {0};
        R.cur = &it;
        for (int ly = 0; ly < l1; ++ly)
          for (int lx = 0; lx < l0; ++lx) {
            it.lid[0] = lx;
            it.lid[1] = ly;
            body();
          }
        continue;
      }
      for (int i = 0; i < n; ++i) {
        R.items[i].lid[0] = i % l0;
        R.items[i].lid[1] = i / l0;
        R.items[i].state = ST_RUN;
        R.items[i].sp = fiber_stack(i);
      }
      int live = n, ended_since_release = 0;
      while (live > 0) {
        int waiting = 0;
        for (int i = 0; i < n; ++i) {
          Item* it = &R.items[i];
          if (it->state == ST_RUN) {
            R.cur = it;
            refcl_swap(&R.sched_sp, it->sp);
            if (it->state == ST_DONE) {
              live--;
              ended_since_release++;
            }
          }
          waiting += it->state == ST_BARRIER;
        }
        if (live > 0 && waiting == live) {
          if (ended_since_release) R.divergent++;
          ended_since_release = 0;
          for (int i = 0; i < n; ++i)
            if (R.items[i].state == ST_BARRIER) R.items[i].state = ST_RUN;
        }
      }
    }
  return 0;
}

#endif
