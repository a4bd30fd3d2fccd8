// solver.cuh -- device side of the B200 solver: a thread group advances one zone at a time.
//
// Data layout: the network (DevNet) is zone-shared and read-only; every group owns a workspace slab
// (WsLayout) holding its zone's rates, Jacobian values, LU values and integrator vectors, so each
// per-zone sweep is a contiguous, coalesced stream. Every phase below is a group-wide loop followed
// by a group barrier; scalar control flow (step-size logic of solver.F90, backward_euler.F90 and
// bader_deuflhard.F90) is evaluated redundantly by all threads of the group from group-reduced
// values, so it is uniform across the group.
//
// The group is a compile-time choice: solver.cu is compiled twice.
//   NUPPN_GROUP_WARP = 0 (namespace nuppn::cta):  the group is the whole CTA, one zone per CTA; the
//                                                  wide phases use every warp, the chains one warp.
//   NUPPN_GROUP_WARP = 1 (namespace nuppn::warp): the group is one warp, one zone per warp and as
//                                                  many zones per CTA as it has warps; every phase,
//                                                  chains included, runs on that warp.
// GT / GN / GID are the thread's rank in its group, the group size and the group's index in the CTA;
// GSYNC() is the group barrier, g_or / g_and its predicate reductions.
#pragma once
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdint.h>

#include "nuppn_internal.h"

#ifndef NUPPN_GROUP_WARP
#define NUPPN_GROUP_WARP 0
#endif

#if NUPPN_GROUP_WARP
#define NUPPN_VNS warp
#define GT ((int)(threadIdx.x & 31u))
#define GN 32
#define GID ((int)(threadIdx.x >> 5))
#define GSYNC() __syncwarp()
#define NUPPN_MAX_GROUPS 8
__device__ __forceinline__ int g_or(int p) { return __any_sync(0xffffffffu, p); }
__device__ __forceinline__ int g_and(int p) { return __all_sync(0xffffffffu, p); }
#else
#define NUPPN_VNS cta
#define GT ((int)threadIdx.x)
#define GN ((int)blockDim.x)
#define GID 0
#define GSYNC() __syncthreads()
#define NUPPN_MAX_GROUPS 1
__device__ __forceinline__ int g_or(int p) { return __syncthreads_or(p); }
__device__ __forceinline__ int g_and(int p) { return __syncthreads_and(p); }
#endif

// groups (zones) in a CTA of `block` threads, for host code
#define NUPPN_GROUPS_PER_CTA(block) (NUPPN_GROUP_WARP ? (block) / 32 : 1)

#define NUPPN_BEGIN \
  namespace nuppn {  \
  namespace NUPPN_VNS {
#define NUPPN_END \
  }                \
  }

NUPPN_BEGIN

#define NUPPN_FULL 0xffffffffu

constexpr int kLongList = 48;   // gather lists longer than this are summed by a whole warp

struct Ws {
  double *v, *rv, *ngv, *ffv, *kdv, *partinter, *G, *flux, *contrib, *jac, *xn, *dxdt;
  double *y, *y_old, *y_cur, *y_new, *y_k, *delta_k, *y_ext, *yscal, *qcol, *yerr, *lu, *bsys, *xsys, *rhs;
  int *first_l;
  uint8_t *eset, *mask;
  int *act_tmp;  // compaction scratch: sys2c, arow, counts
  char *act;     // global fallback of the active-subsystem LU
  char *act_r;   // global fallback of the restricted right-hand side
  int *rhs_key;       // right-hand side items' group keys, then group keys [dg items]
  double *rhs_val;    // their values, then group sums [dg items]
  int *rhs_piece;     // first piece of each active row [nsys+1]; per piece groups, own terms, own offsets; per row own terms
  double *rhs_acc;    // key accumulators of the grouping, one per warp [warps * 8 * (nsys+1)]
  int *rhs_spc;       // species -> active row of the current step, -1 if frozen [nsp]
  uint8_t *cache_mask;  // mask of the last build of the active subsystem [nsp]
  double *cache_xn;     // molar abundances it was built with [nsp]
  int *rhs_rkey;      // each reaction's class of the step [nact]
  double *rhs_rcf;    // its constant [nact]
  uint32_t *rhs_rpk;  // packed reactants of an own-term reaction [nact]
  int *jac_long;      // long Jacobian entries: flags, positions, first pieces [3 * (nnzLU + 1)]
  int *rhs_tag, *rhs_list;
  double *nse_x, *nse_gtot, *nse_mc, *nse_lm, *nse_y1, *nse_sort;  // NSE work arrays
  int *act_otmp; // segment offsets of the active Jacobian entries [nnzLU + 1]
  double *act_dtmp;   // flattened Jacobian contributions [jg items]
  uint8_t *act_btmp;  // flattened entry-set flags [jg items]
  double *bd;         // compact Bader-Deuflhard vectors [(2*kMaxLevels + 8) * nsys]
};

__device__ __forceinline__ Ws ws_bind(char *base, const WsLayout &L) {
  Ws w;
  w.v = (double *)(base + L.v); w.rv = (double *)(base + L.rv); w.ngv = (double *)(base + L.ngv);
  w.ffv = (double *)(base + L.ffv); w.kdv = (double *)(base + L.kdv);
  w.partinter = (double *)(base + L.partinter); w.G = (double *)(base + L.G);
  w.flux = (double *)(base + L.flux); w.contrib = (double *)(base + L.contrib);
  w.first_l = (int *)(base + L.first_l); w.eset = (uint8_t *)(base + L.eset);
  w.jac = (double *)(base + L.jac); w.mask = (uint8_t *)(base + L.mask); w.xn = (double *)(base + L.xn);
  w.dxdt = (double *)(base + L.dxdt); w.y = (double *)(base + L.y); w.y_old = (double *)(base + L.y_old);
  w.y_cur = (double *)(base + L.y_cur); w.y_new = (double *)(base + L.y_new); w.y_k = (double *)(base + L.y_k);
  w.delta_k = (double *)(base + L.delta_k); w.y_ext = (double *)(base + L.y_ext);
  w.yscal = (double *)(base + L.yscal); w.qcol = (double *)(base + L.qcol); w.yerr = (double *)(base + L.yerr);
  w.lu = (double *)(base + L.lu); w.bsys = (double *)(base + L.bsys); w.xsys = (double *)(base + L.xsys);
  w.rhs = (double *)(base + L.rhs);
  w.act_tmp = (int *)(base + L.act_tmp);
  w.act = base + L.act;
  w.act_r = base + L.act_r;
  w.rhs_key = (int *)(base + L.rhs_key);
  w.rhs_val = (double *)(base + L.rhs_val);
  w.rhs_piece = (int *)(base + L.rhs_piece);
  w.rhs_acc = (double *)(base + L.rhs_acc);
  w.rhs_spc = (int *)(base + L.rhs_spc);
  w.cache_mask = (uint8_t *)(base + L.cache_mask);
  w.cache_xn = (double *)(base + L.cache_xn);
  w.rhs_rkey = (int *)(base + L.rhs_rkey);
  w.rhs_rcf = (double *)(base + L.rhs_rcf);
  w.rhs_rpk = (uint32_t *)(base + L.rhs_rpk);
  w.jac_long = (int *)(base + L.jac_long);
  w.rhs_tag = (int *)(base + L.rhs_tag);
  w.rhs_list = (int *)(base + L.rhs_list);
  w.nse_x = (double *)(base + L.nse);
  w.nse_gtot = w.nse_x + L.nse_stride;
  w.nse_mc = w.nse_gtot + L.nse_stride;
  w.nse_lm = w.nse_mc + L.nse_stride;
  w.nse_y1 = w.nse_lm + L.nse_stride;
  w.nse_sort = w.nse_y1 + L.nse_stride;
  w.act_otmp = (int *)(base + L.act_otmp);
  w.act_dtmp = (double *)(base + L.act_dtmp);
  w.act_btmp = (uint8_t *)(base + L.act_btmp);
  w.bd = (double *)(base + L.bd);
  return w;
}

NUPPN_END
