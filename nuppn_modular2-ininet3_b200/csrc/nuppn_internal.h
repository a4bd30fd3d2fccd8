// nuppn_internal.h -- shared host/device structures of the B200 solver library.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/nuppn.h"

namespace nuppn {

constexpr int kMaxLevels = 8;       // Bader-Deuflhard tableau columns (bader_deuflhard.F90:24)
constexpr int kRhsPiece = 1024;     // right-hand side items per piece when grouping frozen-reactant terms
constexpr int kRhsKeysPerRow = 8;   // group keys per active row: (row << 3) | power of its xn
constexpr int kRhsWarps = 8;        // warps of a zone group at most (256 threads), one key accumulator each
constexpr int kPartDim = 24;        // partition-function temperature points (array_sizes.F90:15)

// Network as the device sees it: every pointer is device memory, read-only during solves.
struct DevNet {
  int nsp, nre, nact, ig, nsys, nnzJ, nnzLU;
  int ihe4, ibe8;
  // species
  const double *an, *zn;
  const uint8_t *ciso;
  const int *spart;          // partition row or -1
  const double *gspin_nse;   // ppn_g where the species is in the NSE set, 0 otherwise
  // all reaction slots (rates)
  const int *src, *sidx;
  const double *rfac;
  const uint8_t *crea, *rev_target;
  const int *ilabb;
  const int *scr_mode;       // 0 pair (z1,z2), 1 triple-alpha, 2 n(2a,g), 3 unscreened-slot
  const double *scr_z1, *scr_z2;
  const int *irev;           // slot of the reverse or -1 (considered forwards only)
  const int *rev_sp;         // [nre*4] species for G: a1, a2 (or a1 if na1==2), b1 (-1 -> G=0), b2
  const int *rev_kind;       // 1 capture (ng,pg,ag), 2 other, 0 unusable
  const double *rev_mc;      // capture: m_a1 m_a2/m_b2 *2pi/h^2 ; other: (m_a1 m_a2/m_b1/m_b2)^1.5
  const double *rev_Q;       // Q (MeV) as reverse.F90:279/296
  // active (considered) reactions
  const int *act_slot;       // [nact] slot index
  const int *act_k;          // [nact*8] k1..k8
  const int *act_ice;        // [nact*8] dns2csr_map in reference slot order
  // REACLIB
  int nc, nr;
  const int *rl_first;       // [nr+1]
  const double *rl_a;        // [nc*7]
  const int *rl_info;        // [nr] chapter | vflag<<8 | ecflag<<9 | nireac<<16
  const int *rl_part;        // [nr*6]
  int npart;
  const double *pt9, *pval;  // [24], [npart*24]
  // VITAL templates
  int nv;
  const int *vfirst, *vxfac, *vform;
  const double *vterms, *vdpow;
  // NETGEN
  int ngk, ngn, ngd;
  const double *ngt8, *ngl10t8, *ngflag, *ngane, *ngl10v;
  const int *ngndata;
  // FFN
  int ffv, fft, ffr;
  const double *fft9, *ffrho, *ffl10v;
  // KADoNiS (Akima coefficients [n][ne-1][4])
  int kdn, kde;
  const double *kdE, *kdcoef;
  const double *constr;
  // Jacobian pattern and gathers
  const int *jrow, *jcol, *jdiag;          // jdiag[nsp]: entry of (i,i) or -1
  const int *jg_ptr, *jg_item;             // entry -> (a*8 + s) in reference accumulation order
  const int *jg_oth;                       // per jg item: the other reactant's species, -1 for gamma
  int ndg_item;                            // dg items of all species
  const int *dg_ptr, *dg_item;             // species -> (a*4 + slot) in scatter order
  const double *dg_coef;                   // coefficient of each dg item: -k2, -1, k6, k8
  int njg_long, ndg_long;
  const int *jg_long, *dg_long;            // entries / species whose gather lists are long
  const int *k1_ptr, *k1_list;             // species -> considered reactions it leads (k1), in order
  // NSE set (nse_swj.F90:208-245)
  int nse_num, nse_iprot, nse_ini56, nse_p2;
  const int *nse_idx, *nse_part;
  const double *nse_m, *nse_q, *nse_g, *nse_z, *nse_n, *nse_zoa;
  // system and LU
  const int *sys_of_sp, *sp_of_sys;        // [nsp], [nsys]
  const int *pos_of_entry;                 // [nnzJ] LU position or -1
  const int *lu_src;                       // [nnzLU] Jacobian entry of an LU position or -1 (fill)
  const int *lu_rowptr, *lu_diag, *lu_col; // [nsys+1], [nsys], [nnzLU]
  const int *upd_start;                    // [nnzLU+1] for L entries: start in upd_off
  const uint16_t *upd_off;                 // offsets into the target row
  int nlvL, nlvU;
  const int *lvL_ptr, *lvL_rows, *lvL_grp; // factorization / forward levels
  const int *lvU_ptr, *lvU_rows, *lvU_grp; // backward levels
  // Bader-Deuflhard constants
  int nseq[kMaxLevels + 2];
  double bd_a[kMaxLevels + 2];
  double alf[kMaxLevels + 1][kMaxLevels + 1];
  int kmax, kopt0;
  nuppn_knobs kn;
  // derived constants
  int nvar;                                // count(considerisotope)
};

// Per-CTA workspace layout (byte offsets into one slab).
struct WsLayout {
  size_t v, rv, ngv, ffv, kdv, partinter, G, flux, contrib, first_l, eset, jac, mask, xn, dxdt;
  size_t y, y_old, y_cur, y_new, y_k, delta_k, y_ext, yscal, qcol, yerr, lu, bsys, xsys, rhs;
  size_t act_tmp, act;           // compaction scratch (ints) and the global fallback of the active LU
  size_t act_r;                  // global fall-back of the restricted right-hand side
  size_t act_otmp, act_dtmp, act_btmp, bd;  // flattened-gather scratch, compact BD vectors
  size_t rhs_key, rhs_val, rhs_piece;  // grouping of the right-hand side's frozen-reactant terms
  size_t rhs_acc, rhs_tag, rhs_list;   // per-warp key accumulators of that grouping
  size_t rhs_spc;                      // species -> active row of the step
  size_t cache_mask, cache_xn;         // mask and abundances of the last build of the active subsystem
  size_t rhs_rkey, rhs_rcf, rhs_rpk;   // each reaction's class, constant and packed own term of the step
  size_t jac_long;                     // long Jacobian entries of the step and their pieces
  size_t nse;                    // NSE work arrays [5 * nsp + nse_p2] doubles
  size_t nse_stride;             // nsp: the length of each NSE work array but the last
  size_t bytes;
};

#ifdef __CUDACC__
#define NUPPN_HD __host__ __device__
#else
#define NUPPN_HD
#endif

// Active systems up to kTileMax rows are factored in a dense tile of 32 or 64 rows and solved with
// one (or two) rows per lane of a warp (active_lu.cuh).
constexpr int kTileMax = 64;

NUPPN_HD inline size_t a16(size_t x) { return (x + 15) & ~size_t(15); }

// Tile rows (0, 32 or 64) for an active system of na rows under the knob lu_tile_max
// (0 = kTileMax, negative = never).
NUPPN_HD inline int tile_rows_for(int na, int limit) {
  if (limit < 0) return 0;
  const int lim = (limit == 0 || limit > kTileMax) ? kTileMax : limit;
  return na > lim ? 0 : (na <= 32 ? 32 : 64);
}

// Bytes of the active-subsystem LU for na rows, nnz entries, nwarps warps and a tile of tile_rows
// rows (see active_lu.cuh): int crp[na+1], cdiag[na], arow[na], flagF[na], flagS[na], ccol[nnz],
// csrc[nnz]; without a tile double cval[nnz], wbuf[nwarps*na], rdg[na]; double xs[na], jval[nnz], anc[na],
// xnc[na+1]; uint8 jflag[nnz]; with a tile double T[na * tile_rows] (na columns of tile_rows rows),
// rinv[tile_rows], int perm[tile_rows]; a mixed-precision tile adds float T32[na * tile_rows], rinv32[tile_rows] and double
// srow[tile_rows], scol[tile_rows]. Every array 16-byte aligned.
NUPPN_HD inline size_t act_bytes(int na, int nnz, int nwarps, int tile_rows, bool mixed = false) {
  size_t b = a16((size_t)(na + 1) * 4) + 4 * a16((size_t)na * 4) + 2 * a16((size_t)nnz * 4);
  if (tile_rows == 0) b += a16((size_t)nnz * 8) + a16((size_t)nwarps * na * 8) + a16((size_t)na * 8);
  b += a16((size_t)na * 8);
  b += a16((size_t)nnz * 8) + a16((size_t)na * 8) + a16((size_t)(na + 1) * 8) + a16((size_t)nnz);
  b += (size_t)na * tile_rows * 8 + (size_t)tile_rows * 8;
  if (tile_rows > 0) b += a16((size_t)tile_rows * 4);  // row permutation of the pivoted tile
  if (mixed && tile_rows > 0) b += (size_t)na * tile_rows * 4 + a16((size_t)tile_rows * 4) + 2 * (size_t)tile_rows * 8;
  return b;
}

// Largest act_bytes over every active system of a network with nsys rows and nnz filled entries.
NUPPN_HD inline size_t act_bytes_max(int nsys, int nnz, int nwarps) {
  const int nt = nsys < kTileMax ? nsys : kTileMax;
  size_t full = act_bytes(nsys, nnz, nwarps, 0);
  size_t tile = act_bytes(nt, nt * nt < nnz ? nt * nt : nnz, nwarps, nt <= 32 ? 32 : 64, true);
  return full > tile ? full : tile;
}

// Bytes of the restricted right-hand side for na rows and ngi gather items:
// int gptr[na+1]; float gcoef[ngi]; uint32 grpk[ngi]; double grcv[ngi], gterm[ngi].
NUPPN_HD inline size_t rhs_bytes(int na, int ngi) {
  return a16((size_t)(na + 1) * 4) + 2 * a16((size_t)ngi * 4) + 2 * a16((size_t)ngi * 8);
}

// Serving queue of the device-resident request loop (nuppn_serve_*). Request seq uses slot
// seq % nslots. The host writes its inputs into that slot of device memory (RingIn, x_in, grid) with
// asynchronous copies on one stream, then advances `published` (a device counter) with a copy on the
// same stream, so a request is complete in device memory before it is published. Groups of the
// persistent kernel claim requests in order (claimed, an atomic counter), integrate them and write
// the results to host-mapped memory (RingOut, x_out); RingOut::done = seq + 1 tells the host that
// they are there. The host reuses a slot only after its request is done.
struct RingIn {
  long long seq;       // request number
  int kind, npts, bd, pad;  // kind 0: one integrate_network interval, 1: a tppnp trajectory
  double t9_0, t9_1, rho_0, rho_1, ye, dtwant;
};
struct RingOut {
  long long done;      // seq + 1 once the outputs are written
  int ierr, fail, bd, pad;
  double ye;
  nuppn_zone_stats st;
};
struct ServeQueue {
  const RingIn *in;              // [nslots] device
  RingOut *out;                  // [nslots] host-mapped
  const double *x_in;            // [nslots][nsp] device
  double *x_out;                 // [nslots][nsp] host-mapped
  const double *grid;            // [nslots][3][npts_max] device: time, T9, rho
  const long long *published;    // device: requests published so far
  unsigned long long *claimed;   // device: requests claimed so far
  const int *stop;               // device: nonzero = leave when idle
  int nslots, npts_max;
  int idle_polls;                // empty polls (with a growing sleep, up to ~8 us) before a group leaves
};

// arguments of the persistent integration kernel
struct IntegrateArgs {
  int nz, ldx;
  double *X;
  const double *t9_0, *t9_1, *rho_0, *rho_1, *dtwant;
  double *ye;
  int *ierr;
  nuppn_zone_stats *stats;
  int *bd_state;
  int *counter;
  // zone schedule: the k-th zone taken is order[k] (costliest first, see k_zone_order), or k if null
  const int *order;
  // trajectory mode (npts > 0): per zone npts points of time, T9 and rho ([nz][npts]); tr_fail gets
  // the index of the interval that failed, or -1
  int npts;
  const double *tr_time, *tr_t9, *tr_rho;
  int *tr_fail;
  // serving (queue.in != nullptr, trajectory instantiation): requests come from the queue instead of
  // the arrays above, each a single interval or a trajectory
  ServeQueue queue;
  // several networks in one launch (k_integrate_multi): zone z uses nets[net_of[z]], lays[net_of[z]]
  const DevNet *nets;
  const WsLayout *lays;
  const int *net_of;
  int nnets;
  size_t slab;                   // bytes of each CTA's workspace slab
};

// arguments of the single-phase parity kernel
struct PhaseArgs {
  int nz, ldx, op;  // op: 0 rates, 1 dxdt, 2 jacobian, 3 reduced solve, 4 NSE distribution
  const double *X, *t9, *rho, *ye, *v_in, *dt, *jac_in, *b;
  const uint8_t *eset_in, *mask_in;
  double *out_v, *out_dxdt, *out_jac, *out_x;
  uint8_t *out_eset, *out_mask;
  double *out_mu_p, *out_mu_n;
  int *out_iters, *out_ierr;
};

}  // namespace nuppn
