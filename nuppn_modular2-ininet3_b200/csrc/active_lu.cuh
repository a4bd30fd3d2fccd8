// active_lu.cuh -- the dynamic network's active subsystem (included by solver.cu).
//
// The reference solves only the species its dynamic network selects (jac_rhs.F90:134-197: mask,
// pack, then SuperLU on the reduced matrix, with a new COLAMD/symbolic analysis every time). Here the
// fill-reducing order and the filled pattern are computed once for the whole network (net_host.cpp);
// the filled pattern restricted to the active rows and columns contains the fill of the active
// submatrix in that order, so each zone only has to compact it (once per Jacobian) and can then
// factor and solve it with no symbolic work. Compacted structures live in shared memory when they
// fit the CTA's budget and in the CTA's global workspace otherwise.
//
// Per Jacobian (dev_jacobian_mask, then):
//   dev_compact          active rows and the restricted filled pattern
//   dev_jacobian_active  Jacobian values and entry flags of the active entries (all reactions)
//   dev_compact_rhs      per-species gather items of the right-hand side (all reactions)
// Per factorization / right-hand side / solve: dev_factor_active, dev_dxdt_active, dev_solve_active,
// all on compact vectors indexed by the active row number c. Systems of up to kTileMax rows (the
// usual case: a few tens of species) are factored as a dense tile and solved with rows held in the
// registers of one warp; larger ones use the sparse row-oriented factorization.
#pragma once

NUPPN_BEGIN

constexpr int kSpinLimit = 1 << 22;  // per wait; a timeout marks the zone as failed, never hangs

// Sparse active subsystems up to kOneWarpFactorMax rows are factored, and up to kOneWarpMax rows
// solved, by one warp row after row with no inter-warp flags; larger ones by all warps with per-row
// ready flags (for large systems the factorization has more independent work per row than the
// solves, so it leaves one warp sooner).
constexpr int kOneWarpFactorMax = 192;
constexpr int kOneWarpMax = 512;

// Flags of a compact LU position (jflag): entry set, diagonal, fill (no Jacobian entry).
enum : uint8_t { JF_SET = 1, JF_DIAG = 2, JF_FILL = 4 };

// Flag of a right-hand side item (grpk) that is a group of reactions with a frozen reactant.
constexpr uint32_t kGroupItem = 1u << 31;

struct Act {
  int na, nnz;
  int *crp, *cdiag, *arow, *flagF, *flagS, *ccol, *csrc;
  bool onewarp;      // sparse solve by one warp
  bool onewarp_f;    // sparse factorization by one warp
  bool tile;         // tile_rows > 0
  int tile_rows;     // 0, 32 or 64: dense tile factorization, register-resident solve
  double *cval, *xs, *wbuf;  // sparse path only: L\U values in CSR order, multi-warp scratch
  double *rdg;       // sparse path only: 1 / U(c, c) of each factored row
  double *jval;      // [nnz] Jacobian value of each position (the reference's 1e-99 + contributions)
  uint8_t *jflag;    // [nnz] JF_* flags; JF_SET is cleared when a level drops the entry
  double *anc;       // [na] mass number of active row c
  double *xnc;       // [na+1] molar abundances of the active rows; xnc[na] = 1 (gamma)
  double *T, *rinv;  // tile: T[c*tile_rows + r] = entry (r, c) of L\U; rinv[r] = 1 / U(r, r)
  int *perm;         // tile: original row at each position of the pivoted factor (P b = b[perm])
  // mixed precision (lu_precision = 1, tile systems): T keeps I - hJ unfactored in FP64 for the
  // refinement residuals; T32 / rinv32 hold the FP32 factor of diag(srow) (I - hJ) diag(scol)
  bool mixed;        // the tile has the mixed-precision arrays
  bool mixed_now;    // the current factorization is the FP32 one (false after an FP32 pivot failure)
  float *T32, *rinv32;
  double *srow, *scol;
  int ir_max;        // knobs ir_max_iters, ir_rtol
  double ir_rtol;
  int genF, genS;
  bool in_smem;
  // right-hand side restricted to the dynamic network (see dev_compact_rhs)
  int ngi;
  int *gptr;         // [na+1] gather items of active row c: gptr[c] .. gptr[c+1]-1
  float *gcoef;      // [ngi] term coefficient (-k2, -1, k6 or k8)
  uint32_t *grpk;    // [ngi] compact index of reactant 1 | reactant 2 (na = gamma) << 14 | k2 << 28 | group flag << 31
  double *grcv;      // [ngi] (1/k2!) * rate of the term's reaction (a group's constant: see below)
  double *gterm;     // [ngi] term values of the current sub-step
  bool rhs_in_smem;
};

__device__ __forceinline__ void act_bind(Act &A, char *base, int na, int nnz, int nwarps, int tile_rows, bool mixed) {
  char *p = base;
  A.crp = (int *)p; p += a16((size_t)(na + 1) * 4);
  A.cdiag = (int *)p; p += a16((size_t)na * 4);
  A.arow = (int *)p; p += a16((size_t)na * 4);
  A.flagF = (int *)p; p += a16((size_t)na * 4);
  A.flagS = (int *)p; p += a16((size_t)na * 4);
  A.ccol = (int *)p; p += a16((size_t)nnz * 4);
  A.csrc = (int *)p; p += a16((size_t)nnz * 4);
  if (tile_rows == 0) {
    A.cval = (double *)p; p += a16((size_t)nnz * 8);
    A.wbuf = (double *)p; p += a16((size_t)nwarps * na * 8);
    A.rdg = (double *)p; p += a16((size_t)na * 8);
  } else {
    A.cval = nullptr;
    A.wbuf = nullptr;
    A.rdg = nullptr;
  }
  A.xs = (double *)p; p += a16((size_t)na * 8);
  A.jval = (double *)p; p += a16((size_t)nnz * 8);
  A.anc = (double *)p; p += a16((size_t)na * 8);
  A.xnc = (double *)p; p += a16((size_t)(na + 1) * 8);
  A.jflag = (uint8_t *)p; p += a16((size_t)nnz);
  A.tile_rows = tile_rows;
  A.tile = tile_rows > 0;
  if (A.tile) {
    A.T = (double *)p; p += (size_t)na * tile_rows * 8;
    A.rinv = (double *)p; p += (size_t)tile_rows * 8;
    A.perm = (int *)p; p += a16((size_t)tile_rows * 4);
  } else {
    A.T = nullptr;
    A.rinv = nullptr;
    A.perm = nullptr;
  }
  A.mixed = mixed && A.tile;
  A.mixed_now = false;
  if (A.mixed) {
    A.T32 = (float *)p; p += (size_t)na * tile_rows * 4;
    A.rinv32 = (float *)p; p += a16((size_t)tile_rows * 4);
    A.srow = (double *)p; p += (size_t)tile_rows * 8;
    A.scol = (double *)p;
  } else {
    A.T32 = nullptr;
    A.rinv32 = nullptr;
    A.srow = A.scol = nullptr;
  }
}

// Exclusive scan of v[0..n) in place (block-wide, deterministic); returns the total. Each warp takes
// a contiguous segment and walks it 32 elements at a time, so every load and store is coalesced.
__device__ int block_scan_excl(int *v, int n, int *sint) {
  const int lane = GT & 31, w = GT >> 5, nw = GN >> 5;
  const int seg = (n + nw - 1) / nw, b0 = min(n, w * seg), b1 = min(n, b0 + seg);
  int tot = 0;
  for (int i = b0 + lane; i < b1; i += 32) tot += v[i];
  for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(NUPPN_FULL, tot, o);
  GSYNC();  // sint may still be read by the previous scan
  if (lane == 0) sint[w] = tot;
  GSYNC();
  int base = 0, total = 0;
  for (int i = 0; i < nw; ++i) {
    if (i < w) base += sint[i];
    total += sint[i];
  }
  for (int i0 = b0; i0 < b1; i0 += 32) {
    const int i = i0 + lane;
    const int x = i < b1 ? v[i] : 0;
    int incl = x;
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(NUPPN_FULL, incl, o);
      if (lane >= o) incl += t;
    }
    if (i < b1) v[i] = base + incl - x;
    base += __shfl_sync(NUPPN_FULL, incl, 31);
  }
  GSYNC();
  return total;
}

// Segment of flattened position t, given exclusive segment offsets off[0..n] (off[n] = total).
__device__ __forceinline__ int seg_of(const int *off, int n, int t) {
  int lo = 0, hi = n;  // off[lo] <= t < off[hi]
  while (hi - lo > 1) {
    int m = (lo + hi) >> 1;
    if (off[m] <= t) lo = m; else hi = m;
  }
  return lo;
}

__device__ __forceinline__ bool spin_until(const int *flag, int gen) {
  const volatile int *f = flag;
  int it = 0;
  while (*f < gen) {
    if (++it > kSpinLimit) return false;
    __nanosleep(32);  // leave issue slots to the warp that owns the row being waited for
  }
  __threadfence_block();
  return true;
}

// Compact the active subsystem after the mask is known. smem/smem_bytes: the CTA's budget.
__device__ void dev_compact(const DevNet &N, const Ws &W, Act &A, char *smem, size_t smem_bytes, int *sint) {
  const int tid = GT, nt = GN, lane = tid & 31, w = tid >> 5, nw = nt >> 5;
  int *sys2c = W.act_tmp;                  // [nsys]
  int *tmp_arow = W.act_tmp + N.nsys + 1;  // [nsys]
  int *cnt = W.act_tmp + 2 * (N.nsys + 1); // [nsys+1]
  for (int i = tid; i < N.nsys; i += nt) sys2c[i] = W.mask[N.sp_of_sys[i]] ? 1 : 0;
  GSYNC();
  const int na = block_scan_excl(sys2c, N.nsys, sint);
  for (int i = tid; i < N.nsys; i += nt) {
    if (W.mask[N.sp_of_sys[i]]) tmp_arow[sys2c[i]] = i;
    else sys2c[i] = -1;
  }
  GSYNC();
  for (int c = w; c < na; c += nw) {  // entries per active row: static entries in active columns
    int i = tmp_arow[c], n = 0;
    for (int p = N.lu_rowptr[i] + lane; p < N.lu_rowptr[i + 1]; p += 32) n += sys2c[N.lu_col[p]] >= 0;
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(NUPPN_FULL, n, o);
    if (lane == 0) cnt[c] = n;
  }
  GSYNC();
  const int nnz = block_scan_excl(cnt, na, sint);
  const int trows = tile_rows_for(na, N.kn.lu_tile_max);
  const bool mixed = N.kn.lu_precision == 1 && trows > 0;
  const size_t need = act_bytes(na, nnz, nw, trows, mixed);
  A.na = na;
  A.nnz = nnz;
  A.in_smem = need <= smem_bytes;
  act_bind(A, A.in_smem ? smem : W.act, na, nnz, nw, trows, mixed);
  A.ir_max = N.kn.ir_max_iters;
  A.ir_rtol = N.kn.ir_rtol;
  A.genF = 0;
  A.genS = 0;
  for (int c = tid; c < na; c += nt) {
    A.crp[c] = cnt[c];
    A.arow[c] = tmp_arow[c];
    A.flagF[c] = 0;
    A.flagS[c] = 0;
    A.anc[c] = N.an[N.sp_of_sys[tmp_arow[c]]];
  }
  if (tid == 0) {
    A.crp[na] = nnz;
    A.xnc[na] = 1.0;  // gamma's molar abundance
  }
  for (int c = w; c < na; c += nw) {
    int i = tmp_arow[c], base = cnt[c];
    for (int p0 = N.lu_rowptr[i]; p0 < N.lu_rowptr[i + 1]; p0 += 32) {
      int p = p0 + lane;
      int col = p < N.lu_rowptr[i + 1] ? N.lu_col[p] : -1;
      int cc = col >= 0 ? sys2c[col] : -1;
      unsigned m = __ballot_sync(NUPPN_FULL, cc >= 0);
      if (cc >= 0) {
        int pos = base + __popc(m & ((1u << lane) - 1u));
        A.ccol[pos] = cc;
        A.csrc[pos] = p;
        if (col == i) A.cdiag[c] = pos;
      }
      base += __popc(m);
    }
  }
  GSYNC();
  A.onewarp = na <= (N.kn.lu_onewarp_max > 0 ? N.kn.lu_onewarp_max : kOneWarpMax);
  A.onewarp_f = na <= (N.kn.lu_onewarp_max > 0 ? N.kn.lu_onewarp_max : kOneWarpFactorMax);
}

// One reaction's contribution to Jacobian slot s (jac_rhs.F90:355-392) and whether it sets the
// entry (jac_rhs.F90:399-436) under the growing-mask rule. Needs W.flux[a] (rate test), W.xn, first_l.
__device__ __forceinline__ double jac_contrib(const DevNet &N, const Ws &W, int a, int s, bool &set) {
  set = false;
  if (W.flux[a] == 0.0) return 0.0;
  const int g = N.ig;
  const int *k = N.act_k + (size_t)a * 8;
  const int in1 = k[0], Nin1 = k[1], in2 = k[2], Nin2 = k[3], out1 = k[4], Nout1 = k[5], out2 = k[6], Nout2 = k[7];
  const double v = W.v[N.act_slot[a]], y1 = W.xn[in1], y2 = W.xn[in2];
  const double ain1 = N.an[in1], ain2 = N.an[in2], aout1 = N.an[out1], aout2 = N.an[out2];
  bool cond;
  double d;
  if (s < 4) {
    const double stem = (double)Nin1 * c_fact[Nin1] * c_fact[Nin2] * powi(y2, Nin2) * powi(y1, Nin1 - 1) * v;
    switch (s) {
      case 0: cond = in1 != g; d = (double)(-Nin1) * stem * ain1 / ain1; break;
      case 1: cond = in1 != g && in2 != g; d = (double)(-Nin2) * stem * ain2 / ain1; break;
      case 2: cond = in1 != g && out1 != g; d = (double)Nout1 * stem * aout1 / ain1; break;
      default: cond = in1 != g && out2 != g; d = (double)Nout2 * stem * aout2 / ain1; break;
    }
  } else {
    const double stem = (double)Nin2 * c_fact[Nin1] * c_fact[Nin2] * powi(y1, Nin1) * powi(y2, Nin2 - 1) * v;
    switch (s) {
      case 4: cond = in1 != g && in2 != g; d = (double)(-Nin1) * stem * ain1 / ain2; break;
      case 5: cond = in2 != g; d = (double)(-Nin2) * stem * ain2 / ain2; break;
      case 6: cond = in2 != g && out1 != g; d = (double)Nout1 * stem * aout1 / ain2; break;
      default: cond = in2 != g && out2 != g; d = (double)Nout2 * stem * aout2 / ain2; break;
    }
  }
  if (!cond) return 0.0;
  set = (in2 == g || W.first_l[in2] <= a) && (out1 == g || W.first_l[out1] <= a) && W.first_l[in1] <= a &&
        W.first_l[out2] <= a;
  return d;
}

// Jacobian values (1e-99 + the contributions of every reaction that passes the rate test, masked
// reactants or not, as in the reference) and entry flags for the positions of the active subsystem.
// Runs after dev_compact_rhs. Entries with short static gather lists are evaluated as one flattened,
// block-parallel list and summed by one thread each in the list's order from 1e-99 (the reference's
// accumulation: jac = 1e-99, then += each contribution in reaction order, jac_rhs.F90:309-392).
// The few with long lists (among n, p and alpha: every capture on every nucleus) take the reactions
// whose other reactant is masked or gamma from their list, in pieces of kRhsPiece items (a warp
// sums a piece, lane-strided and then by a fixed butterfly; each entry adds its pieces in order),
// and the reactions with a frozen other reactant from the right-hand side's groups: a group of row i
// with varying factor xn_j^p and constant G contributes d/dxn_j (G xn_j^p) = p G xn_j^(p-1), times
// A_i / A_j, to entry (i, j), which is the sum of those reactions' contributions in the reference
// (their stems, jac_rhs.F90:346-353, with k4 = 1 or k3 = gamma), added in another order. Such a
// reaction never sets an entry (its frozen reactant is never masked, jac_rhs.F90:399-436).
__device__ void dev_jacobian_active(const DevNet &N, const Ws &W, Act &A, int *sint) {
  const int tid = GT, nt = GN, lane = tid & 31, w = tid >> 5, nw = nt >> 5, nnz = A.nnz;
  const int *spc = W.rhs_spc;             // species -> active row (dev_compact_rhs), -1 if frozen
  int *off = W.act_otmp;                  // [nnz+1] short entries' items, then offsets
  int *lfl = W.jac_long;                  // [nnz+1] long-entry flags, then their ranks
  int *lst = W.jac_long + (N.nnzLU + 1);  // [nlong] positions of the long entries, in order
  int *poff = lst + N.nnzLU;              // [nlong+1] their first pieces
  for (int p = tid; p < nnz; p += nt) {
    const int e = N.lu_src[A.csrc[p]];
    const int len = e >= 0 ? N.jg_ptr[e + 1] - N.jg_ptr[e] : 0;
    const bool lng = len > kLongList;
    off[p] = lng ? 0 : len;
    lfl[p] = lng ? 1 : 0;
  }
  GSYNC();
  const int T = block_scan_excl(off, nnz, sint);  // <= the network's jg items: distinct entries
  const int nlong = block_scan_excl(lfl, nnz, sint);
  if (tid == 0) {
    off[nnz] = T;
    lfl[nnz] = nlong;
  }
  GSYNC();
  for (int p = tid; p < nnz; p += nt) {
    if (lfl[p + 1] == lfl[p]) continue;
    const int e = N.lu_src[A.csrc[p]];
    lst[lfl[p]] = p;
    poff[lfl[p]] = (N.jg_ptr[e + 1] - N.jg_ptr[e] + kRhsPiece - 1) / kRhsPiece;
  }
  GSYNC();
  const int NPc = block_scan_excl(poff, nlong, sint);
  if (tid == 0) poff[nlong] = NPc;
  GSYNC();
  double *dv = W.act_dtmp;   // [T] short entries' contributions, then [NPc] long pieces' sums
  uint8_t *sf = W.act_btmp;  // their entry-set flags
  for (int t = tid; t < T; t += nt) {
    const int p = seg_of(off, nnz, t);
    const int e = N.lu_src[A.csrc[p]];
    const int it = N.jg_item[N.jg_ptr[e] + (t - off[p])];
    bool set;
    dv[t] = jac_contrib(N, W, it >> 3, it & 7, set);
    sf[t] = set ? 1 : 0;
  }
  for (int Q = w; Q < NPc; Q += nw) {
    const int L = seg_of(poff, nlong, Q);
    const int e = N.lu_src[A.csrc[lst[L]]];
    const int *items = N.jg_item + N.jg_ptr[e];
    const int t0 = (Q - poff[L]) * kRhsPiece, t1 = min(t0 + kRhsPiece, N.jg_ptr[e + 1] - N.jg_ptr[e]);
    const int *oth = N.jg_oth + N.jg_ptr[e];
    double acc = 0.0;
    int set = 0;
    for (int t = t0 + lane; t < t1; t += 32) {
      const int o = oth[t];
      if (o >= 0 && spc[o] < 0) continue;  // a frozen other reactant: in the groups below
      const int it = items[t];
      bool st;
      acc += jac_contrib(N, W, it >> 3, it & 7, st);
      set |= st ? 1 : 0;
    }
    for (int o = 16; o > 0; o >>= 1) {
      acc += __shfl_xor_sync(NUPPN_FULL, acc, o);
      set |= __shfl_xor_sync(NUPPN_FULL, set, o);
    }
    if (lane == 0) {
      dv[T + Q] = acc;
      sf[T + Q] = (uint8_t)set;
    }
  }
  GSYNC();
  for (int p = tid; p < nnz; p += nt) {
    const int e = N.lu_src[A.csrc[p]];
    if (e < 0) {
      A.jval[p] = 0.0;
      A.jflag[p] = JF_FILL;
      continue;
    }
    double acc;
    int set = 0;
    if (lfl[p + 1] > lfl[p]) {
      const int L = lfl[p];
      double sum = 0.0;
      for (int Q = poff[L]; Q < poff[L + 1]; ++Q) {
        sum += dv[T + Q];
        set |= sf[T + Q];
      }
      const int r = seg_of(A.crp, A.na, p), cj = A.ccol[p];
      const double y = W.xn[N.sp_of_sys[A.arow[cj]]], ar = A.anc[r], ac = A.anc[cj];
      for (int q = A.gptr[r]; q < A.gptr[r + 1]; ++q) {  // the row's groups varying with xn_j
        const uint32_t pk = A.grpk[q];
        if (!(pk & kGroupItem) || (int)(pk & 0x3fff) != cj) continue;
        const int pw = (int)((pk >> 28) & 7);
        sum += (((double)pw * A.grcv[q] * powi(y, pw - 1)) * ar) / ac;
      }
      acc = 1.e-99 + sum;
    } else {
      acc = 1.e-99;
      for (int t = off[p]; t < off[p + 1]; ++t) {
        acc = acc + dv[t];
        set |= sf[t];
      }
    }
    A.jval[p] = acc;
    A.jflag[p] = (uint8_t)((set ? JF_SET : 0) | (N.jdiag[N.jrow[e]] == e ? JF_DIAG : 0));
  }
  GSYNC();
}

// Jacobian values and flags of the compact positions from a full Jacobian in W.jac / W.eset (the
// reduced-solve parity entry point supplies them instead of dev_jacobian_active).
__device__ void dev_load_active_jacobian(const DevNet &N, const Ws &W, Act &A) {
  for (int p = GT; p < A.nnz; p += GN) {
    const int e = N.lu_src[A.csrc[p]];
    if (e < 0) {
      A.jval[p] = 0.0;
      A.jflag[p] = JF_FILL;
    } else {
      A.jval[p] = W.jac[e];
      A.jflag[p] = (uint8_t)((W.eset[e] ? JF_SET : 0) | (N.jdiag[N.jrow[e]] == e ? JF_DIAG : 0));
    }
  }
  GSYNC();
}

// Entry p of I - hJ under reduce_jacobian's rules (jac_rhs.F90:97-140): an entry that was set but
// scales to 0 or -1 is dropped for the rest of this Jacobian's levels; the diagonal of every active
// row is set and gets the identity added.
__device__ __forceinline__ double assemble_entry(Act &A, int p, double h) {
  const uint8_t f = A.jflag[p];
  if (f & JF_FILL) return 0.0;
  double v = A.jval[p] * (-h);
  bool set = (f & JF_SET) != 0;
  if (set && (fabs(v) == 0.0 || v == -1.0)) {
    set = false;
    A.jflag[p] = (uint8_t)(f & ~JF_SET);
  }
  if (f & JF_DIAG) {
    set = true;
    A.jflag[p] = (uint8_t)(A.jflag[p] | JF_SET);
    v = v + 1.0;
  }
  return set ? v : 0.0;
}

__device__ __forceinline__ bool pivot_ok(double d) { return d != 0.0 && isfinite(d); }
__device__ __forceinline__ bool pivot_ok(float d) { return d != 0.0f && isfinite(d); }

// Right-looking elimination of a dense tile by all warps of the group, with row pivoting. At pivot k
// every warp finds the pivot row of column k by SuperLU's threshold rule with u = 1 (dpivotL.c:
// the diagonal when no entry below it is larger in magnitude, else the first largest), the rows are
// exchanged across all columns (perm tracks which original row sits at each position, so that a
// right-hand side b is solved as P b), then every warp forms the multipliers l_r = a_rk / a_kk of the
// rows below in registers (lane l owns rows l + 32 i) and updates its share of the trailing columns
// (m = k+1+w, step nw). Column k is left unscaled during the elimination and scaled at the end by the
// stored reciprocal, the same product a_rk * (1 / a_kk) that SuperLU forms (dpivotL.c:178-180).
// Without pivoting, I - hJ of a large step is not diagonally dominant, and the small components of
// the solution (species depleted by many orders of magnitude) lose their relative accuracy.
// Returns false on a zero or non-finite pivot.
// F = double for the FP64 factor; F = float for the FP32 factor of the mixed-precision mode.
template <int R, typename F = double>
__device__ bool tile_factor_block(F *T, F *rinv, int *perm, int na) {
  constexpr int S = 32 * R;
  const int lane = GT & 31, w = GT >> 5, nw = GN >> 5;
  int bad = 0;
  for (int r = GT; r < na; r += GN) perm[r] = r;
  GSYNC();
  for (int k = 0; k < na; ++k) {
    // pivot row: the same search in every warp (rows k .. na-1 of column k)
    F best = F(-1);
    int bi = k;
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int r = lane + 32 * i;
      if (r >= k && r < na) {
        const F a = fabs(T[k * S + r]);
        if (a > best) { best = a; bi = r; }
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const F ob = __shfl_xor_sync(NUPPN_FULL, best, o);
      const int oi = __shfl_xor_sync(NUPPN_FULL, bi, o);
      if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    const int pr = fabs(T[k * (S + 1)]) >= best ? k : bi;
    GSYNC();  // every warp has read column k (so every warp found the same pivot row) before any swap
    if (pr != k) {  // exchange rows k and pr in every column
      for (int c = GT; c < na; c += GN) {
        const F t = T[c * S + k];
        T[c * S + k] = T[c * S + pr];
        T[c * S + pr] = t;
      }
      if (GT == 0) {
        const int t = perm[k];
        perm[k] = perm[pr];
        perm[pr] = t;
      }
      GSYNC();
    }
    const F piv = T[k * (S + 1)];
    bad |= !pivot_ok(piv);
    const F rp = F(1) / piv;
    if (GT == 0) rinv[k] = rp;
    F l[R];
    bool any = false;
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int r = lane + 32 * i;
      l[i] = F(0);
      if (r > k && r < na) {
        const F a = T[k * S + r];
        l[i] = a != F(0) ? a * rp : F(0);
      }
      any |= l[i] != F(0);
    }
    if (__any_sync(NUPPN_FULL, any)) {
#pragma unroll 2
      for (int m = k + 1 + w; m < na; m += nw) {
        const F u = T[m * S + k];
#pragma unroll
        for (int i = 0; i < R; ++i)
          if (l[i] != F(0)) T[m * S + lane + 32 * i] -= l[i] * u;
      }
    }
    GSYNC();
  }
  for (int i = GT; i < na * S; i += GN) {  // L columns: a_rk * (1 / a_kk)
    const int c = i / S, r = i - c * S;
    if (r > c && r < na) {
      const F a = T[i];
      if (a != F(0)) T[i] = a * rinv[c];
    }
  }
  return g_or(bad) == 0;
}

// Right-hand side of the calling warp (rows lane + 32 i in x) into the factor's row order: x_r becomes
// b_perm[r] (P b). scratch: na doubles no one else uses meanwhile.
template <int R, typename F>
__device__ __forceinline__ void tile_permute_rhs(F (&x)[R], const int *perm, int na, double *scratch, int lane) {
#pragma unroll
  for (int i = 0; i < R; ++i)
    if (lane + 32 * i < na) scratch[lane + 32 * i] = (double)x[i];
  __syncwarp();
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int r = lane + 32 * i;
    x[i] = r < na ? (F)scratch[perm[r]] : F(0);
  }
  __syncwarp();
}

// Power of two that brings |m| into [1, 2) (1 for 0 or non-finite m).
__device__ __forceinline__ double pow2_scale(double m) {
  return (m > 0.0 && isfinite(m)) ? ldexp(1.0, -ilogb(m)) : 1.0;
}

// Mixed-precision factorization of the assembled tile T (I - hJ, FP64, left unfactored): columns,
// then rows, are scaled by powers of two to a largest entry in [1, 2) (exact in FP64; active
// systems hold entries from ~1e-99 to ~1e110, beyond FP32's range), the scaled matrix is rounded to
// FP32 and factored there. Entries that underflow FP32 become zeros of the FP32 factor only; the
// FP64 residuals of the refinement still see them. Returns false on a zero or non-finite FP32 pivot.
template <int R>
__device__ bool tile_factor_mixed(Act &A, int na) {
  constexpr int S = 32 * R;
  const int tid = GT, nt = GN, lane = tid & 31, w = tid >> 5, nw = nt >> 5;
  const double *T = A.T;
  for (int c = w; c < na; c += nw) {  // column scales (columns are contiguous)
    double m = 0.0;
    for (int r = lane; r < na; r += 32) m = fmax(m, fabs(T[c * S + r]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(NUPPN_FULL, m, o));
    if (lane == 0) A.scol[c] = pow2_scale(m);
  }
  GSYNC();
  for (int r = tid; r < na; r += nt) {  // row scales of the column-scaled matrix
    double m = 0.0;
    for (int c = 0; c < na; ++c) m = fmax(m, fabs(T[c * S + r]) * A.scol[c]);
    A.srow[r] = pow2_scale(m);
  }
  GSYNC();
  for (int i = tid; i < na * S; i += nt) {
    const int c = i / S, r = i - c * S;
    A.T32[i] = r < na ? (float)(T[i] * A.scol[c] * A.srow[r]) : 0.0f;
  }
  GSYNC();
  return tile_factor_block<R, float>(A.T32, A.rinv32, A.perm, na);
}

// Forward and backward substitution of a factored tile by one warp, x[i] holding row lane + 32 i.
// Columns go in blocks of four: every lane loads the block's entries of its rows first (they do not
// depend on x), forms the block's four final values from four broadcasts (the small triangle solved
// redundantly), then applies the four columns to its rows. Each row sees exactly the operations of
// the column-by-column order (column-oriented, like SuperLU's dgstrs; a zero entry is skipped); the
// diagonal is divided out (div_piv, from the reciprocal the factorization stored).
template <int R, typename F>
__device__ __forceinline__ F tile_row(const F (&x)[R], int r) {
  return (R == 1 || r < 32) ? x[0] : x[R - 1];
}

__device__ __forceinline__ double sub_nz(double x, double a, double v) {  // x - a*v, skipped for a == 0
  const double t = x - a * v;
  return a != 0.0 ? t : x;
}
__device__ __forceinline__ float sub_nz(float x, float a, float v) {
  const float t = x - a * v;
  return a != 0.0f ? t : x;
}

// a / d rounded to nearest, as SuperLU's triangular solve divides by U(c, c) (dgstrs.c:248,
// dmyblas2.c:139), formed from r = 1 / d (itself a rounded division) by one correction step of
// Markstein's method (P. Markstein, IBM J. Res. Develop. 34(1), 1990): q0 = a r is within an ulp of
// a / d, the residual e = a - d q0 is exact under an FMA, and q0 + e r is the correctly rounded
// quotient. The theorem needs the residual exact and every intermediate normal, which holds for a,
// q0 and d within [1e-280, 1e280] (the residual is exact down to |a| ~ 1e-292); a = +0 gives the
// right signed zero as well. Otherwise `bad` is raised (a test off the dependency chain) and the
// caller repeats the solve with plain division; -0 goes that way too (the correction would return
// +0 for -0 / d, d > 0). Multiplying by r alone differs from the quotient by an ulp now and then,
// which is enough to change the step control of an ill-conditioned system (a 1e10-scale
// cancellation of rows holding U entries near 1e109 against x near 1e-99).
template <bool kPlain>
__device__ __forceinline__ float div_piv(float a, float d, float r, int &) {  // FP32 factor: refined
  return a * r;
}
template <bool kPlain>
__device__ __forceinline__ double div_piv(double a, double d, double r, int &bad) {
  if (kPlain) return a / d;
  const double q0 = a * r;
  const double e = fma(-d, q0, a);
  const double m = fabs(q0), n = fabs(a), dd = fabs(d);
  const bool ok = (m > 1e-280 && m < 1e280 && n > 1e-280 && n < 1e280) || (a == 0.0 && !signbit(a));
  bad |= !(ok && dd > 1e-280 && dd < 1e280);
  return fma(e, r, q0);
}

template <int R, bool kPlain, typename F = double>
__device__ __forceinline__ void tile_solve_core(const F *T, const F *rinv, int na, F (&x)[R], const F (&ri)[R],
                                                int lane, int &bad) {
  constexpr int S = 32 * R;
  int c = 0;
  for (; c + 4 < na; c += 4) {  // forward, columns c .. c+3 (the last column has no entries below)
    F a[R][4];
#pragma unroll
    for (int i = 0; i < R; ++i)
#pragma unroll
      for (int k = 0; k < 4; ++k) a[i][k] = T[(c + k) * S + lane + 32 * i];
    const F l10 = T[c * S + c + 1], l20 = T[c * S + c + 2], l30 = T[c * S + c + 3];
    const F l21 = T[(c + 1) * S + c + 2], l31 = T[(c + 1) * S + c + 3], l32 = T[(c + 2) * S + c + 3];
    const F v0 = __shfl_sync(NUPPN_FULL, tile_row<R>(x, c), c & 31);
    const F u1 = __shfl_sync(NUPPN_FULL, tile_row<R>(x, c + 1), (c + 1) & 31);
    const F u2 = __shfl_sync(NUPPN_FULL, tile_row<R>(x, c + 2), (c + 2) & 31);
    const F u3 = __shfl_sync(NUPPN_FULL, tile_row<R>(x, c + 3), (c + 3) & 31);
    const F v1 = sub_nz(u1, l10, v0);
    const F v2 = sub_nz(sub_nz(u2, l20, v0), l21, v1);
    const F v3 = sub_nz(sub_nz(sub_nz(u3, l30, v0), l31, v1), l32, v2);
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int r = lane + 32 * i;
      const F t = sub_nz(sub_nz(sub_nz(sub_nz(x[i], a[i][0], v0), a[i][1], v1), a[i][2], v2), a[i][3], v3);
      x[i] = r == c + 1 ? v1 : r == c + 2 ? v2 : r == c + 3 ? v3 : (r > c + 3 ? t : x[i]);
    }
  }
  for (; c < na - 1; ++c) {
    F a[R];
#pragma unroll
    for (int i = 0; i < R; ++i) a[i] = T[c * S + lane + 32 * i];
    const F xc = __shfl_sync(NUPPN_FULL, tile_row<R>(x, c), c & 31);
#pragma unroll
    for (int i = 0; i < R; ++i)
      if (lane + 32 * i > c) x[i] = sub_nz(x[i], a[i], xc);
  }
  c = na - 1;
  for (; c >= 3; c -= 4) {  // backward, columns c, c-1, c-2, c-3
    F a[R][4];
#pragma unroll
    for (int i = 0; i < R; ++i)
#pragma unroll
      for (int k = 0; k < 4; ++k) a[i][k] = T[(c - k) * S + lane + 32 * i];
    const F r3 = rinv[c], r2 = rinv[c - 1], r1 = rinv[c - 2], r0 = rinv[c - 3];
    const F e23 = T[c * S + c - 1], e13 = T[c * S + c - 2], e03 = T[c * S + c - 3];
    const F e12 = T[(c - 1) * S + c - 2], e02 = T[(c - 1) * S + c - 3], e01 = T[(c - 2) * S + c - 3];
    const F u3 = __shfl_sync(NUPPN_FULL, tile_row<R>(x, c), c & 31);
    const F u2 = __shfl_sync(NUPPN_FULL, tile_row<R>(x, c - 1), (c - 1) & 31);
    const F u1 = __shfl_sync(NUPPN_FULL, tile_row<R>(x, c - 2), (c - 2) & 31);
    const F u0 = __shfl_sync(NUPPN_FULL, tile_row<R>(x, c - 3), (c - 3) & 31);
    const F d3 = T[c * (S + 1)], d2 = T[(c - 1) * (S + 1)], d1 = T[(c - 2) * (S + 1)], d0 = T[(c - 3) * (S + 1)];
    const F w3 = div_piv<kPlain>(u3, d3, r3, bad);
    const F w2 = div_piv<kPlain>(sub_nz(u2, e23, w3), d2, r2, bad);
    const F w1 = div_piv<kPlain>(sub_nz(sub_nz(u1, e13, w3), e12, w2), d1, r1, bad);
    const F w0 = div_piv<kPlain>(sub_nz(sub_nz(sub_nz(u0, e03, w3), e02, w2), e01, w1), d0, r0, bad);
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int r = lane + 32 * i;
      const F t = sub_nz(sub_nz(sub_nz(sub_nz(x[i], a[i][0], w3), a[i][1], w2), a[i][2], w1), a[i][3], w0);
      x[i] = r == c ? w3 : r == c - 1 ? w2 : r == c - 2 ? w1 : r == c - 3 ? w0 : (r < c - 3 ? t : x[i]);
    }
  }
  for (; c >= 0; --c) {
    F a[R];
#pragma unroll
    for (int i = 0; i < R; ++i) {
      a[i] = T[c * S + lane + 32 * i];
      if (lane + 32 * i == c) x[i] = div_piv<kPlain>(x[i], a[i], ri[i], bad);
    }
    const F xc = __shfl_sync(NUPPN_FULL, tile_row<R>(x, c), c & 31);
#pragma unroll
    for (int i = 0; i < R; ++i)
      if (lane + 32 * i < c) x[i] = sub_nz(x[i], a[i], xc);
  }
}

template <int R>
__device__ __forceinline__ void tile_solve_regs(const double *T, const double *rinv, int na, double (&x)[R],
                                                const double (&ri)[R], int lane) {
  double x0[R];
#pragma unroll
  for (int i = 0; i < R; ++i) x0[i] = x[i];
  int bad = 0;
  tile_solve_core<R, false>(T, rinv, na, x, ri, lane, bad);
  if (__any_sync(NUPPN_FULL, bad)) {  // an operand outside div_piv's range: divide
#pragma unroll
    for (int i = 0; i < R; ++i) x[i] = x0[i];
    tile_solve_core<R, true>(T, rinv, na, x, ri, lane, bad);
  }
}

// Mixed-precision solve of (I - hJ) x = b by the calling warp, b in x on entry (rows lane + 32 i):
// x = 0, r = b; repeat: dx = scol * FP32-solve(srow * r * 2^-e) * 2^e (2^-e brings the scaled
// residual's largest entry into [1, 2), so it stays in FP32's range), x += dx, stop after
// ir_max_iters corrections or when max|dx| <= ir_rtol * max|x|, else r = b - (I - hJ) x in FP64 from
// the unfactored tile. Returns the number of FP64 residuals formed (the refinement sweeps).
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(NUPPN_FULL, v, o));
  return v;
}
template <int R>
__device__ int tile_solve_mixed(const Act &A, double (&x)[R], int lane) {
  constexpr int S = 32 * R;
  const int na = A.na;
  double b[R], sr[R], sc[R], r[R];
  float ri[R];
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int row = lane + 32 * i;
    const bool on = row < na;
    b[i] = on ? x[i] : 0.0;
    r[i] = b[i];
    sr[i] = on ? A.srow[row] : 0.0;
    sc[i] = on ? A.scol[row] : 0.0;
    ri[i] = on ? A.rinv32[row] : 0.0f;
    x[i] = 0.0;
  }
  int sweeps = 0;
  for (int it = 0;; ++it) {
    double m = 0.0;
#pragma unroll
    for (int i = 0; i < R; ++i) m = fmax(m, fabs(r[i] * sr[i]));
    m = warp_max(m);
    if (!(m > 0.0) || !isfinite(m)) break;  // exact (r = 0), or nothing left to refine
    const int e = ilogb(m);
    float f[R];
#pragma unroll
    for (int i = 0; i < R; ++i) f[i] = (float)ldexp(r[i] * sr[i], -e);
    tile_permute_rhs<R>(f, A.perm, na, A.xs, lane);  // the FP32 factor is of P diag(srow) (I - hJ) diag(scol)
    int bad = 0;
    tile_solve_core<R, false, float>(A.T32, A.rinv32, na, f, ri, lane, bad);
    double dm = 0.0, xm = 0.0;
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const double dx = ldexp((double)f[i], e) * sc[i];
      x[i] += dx;
      dm = fmax(dm, fabs(dx));
      xm = fmax(xm, fabs(x[i]));
    }
    if (it >= A.ir_max || warp_max(dm) <= A.ir_rtol * warp_max(xm)) break;
    // r = b - (I - hJ) x, row-oriented over the unfactored FP64 tile
#pragma unroll
    for (int i = 0; i < R; ++i) r[i] = b[i];
    for (int c = 0; c < na; ++c) {
      const double xc = __shfl_sync(NUPPN_FULL, tile_row<R>(x, c), c & 31);
#pragma unroll
      for (int i = 0; i < R; ++i) r[i] = sub_nz(r[i], A.T[c * S + lane + 32 * i], xc);
    }
    ++sweeps;
  }
  return sweeps;
}

// Tile solve in place on A.xs by the calling warp. The FP64 factor is of P (I - hJ): its right-hand
// side is read in the factor's row order; the mixed-precision solve permutes its own FP32 right-hand
// sides (its residuals are formed in the original row order).
template <int R>
__device__ void tile_solve_xs(const Act &A, int lane) {
  double x[R], ri[R];
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int r = lane + 32 * i;
    x[i] = r < A.na ? A.xs[A.mixed_now ? r : A.perm[r]] : 0.0;
    ri[i] = r < A.na ? A.rinv[r] : 0.0;
  }
  __syncwarp();  // every lane has read A.xs before any lane writes it (in the mixed solve or below)
  if (A.mixed_now) tile_solve_mixed<R>(A, x, lane);
  else tile_solve_regs<R>(A.T, A.rinv, A.na, x, ri, lane);
#pragma unroll
  for (int i = 0; i < R; ++i)
    if (lane + 32 * i < A.na) A.xs[lane + 32 * i] = x[i];
}

// I - hJ on the active subsystem and its factorization in the static order: dense tiles with row
// pivoting (tile_factor_block), larger systems with diagonal pivots.
// Returns false on a zero or non-finite pivot, or if a dependency wait timed out.
__device__ bool dev_factor_active(const DevNet &N, const Ws &W, Act &A, double h) {
  const int tid = GT, nt = GN, lane = tid & 31, w = tid >> 5, nw = nt >> 5;
  const int na = A.na;
  if (A.tile) {
    // dense tile, column-major: T[c*S + r] = entry (r, c); rows na..S-1 stay zero
    const int S = A.tile_rows;
    double *T = A.T;
    for (int i = tid; i < na * S; i += nt) T[i] = 0.0;
    GSYNC();
    for (int c = w; c < na; c += nw)
      for (int p = A.crp[c] + lane; p < A.crp[c + 1]; p += 32) T[A.ccol[p] * S + c] = assemble_entry(A, p, h);
    GSYNC();
    if (A.mixed) {
      A.mixed_now = S == 32 ? tile_factor_mixed<1>(A, na) : tile_factor_mixed<2>(A, na);
      if (A.mixed_now) return true;  // otherwise factor in FP64 (T is still unfactored)
    }
    return S == 32 ? tile_factor_block<1>(T, A.rinv, A.perm, na) : tile_factor_block<2>(T, A.rinv, A.perm, na);
  }
  for (int p = tid; p < A.nnz; p += nt) A.cval[p] = assemble_entry(A, p, h);
  GSYNC();
  if (A.onewarp_f) {  // one warp, rows in order
    int bad = 0;
    if (w == 0) {
      const int *crp = A.crp, *cdiag = A.cdiag, *ccol = A.ccol;  // plain: rewritten per Jacobian
      double *cval = A.cval, *wb = A.wbuf, *rdg = A.rdg;
      for (int c = 0; c < na; ++c) {
        const int rs = crp[c], re = crp[c + 1], dg = cdiag[c];
        for (int p = rs + lane; p < re; p += 32) wb[ccol[p]] = cval[p];
        __syncwarp();
        for (int p = rs; p < dg; ++p) {
          const int j = ccol[p];
          const double a = wb[j];
          if (a != 0.0) {
            const double l = a * rdg[j];
            const int qe = crp[j + 1];
            for (int q = cdiag[j] + 1 + lane; q < qe; q += 32) wb[ccol[q]] -= l * cval[q];
            __syncwarp();
            if (lane == 0) wb[j] = l;
          }
          __syncwarp();
        }
        for (int p = rs + lane; p < re; p += 32) cval[p] = wb[ccol[p]];
        __syncwarp();
        bad |= !pivot_ok(cval[dg]);
        if (lane == 0) rdg[c] = 1.0 / cval[dg];
        __syncwarp();
      }
    }
    return g_or(bad) == 0;
  }
  const int gen = ++A.genF;
  bool ok = true;
  double *wb = A.wbuf + (size_t)w * na;
  for (int c = w; c < na; c += nw) {
    const int rs = A.crp[c], re = A.crp[c + 1], dg = A.cdiag[c];
    for (int p = rs + lane; p < re; p += 32) wb[A.ccol[p]] = A.cval[p];
    __syncwarp();
    for (int p = rs; p < dg; ++p) {
      const int j = A.ccol[p];
      if (!spin_until(&A.flagF[j], gen)) ok = false;
      __syncwarp();
      const double a = wb[j];
      if (a != 0.0) {
        const double l = a * A.rdg[j];
        const int qe = A.crp[j + 1];
        for (int q = A.cdiag[j] + 1 + lane; q < qe; q += 32) wb[A.ccol[q]] -= l * A.cval[q];
        __syncwarp();
        if (lane == 0) wb[j] = l;
      }
      __syncwarp();
    }
    for (int p = rs + lane; p < re; p += 32) A.cval[p] = wb[A.ccol[p]];
    __syncwarp();
    if (!pivot_ok(A.cval[dg])) ok = false;
    if (lane == 0) A.rdg[c] = 1.0 / A.cval[dg];
    __threadfence_block();
    __syncwarp();
    if (lane == 0) *(volatile int *)&A.flagF[c] = gen;
  }
  GSYNC();
  return g_and(ok) != 0;
}

// Solve the factored active subsystem in place on A.xs (compact right-hand side in, solution out).
__device__ bool dev_solve_active(Act &A) {
  const int tid = GT, lane = tid & 31, w = tid >> 5, nw = GN >> 5;
  if (A.tile) {
    if (w == 0) {
      if (A.tile_rows == 32) tile_solve_xs<1>(A, lane);
      else tile_solve_xs<2>(A, lane);
    }
    GSYNC();
    return true;
  }
  if (A.onewarp) {  // one warp: forward then backward substitution, a row at a time
    if (w == 0) {
      // plain pointers: the factors are rewritten within the kernel, so loads must not go through
      // the non-coherent read-only cache
      const int *crp = A.crp, *cdiag = A.cdiag, *ccol = A.ccol;
      const double *cval = A.cval;
      double *xs = A.xs;
      for (int c = 0; c < A.na; ++c) {
        double s = 0.0;
        for (int p = crp[c] + lane; p < cdiag[c]; p += 32) s += cval[p] * xs[ccol[p]];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(NUPPN_FULL, s, o);
        if (lane == 0) xs[c] = xs[c] - s;
        __syncwarp();
      }
      for (int c = A.na - 1; c >= 0; --c) {
        double s = 0.0;
        for (int p = cdiag[c] + 1 + lane; p < crp[c + 1]; p += 32) s += cval[p] * xs[ccol[p]];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(NUPPN_FULL, s, o);
        if (lane == 0) xs[c] = (xs[c] - s) / cval[cdiag[c]];
        __syncwarp();
      }
    }
    GSYNC();
    return true;
  }
  bool ok = true;
  const int g1 = ++A.genS;
  for (int c = w; c < A.na; c += nw) {
    double s = 0.0;
    for (int p = A.crp[c] + lane; p < A.cdiag[c]; p += 32) {
      const int j = A.ccol[p];
      if (!spin_until(&A.flagS[j], g1)) ok = false;
      s += A.cval[p] * *(volatile double *)&A.xs[j];
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(NUPPN_FULL, s, o);
    if (lane == 0) {
      A.xs[c] = A.xs[c] - s;
      __threadfence_block();
      *(volatile int *)&A.flagS[c] = g1;
    }
    __syncwarp();
  }
  GSYNC();
  const int g2 = ++A.genS;
  for (int q = w; q < A.na; q += nw) {
    const int c = A.na - 1 - q;
    double s = 0.0;
    for (int p = A.cdiag[c] + 1 + lane; p < A.crp[c + 1]; p += 32) {
      const int j = A.ccol[p];
      if (!spin_until(&A.flagS[j], g2)) ok = false;
      s += A.cval[p] * *(volatile double *)&A.xs[j];
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(NUPPN_FULL, s, o);
    if (lane == 0) {
      A.xs[c] = (A.xs[c] - s) / A.cval[A.cdiag[c]];
      __threadfence_block();
      *(volatile int *)&A.flagS[c] = g2;
    }
    __syncwarp();
  }
  GSYNC();
  return g_and(ok) != 0;
}

// Species-indexed solve for the parity entry point: x = 0 off the active set.
__device__ bool dev_solve_species(const DevNet &N, Act &A, const double *rhs, double *x) {
  for (int c = GT; c < A.na; c += GN) A.xs[c] = rhs[N.sp_of_sys[A.arow[c]]];
  for (int s = GT; s < N.nsp; s += GN) x[s] = 0.0;
  GSYNC();
  bool ok = dev_solve_active(A);
  for (int c = GT; c < A.na; c += GN) x[N.sp_of_sys[A.arow[c]]] = A.xs[c];
  GSYNC();
  return ok;
}

// ---------------------------------------------------------------------------------------------
// Right-hand side restricted to the dynamic network (after dev_compact).
//
// Within one step only dX/dt of masked species is used (the correction is zero elsewhere, as in
// ddecompac, jac_rhs.F90:584-608) and unmasked abundances stay frozen at the step's values, but
// calculate_dxdt (jac_rhs.F90:217-278) still sums every considered reaction into the masked rows,
// those with a frozen reactant included. Such a reaction failed the dynamic-network test at the
// start of the step, yet its flux can grow within the step with its masked reactant: neutron
// captures on frozen seed nuclei take up neutrons once a neutron source has switched on. Each masked
// row therefore gets
//  - one term per reaction whose reactants are all masked (or gamma): the slot's coefficient (-k2,
//    -1, k6 or k8 for k1, k3, k5, k7), the reaction's (1/k2!) * rate and the compact indices of its
//    reactants, evaluated from each sub-step's abundances in the reference's order (reaction, then
//    slot);
//  - one term per group of reactions with a frozen reactant that share their varying factor (the
//    masked reactant's xn to its power, or none when every reactant is frozen or gamma): the
//    group's constant, the sum over its reactions of coefficient * (1/k2!) * rate * the frozen
//    reactant's xn (to the power k2 for the first reactant), formed once per step. A group sums in
//    another order than the reference's loop, which changes the row's sum at the rounding level.
// Per step: every reaction is classified once (rhs_classify_reactions); a row's static list is cut
// into pieces of kRhsPiece items, a warp counts a piece's own terms and sums its other items per
// key (lane-private sums, then a fixed butterfly per key: rhs_piece), a warp per row adds its
// pieces' groups in piece order (group_items), and the own terms are placed in the static list's
// order. Every sum depends only on the items' positions, so results are bit-reproducible.

// Every considered reaction classified once per step, block-parallel and coalesced over reactions:
// rkey[a] = -1 if its reactants are all masked or gamma (each of its slots in a masked row is then a
// term of its own); otherwise its group key, (compact row of its masked reactant << 3) | that
// reactant's power, or (na << 3) | 1 when every reactant is frozen or gamma (a constant flux), and
// rcf[a] = (1/k2!) v * the frozen reactants' xn (xn1^k2, xn2) in the reference's order of products.
// For a reaction of the first kind, rcf[a] = (1/k2!) v and rpk[a] packs its term's reactants as the
// gather items do (compact row of k1 | of k3, na for gamma, << 14 | k2 << 28).
// spc: species -> compact row, -1 if frozen (gamma included).
__device__ __forceinline__ void rhs_classify_reactions(const DevNet &N, const Ws &W, const int *spc, int na, int *rkey,
                                                       double *rcf, uint32_t *rpk) {
  const int g = N.ig;
  const int4 *kp = reinterpret_cast<const int4 *>(N.act_k);
#pragma unroll 2
  for (int a = GT; a < N.nact; a += GN) {
    const int4 k = kp[2 * (size_t)a];
    const int c1 = spc[k.x], c2 = k.z == g ? na : spc[k.z];
    const bool m1 = c1 >= 0, m2 = c2 >= 0;
    double cf = c_fact[k.y] * W.v[N.act_slot[a]];
    if (m1 && m2) {
      rkey[a] = -1;
      rcf[a] = cf;
      rpk[a] = (uint32_t)c1 | ((uint32_t)c2 << 14) | ((uint32_t)k.y << 28);
      continue;
    }
    if (!m1) cf = cf * powi(W.xn[k.x], k.y);
    if (!m2) cf = cf * W.xn[k.z];
    rkey[a] = m1 ? (c1 << 3) | k.y : (m2 && c2 < na ? (c2 << 3) | 1 : (na << 3) | 1);
    rcf[a] = cf;
  }
}

// Per-warp key accumulator in the CTA's workspace: acc[key] the running sum of a key, tag[key] 1 once
// the key has a value in the current piece or row, list[] the keys in the order they first came.
// Entries are zero outside the keys in the list, which are cleared when the list is emitted.
struct KeyAcc {
  double *acc;
  int *tag, *list;
};

// The warp's 32 (key, val) pairs (key < 0: none) added to its accumulator. The values of one key
// are summed by a butterfly, which gives every lane the same bits whatever their order, then lane 0
// adds the sum to acc[key]; keys are taken in the order of their first lane, so the sums and the
// order of the list depend only on the positions of the items. n: keys in the list (warp-uniform).
__device__ __forceinline__ void group_chunk(int key, double val, const KeyAcc &K, int &n) {
  const int lane = threadIdx.x & 31;
  unsigned pend = __ballot_sync(NUPPN_FULL, key >= 0);
  while (pend) {
    const int k0 = __shfl_sync(NUPPN_FULL, key, __ffs(pend) - 1);
    const bool mine = key == k0;
    double v = mine ? val : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(NUPPN_FULL, v, o);
    int fresh = 0;
    if (lane == 0) {
      if (K.tag[k0] == 0) {
        K.tag[k0] = 1;
        K.list[n] = k0;
        K.acc[k0] = v;
        fresh = 1;
      } else {
        K.acc[k0] = K.acc[k0] + v;
      }
    }
    n += __shfl_sync(NUPPN_FULL, fresh, 0);
    pend &= ~__ballot_sync(NUPPN_FULL, mine);
  }
}

// The accumulator's n keys and sums written to key[i], val[i] (i < n) and cleared.
__device__ __forceinline__ void group_emit(const KeyAcc &K, int n, int *key, double *val) {
  __syncwarp();  // lane 0's accumulator writes are visible to the warp
  for (int i = threadIdx.x & 31; i < n; i += 32) {
    const int k = K.list[i];
    key[i] = k;
    val[i] = K.acc[k];
    K.acc[k] = 0.0;
    K.tag[k] = 0;
  }
  __syncwarp();
}

__device__ __forceinline__ void put_group_item(Act &A, int q, int key, double sum) {
  A.gcoef[q] = 1.0f;
  A.grcv[q] = sum;
  A.grpk[q] = (uint32_t)(key >> 3) | ((uint32_t)A.na << 14) | ((uint32_t)(key & 7) << 28) | kGroupItem;
}

// The groups of the items key[0..n) (-1: none), written over key[0..groups) and val[0..groups);
// returns the number of groups. Up to 32 keys: lane i holds the i-th key (in the order of first
// appearance), every lane adds its own items (the n items taken 32 at a time, lane l the l-th of
// each chunk) into a private sum per key, and the 32 private sums of a key are added by a
// butterfly, which gives every lane the same bits whatever their order. The result depends only on
// the items' positions. Past 32 keys the items are grouped again through the workspace
// accumulator (K) instead.
__device__ __forceinline__ int group_items(int *key, double *val, int n, const KeyAcc &K) {
  const int lane = threadIdx.x & 31;
  double lacc[32];
  int gk = -1, ng = 0;
  bool ovf = false;
  int kn = lane < n ? key[lane] : -1;
  double vn = lane < n ? val[lane] : 0.0;
  for (int b = 0; b < n; b += 32) {
    const int k = kn;
    const double v = vn;
    const int bn = b + 32 + lane;  // the next chunk's loads go out before this chunk's work
    kn = bn < n ? key[bn] : -1;
    vn = bn < n ? val[bn] : 0.0;
    int slot = -1;
    for (int j = 0; j < ng; ++j)
      if (__shfl_sync(NUPPN_FULL, gk, j) == k) slot = j;
    unsigned pend = __ballot_sync(NUPPN_FULL, k >= 0 && slot < 0);
    while (pend) {  // keys seen for the first time, in the order of their first lane
      const int k0 = __shfl_sync(NUPPN_FULL, k, __ffs(pend) - 1);
      if (ng < 32) {
        if (lane == ng) gk = k0;
        lacc[ng] = 0.0;
        if (k == k0) slot = ng;
        ++ng;
      } else {
        ovf = true;
      }
      pend &= ~__ballot_sync(NUPPN_FULL, k == k0);
    }
    if (ovf) break;
    if (slot >= 0) lacc[slot] += v;
  }
  if (!ovf) {
    double gs = 0.0;
    for (int j = 0; j < ng; ++j) {
      double t = lacc[j];
      for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(NUPPN_FULL, t, o);
      if (lane == j) gs = t;
    }
    __syncwarp();
    if (lane < ng) {
      key[lane] = gk;
      val[lane] = gs;
    }
    __syncwarp();
    return ng;
  }
  int nk = 0;
  for (int b = 0; b < n; b += 32) {
    const bool in = b + lane < n;
    group_chunk(in ? key[b + lane] : -1, in ? val[b + lane] : 0.0, K, nk);
  }
  group_emit(K, nk, key, val);
  return nk;
}

// One piece of a masked row's static list, items [t0, t1) (items[t] = reaction a << 2 | slot m,
// coefs[t] the slot's coefficient -k2, -1, k6 or k8), taken by one warp 32 at a time: items of
// reactions whose reactants are all masked or gamma (rkey -1) are counted into own (they become terms
// of their own), the others are summed per group key (value = coefficient * rcf[a]) straight from
// registers. Up to 32 keys: lane i holds the i-th key (in the order of first appearance), each lane
// adds its own items into a private sum per key, and a key's 32 private sums are added by a
// butterfly, which gives every lane the same bits whatever their order. Past 32 keys the piece is
// grouped again through the workspace accumulator K. The groups are written to gkey / gval, the
// number of groups returned.
__device__ __forceinline__ int rhs_piece(const int *rkey, const double *rcf, const int *items, const double *coefs,
                                         int t0, int t1, int *gkey, double *gval, const KeyAcc &K, int &own) {
  const int lane = threadIdx.x & 31;
  double lacc[32];
  int gk = -1, ng = 0, nown = 0;
  bool ovf = false;
  for (int b = t0; b < t1 && !ovf; b += 32) {
    const int t = b + lane;
    const int a = t < t1 ? items[t] >> 2 : 0;
    const int k = t < t1 ? rkey[a] : -2;
    const double v = k >= 0 ? coefs[t] * rcf[a] : 0.0;
    nown += __popc(__ballot_sync(NUPPN_FULL, k == -1));
    int slot = -1;
    for (int j = 0; j < ng; ++j)
      if (__shfl_sync(NUPPN_FULL, gk, j) == k) slot = j;
    unsigned pend = __ballot_sync(NUPPN_FULL, k >= 0 && slot < 0);
    while (pend) {  // keys seen for the first time, in the order of their first lane
      const int k0 = __shfl_sync(NUPPN_FULL, k, __ffs(pend) - 1);
      if (ng < 32) {
        if (lane == ng) gk = k0;
        lacc[ng] = 0.0;
        if (k == k0) slot = ng;
        ++ng;
      } else {
        ovf = true;
      }
      pend &= ~__ballot_sync(NUPPN_FULL, k == k0);
    }
    if (slot >= 0) lacc[slot] += v;
  }
  if (!ovf) {
    double gs = 0.0;
    for (int j = 0; j < ng; ++j) {
      double x = lacc[j];
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(NUPPN_FULL, x, o);
      if (lane == j) gs = x;
    }
    if (lane < ng) {
      gkey[lane] = gk;
      gval[lane] = gs;
    }
    __syncwarp();
    own = nown;
    return ng;
  }
  int nk = 0;
  nown = 0;
  for (int b = t0; b < t1; b += 32) {
    const int t = b + lane;
    const int a = t < t1 ? items[t] >> 2 : 0;
    const int k = t < t1 ? rkey[a] : -2;
    nown += __popc(__ballot_sync(NUPPN_FULL, k == -1));
    group_chunk(k >= 0 ? k : -1, k >= 0 ? coefs[t] * rcf[a] : 0.0, K, nk);
  }
  group_emit(K, nk, gkey, gval);
  own = nown;
  return nk;
}

__device__ void dev_compact_rhs(const DevNet &N, const Ws &W, Act &A, char *smem, size_t smem_bytes, int *sint) {
  const int tid = GT, nt = GN, lane = tid & 31, w = tid >> 5, nw = nt >> 5;
  const int *sys2c = W.act_tmp;              // system index -> active row (dev_compact), -1 if frozen
  int *cnt = W.act_tmp + 2 * (N.nsys + 1);   // [na+1] gather items per row, then row offsets
  int *off = W.act_tmp + 3 * (N.nsys + 1);   // [na+1] offsets of the rows' static lists
  int *fkey = W.rhs_key;                     // [T] each piece's groups over its first items, then a row's
  double *fval = W.rhs_val;                  // [T] their sums
  const int npmax = (N.nsys + 1) + N.ndg_item / kRhsPiece + 1;
  int *pofs = W.rhs_piece;                   // [na+1] first piece of each row
  int *pcnt = W.rhs_piece + (N.nsys + 1);    // [pieces] groups of each piece
  int *pown = pcnt + npmax;                  // [pieces] own terms of each piece
  int *poof = pown + npmax;                  // [pieces] own terms of the row's earlier pieces
  int *rown = poof + npmax;                  // [na] own terms of each row
  int *spc = W.rhs_spc;                      // [nsp] species -> active row, -1 if frozen
  int *rkey = W.rhs_rkey;                    // [nact] each reaction's class: -1 own terms, else group key
  double *rcf = W.rhs_rcf;                   // [nact] its frozen factors' constant
  uint32_t *rpk = W.rhs_rpk;                 // [nact] packed reactants of a reaction of own terms
  const int na = A.na, nkey = (na + 1) << 3;
  const size_t kw = (size_t)w * kRhsKeysPerRow * (N.nsys + 1);  // this warp's accumulator
  const KeyAcc K = {W.rhs_acc + kw, W.rhs_tag + kw, W.rhs_list + kw};
  for (int i = lane; i < nkey; i += 32) {  // the workspace may hold anything: clear the keys of na rows
    K.acc[i] = 0.0;
    K.tag[i] = 0;
  }
  for (int sp = tid; sp < N.nsp; sp += nt) {
    const int q = N.sys_of_sp[sp];
    spc[sp] = q >= 0 ? sys2c[q] : -1;
  }
  for (int c = tid; c < na; c += nt) {
    const int sp = N.sp_of_sys[A.arow[c]];
    const int len = N.dg_ptr[sp + 1] - N.dg_ptr[sp];
    off[c] = len;
    pofs[c] = (len + kRhsPiece - 1) / kRhsPiece;
  }
  GSYNC();
  rhs_classify_reactions(N, W, spc, na, rkey, rcf, rpk);
  const int T = block_scan_excl(off, na, sint);
  const int NP = block_scan_excl(pofs, na, sint);
  if (tid == 0) {
    off[na] = T;
    pofs[na] = NP;
  }
  GSYNC();
  // each piece (a warp): its own terms counted, its frozen-reactant items grouped
  for (int P = w; P < NP; P += nw) {
    const int c = seg_of(pofs, na, P);
    const int t0 = off[c] + (P - pofs[c]) * kRhsPiece, t1 = min(t0 + kRhsPiece, off[c + 1]);
    const int base = N.dg_ptr[N.sp_of_sys[A.arow[c]]] - off[c];
    int own = 0;
    const int n = rhs_piece(rkey, rcf, N.dg_item + base, N.dg_coef + base, t0, t1, fkey + t0, fval + t0, K, own);
    if (lane == 0) {
      pcnt[P] = n;
      pown[P] = own;
    }
  }
  GSYNC();
  for (int c = w; c < na; c += nw) {  // per row: own terms before each piece; several pieces' groups merged
    const int p0 = pofs[c], npc = pofs[c + 1] - p0;
    int own = 0;
    for (int P = p0; P < p0 + npc; ++P) {
      if (lane == 0) poof[P] = own;
      own += pown[P];
    }
    int n = npc == 1 ? pcnt[p0] : 0;
    if (npc > 1) {
      // move the pieces' groups together at the row's start, in piece order, then group them
      for (int P = p0; P < p0 + npc; ++P) {
        const int s0 = off[c] + (P - p0) * kRhsPiece, np = pcnt[P];
        for (int b = 0; b < np; b += 32) {  // s0 >= off[c] + n: moves go down or stay
          const int i = b + lane;
          const int k = i < np ? fkey[s0 + i] : -1;
          const double v = i < np ? fval[s0 + i] : 0.0;
          __syncwarp();
          if (i < np) {
            fkey[off[c] + n + i] = k;
            fval[off[c] + n + i] = v;
          }
          __syncwarp();
        }
        n += np;
      }
      n = group_items(fkey + off[c], fval + off[c], n, K);
    }
    if (lane == 0) {
      cnt[c] = own + n;
      rown[c] = own;
    }
  }
  GSYNC();
  const int ngi = block_scan_excl(cnt, na, sint);
  const size_t lu_need = act_bytes(na, A.nnz, nw, A.tile_rows, A.mixed), need = rhs_bytes(na, ngi);
  char *base;
  if (A.in_smem && lu_need + need <= smem_bytes) {
    base = smem + lu_need;
    A.rhs_in_smem = true;
  } else {
    base = W.act_r;
    A.rhs_in_smem = false;
  }
  A.gptr = (int *)base; base += a16((size_t)(na + 1) * 4);
  A.gcoef = (float *)base; base += a16((size_t)ngi * 4);
  A.grpk = (uint32_t *)base; base += a16((size_t)ngi * 4);
  A.grcv = (double *)base; base += a16((size_t)ngi * 8);
  A.gterm = (double *)base;
  A.ngi = ngi;
  for (int c = tid; c <= na; c += nt) A.gptr[c] = c < na ? cnt[c] : ngi;
  for (int P = w; P < NP; P += nw) {  // own terms first, in the static list's order (a warp per piece)
    const int c = seg_of(pofs, na, P);
    const int t0 = off[c] + (P - pofs[c]) * kRhsPiece, t1 = min(t0 + kRhsPiece, off[c + 1]);
    const int base = N.dg_ptr[N.sp_of_sys[A.arow[c]]] - off[c];
    int q = cnt[c] + poof[P];
    for (int b = t0; b < t1; b += 32) {
      const int t = b + lane;
      const int a = t < t1 ? N.dg_item[base + t] >> 2 : 0;
      const bool own = t < t1 && rkey[a] == -1;
      const unsigned m = __ballot_sync(NUPPN_FULL, own);
      if (own) {
        const int qq = q + __popc(m & ((1u << lane) - 1u));
        A.gcoef[qq] = (float)N.dg_coef[base + t];  // -k2, -1, k6 or k8: small integers, exact
        A.grcv[qq] = rcf[a];
        A.grpk[qq] = rpk[a];
      }
      q += __popc(m);
    }
  }
  for (int c = w; c < na; c += nw) {  // then the row's groups
    const int own = rown[c];
    const int q0 = cnt[c] + own, ng = (c + 1 < na ? cnt[c + 1] : ngi) - q0;
    for (int i = lane; i < ng; i += 32) put_group_item(A, q0 + i, fkey[off[c] + i], fval[off[c] + i]);
  }
  GSYNC();
}

// Term q of the right-hand side from the compact molar abundances A.xnc: coefficient times the
// reaction's flux (1/k2!) v xn(k1)^k2 xn(k3), as in calculate_dxdt (jac_rhs.F90:245-252).
__device__ __forceinline__ double powi_small(double x, int m) {  // powi's products for m = 1, 2, 3
  return m == 1 ? x : m == 2 ? x * x : m == 3 ? x * (x * x) : powi(x, m);
}

__device__ __forceinline__ double rhs_term(const Act &A, int q) {
  const uint32_t pk = A.grpk[q];
  const double flux = A.grcv[q] * powi_small(A.xnc[pk & 0x3fff], (int)((pk >> 28) & 7)) * A.xnc[(pk >> 14) & 0x3fff];
  return (double)A.gcoef[q] * flux;
}

// dX/dt of active row c from the terms in A.gterm, accumulated in the reference's order and
// multiplied by A at the end (jac_rhs.F90:266-270).
__device__ __forceinline__ double gather_dxdt(const Act &A, int c) {
  double acc = 0.0;
  const int q1 = A.gptr[c + 1];
#pragma unroll 4
  for (int q = A.gptr[c]; q < q1; ++q) acc = acc + A.gterm[q];
  return acc * A.anc[c];
}

// calculate_dxdt on the active rows: compact abundances yc in, compact dX/dt out.
__device__ void dev_dxdt_active(const Act &A, const double *yc, double *dxc) {
  const int tid = GT, nt = GN;
  for (int c = tid; c < A.na; c += nt) A.xnc[c] = yc[c] / A.anc[c];
  GSYNC();
#pragma unroll 4
  for (int q = tid; q < A.ngi; q += nt) A.gterm[q] = rhs_term(A, q);
  GSYNC();
  for (int c = tid; c < A.na; c += nt) dxc[c] = gather_dxdt(A, c);
  GSYNC();
}

NUPPN_END
