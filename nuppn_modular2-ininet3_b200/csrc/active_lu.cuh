// active_lu.cuh -- the dynamic network's active subsystem (included by solver.cu).
//
// The reference solves only the species its dynamic network selects (jac_rhs.F90:134-197: mask,
// pack, then SuperLU on the reduced matrix, with a new COLAMD/symbolic analysis every time). Here the
// fill-reducing order and the filled pattern are computed once for the whole network (net_host.cpp);
// the filled pattern restricted to the active rows and columns is closed under fill in that order,
// so each zone only has to compact it (once per Jacobian) and can then factor and solve it with no
// symbolic work. Compacted structures live in shared memory when they fit the CTA's budget and in
// the CTA's global workspace otherwise.
//
// Per Jacobian (dev_jacobian_mask, then):
//   dev_compact          active rows and the restricted filled pattern
//   dev_jacobian_active  Jacobian values and entry flags of the active entries (all reactions)
//   dev_compact_rhs      the reactions a step needs and the per-species gather lists
// Per factorization / right-hand side / solve: dev_factor_active, dev_dxdt_active, dev_solve_active,
// all on compact vectors indexed by the active row number c.
#pragma once

namespace nuppn {

constexpr int kSpinLimit = 1 << 22;  // per wait; a timeout marks the zone as failed, never hangs

// Active subsystems up to this size are factored and solved by one warp, row after row, with no
// inter-warp flags: for the few tens of species a dynamic network usually keeps, the dependency
// chain is the whole cost and a single warp walks it fastest.
constexpr int kOneWarpMax = 192;

struct Act {
  int na, nnz;
  int *crp, *cdiag, *arow, *flagF, *flagS, *ccol, *csrc;
  bool onewarp;  // factor/solve by one warp (small systems)
  double *cval, *xs, *wbuf;
  int genF, genS;
  bool in_smem;
  // right-hand side restricted to the dynamic network (see dev_compact_rhs)
  int nar, ngi;
  int *ar, *gptr, *gitem;
  float *gcoef;
  double *flux;
  bool rhs_in_smem;
};

// Bytes of the restricted right-hand side: int ar[nar], gptr[na+1], gitem[ngi]; float gcoef[ngi];
// double flux[nar]; 16-byte aligned arrays.
__host__ __device__ inline size_t rhs_bytes(int na, int nar, int ngi) {
  auto a16 = [](size_t x) { return (x + 15) & ~size_t(15); };
  return a16((size_t)nar * 4) + a16((size_t)(na + 1) * 4) + a16((size_t)ngi * 4) + a16((size_t)ngi * 4) +
         a16((size_t)nar * 8);
}

__device__ __forceinline__ void act_bind(Act &A, char *base, int na, int nnz, int nwarps) {
  auto a16 = [](size_t x) { return (x + 15) & ~size_t(15); };
  char *p = base;
  A.crp = (int *)p; p += a16((size_t)(na + 1) * 4);
  A.cdiag = (int *)p; p += a16((size_t)na * 4);
  A.arow = (int *)p; p += a16((size_t)na * 4);
  A.flagF = (int *)p; p += a16((size_t)na * 4);
  A.flagS = (int *)p; p += a16((size_t)na * 4);
  A.ccol = (int *)p; p += a16((size_t)nnz * 4);
  A.csrc = (int *)p; p += a16((size_t)nnz * 4);
  A.cval = (double *)p; p += a16((size_t)nnz * 8);
  A.xs = (double *)p; p += a16((size_t)na * 8);
  A.wbuf = (double *)p;
}

// Exclusive scan of v[0..n) in place (block-wide, deterministic); returns the total.
__device__ int block_scan_excl(int *v, int n, int *sint) {
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, w = tid >> 5, nw = nt >> 5;
  const int ch = (n + nt - 1) / nt, b0 = min(n, tid * ch), b1 = min(n, b0 + ch);
  int s = 0;
  for (int i = b0; i < b1; ++i) s += v[i];
  int incl = s;
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(NUPPN_FULL, incl, o);
    if (lane >= o) incl += t;
  }
  __syncthreads();
  if (lane == 31) sint[w] = incl;
  __syncthreads();
  int wbase = 0, total = 0;
  for (int i = 0; i < nw; ++i) {
    if (i < w) wbase += sint[i];
    total += sint[i];
  }
  int run = wbase + incl - s;
  for (int i = b0; i < b1; ++i) {
    int x = v[i];
    v[i] = run;
    run += x;
  }
  __syncthreads();
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
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, w = tid >> 5, nw = nt >> 5;
  int *sys2c = W.act_tmp;                  // [nsys]
  int *tmp_arow = W.act_tmp + N.nsys + 1;  // [nsys]
  int *cnt = W.act_tmp + 2 * (N.nsys + 1); // [nsys+1]
  for (int i = tid; i < N.nsys; i += nt) sys2c[i] = W.mask[N.sp_of_sys[i]] ? 1 : 0;
  __syncthreads();
  const int na = block_scan_excl(sys2c, N.nsys, sint);
  for (int i = tid; i < N.nsys; i += nt) {
    if (W.mask[N.sp_of_sys[i]]) tmp_arow[sys2c[i]] = i;
    else sys2c[i] = -1;
  }
  __syncthreads();
  for (int c = w; c < na; c += nw) {  // entries per active row: static entries in active columns
    int i = tmp_arow[c], n = 0;
    for (int p = N.lu_rowptr[i] + lane; p < N.lu_rowptr[i + 1]; p += 32) n += sys2c[N.lu_col[p]] >= 0;
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(NUPPN_FULL, n, o);
    if (lane == 0) cnt[c] = n;
  }
  __syncthreads();
  const int nnz = block_scan_excl(cnt, na, sint);
  const size_t need = act_bytes(na, nnz, nw);
  A.na = na;
  A.nnz = nnz;
  A.in_smem = need <= smem_bytes;
  act_bind(A, A.in_smem ? smem : W.act, na, nnz, nw);
  A.genF = 0;
  A.genS = 0;
  for (int c = tid; c < na; c += nt) {
    A.crp[c] = cnt[c];
    A.arow[c] = tmp_arow[c];
    A.flagF[c] = 0;
    A.flagS[c] = 0;
  }
  if (tid == 0) A.crp[na] = nnz;
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
  __syncthreads();
  A.onewarp = na <= (N.kn.lu_onewarp_max > 0 ? N.kn.lu_onewarp_max : kOneWarpMax);
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

// Jacobian values (1e-99 + the reaction contributions, every reaction as in the reference) and entry
// flags for the entries of the active subsystem. The contributions of all active entries are
// evaluated as one flattened, block-parallel list; each entry is then summed by a warp.
__device__ void dev_jacobian_active(const DevNet &N, const Ws &W, const Act &A, int *sint) {
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, w = tid >> 5, nw = nt >> 5;
  int *off = W.act_otmp;  // [nnz+1] <= nnzLU + 1
  for (int p = tid; p < A.nnz; p += nt) {
    const int e = N.lu_src[A.csrc[p]];
    off[p] = e >= 0 ? N.jg_ptr[e + 1] - N.jg_ptr[e] : 0;
  }
  __syncthreads();
  const int T = block_scan_excl(off, A.nnz, sint);
  if (tid == 0) off[A.nnz] = T;
  __syncthreads();
  double *dv = W.act_dtmp;
  uint8_t *sf = W.act_btmp;
  for (int t = tid; t < T; t += nt) {
    const int p = seg_of(off, A.nnz, t);
    const int e = N.lu_src[A.csrc[p]];
    const int it = N.jg_item[N.jg_ptr[e] + (t - off[p])];
    bool set;
    dv[t] = jac_contrib(N, W, it >> 3, it & 7, set);
    sf[t] = set ? 1 : 0;
  }
  __syncthreads();
  for (int p = w; p < A.nnz; p += nw) {
    const int e = N.lu_src[A.csrc[p]];
    if (e < 0) continue;
    double acc = 0.0;
    int set = 0;
    for (int t = off[p] + lane; t < off[p + 1]; t += 32) {
      acc += dv[t];
      set |= sf[t];
    }
    for (int o = 16; o > 0; o >>= 1) {
      acc += __shfl_xor_sync(NUPPN_FULL, acc, o);
      set |= __shfl_xor_sync(NUPPN_FULL, set, o);
    }
    if (lane == 0) {
      W.jac[e] = 1.e-99 + acc;
      W.eset[e] = (uint8_t)set;
    }
  }
  __syncthreads();
}

// I - hJ on the active subsystem (reduce_jacobian semantics) and its factorization.
// Returns false if a dependency wait timed out.
__device__ bool dev_factor_active(const DevNet &N, const Ws &W, Act &A, double h) {
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, w = tid >> 5, nw = nt >> 5;
  for (int p = tid; p < A.nnz; p += nt) {
    int e = N.lu_src[A.csrc[p]];
    double val = 0.0;
    if (e >= 0) {
      double v = W.jac[e] * (-h);
      bool set = W.eset[e] != 0;
      if (set && (fabs(v) == 0.0 || v == -1.0)) { set = false; W.eset[e] = 0; }
      if (N.jdiag[N.jrow[e]] == e) { set = true; W.eset[e] = 1; v = v + 1.0; }  // active rows are masked
      if (set) val = v;
    }
    A.cval[p] = val;
  }
  __syncthreads();
  if (A.onewarp) {  // one warp, rows in order
    if (w == 0) {
      const int na = A.na;
      const int *crp = A.crp, *cdiag = A.cdiag, *ccol = A.ccol;  // plain: rewritten per Jacobian
      double *cval = A.cval, *wb = A.wbuf;
      for (int c = 0; c < na; ++c) {
        const int rs = crp[c], re = crp[c + 1], dg = cdiag[c];
        for (int p = rs + lane; p < re; p += 32) wb[ccol[p]] = cval[p];
        __syncwarp();
        for (int p = rs; p < dg; ++p) {
          const int j = ccol[p];
          const double a = wb[j];
          if (a != 0.0) {
            const double l = a / cval[cdiag[j]];
            const int qe = crp[j + 1];
            for (int q = cdiag[j] + 1 + lane; q < qe; q += 32) wb[ccol[q]] -= l * cval[q];
            __syncwarp();
            if (lane == 0) wb[j] = l;
          }
          __syncwarp();
        }
        for (int p = rs + lane; p < re; p += 32) cval[p] = wb[ccol[p]];
        __syncwarp();
      }
    }
    __syncthreads();
    return true;
  }
  const int gen = ++A.genF;
  bool ok = true;
  double *wb = A.wbuf + (size_t)w * A.na;
  for (int c = w; c < A.na; c += nw) {
    const int rs = A.crp[c], re = A.crp[c + 1], dg = A.cdiag[c];
    for (int p = rs + lane; p < re; p += 32) wb[A.ccol[p]] = A.cval[p];
    __syncwarp();
    for (int p = rs; p < dg; ++p) {
      const int j = A.ccol[p];
      if (!spin_until(&A.flagF[j], gen)) ok = false;
      __syncwarp();
      const double a = wb[j];
      if (a != 0.0) {
        const double l = a / A.cval[A.cdiag[j]];
        const int qe = A.crp[j + 1];
        for (int q = A.cdiag[j] + 1 + lane; q < qe; q += 32) wb[A.ccol[q]] -= l * A.cval[q];
        __syncwarp();
        if (lane == 0) wb[j] = l;
      }
      __syncwarp();
    }
    for (int p = rs + lane; p < re; p += 32) A.cval[p] = wb[A.ccol[p]];
    __threadfence_block();
    __syncwarp();
    if (lane == 0) *(volatile int *)&A.flagF[c] = gen;
  }
  __syncthreads();
  return __syncthreads_and(ok) != 0;
}

// Solve the factored active subsystem in place on A.xs (compact right-hand side in, solution out).
__device__ bool dev_solve_active(Act &A) {
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, nw = blockDim.x >> 5;
  if (A.onewarp) {  // one warp: forward then backward substitution, a row at a time
    if (w == 0) {
      // plain pointers: the factors and levels are rewritten within the kernel, so loads must not
      // go through the non-coherent read-only cache
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
    __syncthreads();
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
  __syncthreads();
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
  __syncthreads();
  return __syncthreads_and(ok) != 0;
}

// Species-indexed solve for the parity entry point: x = 0 off the active set.
__device__ bool dev_solve_species(const DevNet &N, Act &A, const double *rhs, double *x) {
  for (int c = threadIdx.x; c < A.na; c += blockDim.x) A.xs[c] = rhs[N.sp_of_sys[A.arow[c]]];
  for (int s = threadIdx.x; s < N.nsp; s += blockDim.x) x[s] = 0.0;
  __syncthreads();
  bool ok = dev_solve_active(A);
  for (int c = threadIdx.x; c < A.na; c += blockDim.x) x[N.sp_of_sys[A.arow[c]]] = A.xs[c];
  __syncthreads();
  return ok;
}

// ---------------------------------------------------------------------------------------------
// Right-hand side restricted to the dynamic network (after dev_compact).
//
// Within one step only dX/dt of masked species is used (the rest of the correction is zero, as in
// ddecompac, jac_rhs.F90:584-608) and unmasked abundances stay frozen. A reaction with an unmasked
// reactant did not pass the dynamic-network test (its flux is <= cyminformal/dt, jac_rhs.F90:350-353,
// or all its participants would be masked), and that flux cannot grow within the step beyond the
// change of its masked reactant. So the step keeps exactly the reactions whose reactants are all
// masked (or gamma), and each masked species sums their contributions in the reference's order
// (reaction order, then k1, k3, k5, k7).
__device__ void dev_compact_rhs(const DevNet &N, const Ws &W, Act &A, char *smem, size_t smem_bytes, int *sint) {
  const int tid = threadIdx.x, nt = blockDim.x, nw = nt >> 5;
  int *rmap = W.act_rtmp;                    // [nact]
  int *off = W.act_tmp + 3 * (N.nsys + 1);   // [na+1] segment offsets of the static species lists
  int *flag = W.act_itmp;                    // [T] kept flags -> positions
  const int g = N.ig;
  for (int a = tid; a < N.nact; a += nt) {
    const int *k = N.act_k + (size_t)a * 8;
    rmap[a] = (W.mask[k[0]] && (k[2] == g || W.mask[k[2]])) ? 1 : 0;
  }
  for (int c = tid; c < A.na; c += nt) {
    const int s = N.sp_of_sys[A.arow[c]];
    off[c] = N.dg_ptr[s + 1] - N.dg_ptr[s];
  }
  __syncthreads();
  const int nar = block_scan_excl(rmap, N.nact, sint);
  const int T = block_scan_excl(off, A.na, sint);
  if (tid == 0) off[A.na] = T;
  for (int a = tid; a < N.nact; a += nt) {  // rmap: kept reaction -> compact index, else -1
    const int *k = N.act_k + (size_t)a * 8;
    if (!(W.mask[k[0]] && (k[2] == g || W.mask[k[2]]))) rmap[a] = -1;
  }
  __syncthreads();
  for (int t = tid; t < T; t += nt) {  // flattened static lists of the masked species
    const int c = seg_of(off, A.na, t);
    const int s = N.sp_of_sys[A.arow[c]];
    flag[t] = rmap[N.dg_item[N.dg_ptr[s] + (t - off[c])] >> 2] >= 0 ? 1 : 0;
  }
  __syncthreads();
  const int ngi = block_scan_excl(flag, T, sint);
  const size_t lu_need = act_bytes(A.na, A.nnz, nw), need = rhs_bytes(A.na, nar, ngi);
  char *base;
  if (A.in_smem && lu_need + need <= smem_bytes) {
    base = smem + lu_need;
    A.rhs_in_smem = true;
  } else {
    base = W.act_r;
    A.rhs_in_smem = false;
  }
  auto a16 = [](size_t x) { return (x + 15) & ~size_t(15); };
  A.ar = (int *)base; base += a16((size_t)nar * 4);
  A.gptr = (int *)base; base += a16((size_t)(A.na + 1) * 4);
  A.gitem = (int *)base; base += a16((size_t)ngi * 4);
  A.gcoef = (float *)base; base += a16((size_t)ngi * 4);
  A.flux = (double *)base;
  A.nar = nar;
  A.ngi = ngi;
  for (int a = tid; a < N.nact; a += nt)
    if (rmap[a] >= 0) A.ar[rmap[a]] = a;
  for (int c = tid; c <= A.na; c += nt) A.gptr[c] = (c < A.na && off[c] < T) ? flag[off[c]] : ngi;
  for (int t = tid; t < T; t += nt) {
    const int c = seg_of(off, A.na, t);
    const int s = N.sp_of_sys[A.arow[c]];
    const int p = N.dg_ptr[s] + (t - off[c]);
    const int r = rmap[N.dg_item[p] >> 2];
    if (r >= 0) {
      A.gitem[flag[t]] = r;
      A.gcoef[flag[t]] = (float)N.dg_coef[p];
    }
  }
  if (tid == 0) W.xn[g] = 1.0;  // gamma's molar abundance
  __syncthreads();
}

// calculate_dxdt restricted to the kept reactions: compact abundances yc in, compact dX/dt out.
__device__ void dev_dxdt_active(const DevNet &N, const Ws &W, const Act &A, const double *yc, double *dxc) {
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int c = tid; c < A.na; c += nt) {
    const int s = N.sp_of_sys[A.arow[c]];
    W.xn[s] = yc[c] / N.an[s];
  }
  __syncthreads();
  for (int r = tid; r < A.nar; r += nt) {
    const int a = A.ar[r];
    const int *k = N.act_k + (size_t)a * 8;
    A.flux[r] = c_fact[k[1]] * W.v[N.act_slot[a]] * powi(W.xn[k[0]], k[1]) * W.xn[k[2]];
  }
  __syncthreads();
  for (int c = tid; c < A.na; c += nt) {
    double acc = 0.0;
    for (int p = A.gptr[c]; p < A.gptr[c + 1]; ++p) acc = acc + (double)A.gcoef[p] * A.flux[A.gitem[p]];
    dxc[c] = acc * N.an[N.sp_of_sys[A.arow[c]]];
  }
  __syncthreads();
}

}  // namespace nuppn
