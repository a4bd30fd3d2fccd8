// mixing.cu -- mppnp's diffusive mixing of abundances between mass shells (do_mixing with idifmix = 1,
// frames/mppnp/source/mixing.F90:34-342).
//
// Each cycle mppnp mixes the abundances of its m shells by one fully implicit diffusion step:
// mix_calculate_D_Lagrangian turns the Eulerian coefficient into a Lagrangian one, matrixdiffus
// (mass coordinates xm, code_source GNV/EVL) or matrixdiffus_mesa (shell masses dq, MES) builds one
// tridiagonal matrix (a, b, c) for the step, and mixdiff08 solves it by tridag (the Thomas
// algorithm, Numerical Recipes) for every considered species but the last slot, each column of the
// abundances X[shell][species] on its own.
//
// Here the matrix and its factorization (tridag's bet and gam, the same for every species) are
// built once on the host in the reference's order of operations, and the device does the
// substitutions: one thread per species walks the shells down and back up. The abundances are
// addressed as X[shell * shell_stride + species * species_stride], so both a shell-major array
// (species_stride 1: a warp reads consecutive species of one shell) and mppnp's own yps(msl, nsp)
// (shell_stride 1, species_stride msl: each thread walks one contiguous column, 16 shells per 128-byte
// line) are mixed in place. The recurrence is one FP64 divide per shell and step; the loads of the
// right-hand side do not depend on it, so each thread keeps the next kMixAhead of them in flight. Every
// operation is the one tridag performs, in its order, so the result equals the reference's bit for
// bit (--fmad=false keeps r - a u unfused).
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "net_host.h"

namespace nuppn {

namespace {

// reduce_term (mixing.F90:327-340)
inline void reduce_term(double alpha, double onedxr, double &d_coeff, double sig) {
  if (alpha * onedxr * d_coeff > sig) d_coeff = sig / (alpha * onedxr);
}

constexpr int kMixAhead = 8;

__global__ void k_mix_columns(int m, int ncol, double *X, long long sh, long long sp, const double *a,
                              const double *gam, const double *bet, const unsigned char *cons) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ncol || (cons && !cons[s])) return;
  double *x = X + (long long)s * sp;
  double r[kMixAhead];
  // forward: u(1) = r(1) / bet(1); u(j) = (r(j) - a(j) u(j-1)) / bet(j)
#pragma unroll
  for (int k = 0; k < kMixAhead; ++k) r[k] = k < m ? x[k * sh] : 0.0;
  double u = 0.0;
  for (int j0 = 0; j0 < m; j0 += kMixAhead) {
#pragma unroll
    for (int k = 0; k < kMixAhead; ++k) {
      const int j = j0 + k;
      if (j < m) {
        const double rj = r[k];
        r[k] = j + kMixAhead < m ? x[(long long)(j + kMixAhead) * sh] : 0.0;
        u = j == 0 ? rj / bet[0] : (rj - a[j] * u) / bet[j];
        x[(long long)j * sh] = u;
      }
    }
  }
  // back: u(j) = u(j) - gam(j+1) u(j+1), j = m-2 .. 0 (u holds u(m-1))
#pragma unroll
  for (int k = 0; k < kMixAhead; ++k) r[k] = m - 2 - k >= 0 ? x[(long long)(m - 2 - k) * sh] : 0.0;
  for (int j0 = m - 2; j0 >= 0; j0 -= kMixAhead) {
#pragma unroll
    for (int k = 0; k < kMixAhead; ++k) {
      const int j = j0 - k;
      if (j >= 0) {
        const double rj = r[k];
        r[k] = j - kMixAhead >= 0 ? x[(long long)(j - kMixAhead) * sh] : 0.0;
        u = rj - gam[j + 1] * u;
        x[(long long)j * sh] = u;
      }
    }
  }
}

}  // namespace

std::string mix_d_lagrangian(int m, const double *d_eul, const double *rho, const double *rad, double *d_lagr) {
  const double dconst = 3.0589703419947736e-11;  // 4 pi Rsun^2 / Msun (mixing.F90:79)
  for (int j = 0; j < m; ++j) {
    d_lagr[j] = 0.0;
    if (d_eul[j] <= 0.0) continue;
    double lnrho, lnrad;
    if (j == 0) {
      lnrho = std::log(rho[j]);
      lnrad = std::log(rad[j]);
    } else {
      lnrho = (std::log(rho[j]) + std::log(rho[j - 1])) / 2.0;
      lnrad = (std::log(rad[j]) + std::log(rad[j - 1])) / 2.0;
    }
    d_lagr[j] = d_eul[j] * std::pow(dconst, 2.0) * std::exp(2.0 * (2.0 * lnrad + lnrho));
  }
  return std::string();
}

std::string mix_matrix(int m, const double *xm, const double *dq, double *d, double h, double sig, bool mesa,
                       std::vector<double> &a, std::vector<double> &b, std::vector<double> &c) {
  if (m < 2) return "mixing needs at least 2 shells";
  a.assign(m, 0.0);
  b.assign(m, 0.0);
  c.assign(m, 0.0);
  if (!mesa) {  // matrixdiffus (mixing.F90:176-250), 0-based shells
    double xr = xm[1] - xm[0];
    double alpha = d[1] * h / (xr * xr);
    if (sig < alpha) alpha = sig;
    a[0] = 0.0;
    b[0] = 1. + alpha;
    c[0] = -1.0 * alpha;
    for (int j = 1; j < m - 1; ++j) {
      const double xl = xm[j] - xm[j - 1];
      xr = xm[j + 1] - xm[j];
      const double xmm = 0.5 * (xm[j + 1] - xm[j - 1]);
      alpha = h / xmm;
      if (sig < d[j + 1] * alpha / xr) d[j + 1] = sig / alpha * xr;
      a[j] = -1.0 * d[j] * alpha / xl;
      b[j] = 1.0 + (d[j + 1] / xr + d[j] / xl) * alpha;
      c[j] = -1.0 * d[j + 1] * alpha / xr;
      if (xl == 0.0 || xr == 0.0) return "dm = 0 in the diffusion matrix";
    }
    const double xl = xm[m - 1] - xm[m - 2];
    alpha = d[m - 1] * h / (xl * xl);
    a[m - 1] = -1.0 * alpha;
    b[m - 1] = 1.0 + alpha;
    c[m - 1] = 0.0;
    if (xl == 0.0 || xr == 0.0) return "dm = 0 in the diffusion matrix";
  } else {  // matrixdiffus_mesa (mixing.F90:254-323)
    if (!(dq[0] > 0.0)) return "dq = 0 or NaN in the diffusion matrix";
    std::vector<double> dr(m, 0.0);
    dr[0] = d[0];
    double xr = dq[0], alpha = h / xr, term_c = 1.0 / xr, d_coeff = d[1];
    reduce_term(alpha, term_c, d_coeff, sig);
    dr[1] = d_coeff;
    a[0] = 0.0;
    b[0] = 1.0 + term_c * alpha * dr[1];
    c[0] = -1.0 * term_c * alpha * dr[1];
    for (int j = 1; j < m - 1; ++j) {
      const double xl = dq[j - 1];
      xr = dq[j];
      const double xmm = 0.5 * (dq[j] + dq[j - 1]);
      alpha = h / xmm;
      const double term_a = 1.0 / xl;
      term_c = 1.0 / xr;
      d_coeff = d[j + 1];
      reduce_term(alpha, term_c, d_coeff, sig);
      dr[j + 1] = d_coeff;
      const double term_b = term_c * dr[j + 1] + term_a * dr[j];
      a[j] = -1.0 * term_a * dr[j] * alpha;
      b[j] = 1.0 + term_b * alpha;
      c[j] = -1.0 * term_c * dr[j + 1] * alpha;
    }
    const double xl = dq[m - 1];
    alpha = h / (xl * xl);
    a[m - 1] = -1.0 * alpha * d[m - 1];
    b[m - 1] = 1.0 + alpha * d[m - 1];
    c[m - 1] = 0.0;
  }
  return std::string();
}

std::string tridag_factor(int m, const std::vector<double> &a, const std::vector<double> &b,
                          const std::vector<double> &c, std::vector<double> &gam, std::vector<double> &bet) {
  // tridag (mixing.F90:150-174): bet and gam depend on the matrix only
  gam.assign(m, 0.0);
  bet.assign(m, 0.0);
  if (b[0] == 0.0) return "tridag: rewrite equations (b(1) = 0)";
  double bt = b[0];
  bet[0] = bt;
  for (int j = 1; j < m; ++j) {
    gam[j] = c[j - 1] / bt;
    bt = b[j] - a[j] * gam[j];
    if (bt == 0.0) return "tridag: the matrix is singular";
    bet[j] = bt;
  }
  return std::string();
}

cudaError_t launch_mix_columns(int m, int ncol, double *X, long long shell_stride, long long species_stride,
                               const double *a, const double *gam, const double *bet, const unsigned char *cons,
                               cudaStream_t stream) {
  if (ncol <= 0) return cudaSuccess;
  // one warp per CTA: the ~1100 columns of a large network spread over ~35 SMs instead of ~9
  const int block = 32, grid = (ncol + block - 1) / block;
  k_mix_columns<<<grid, block, 0, stream>>>(m, ncol, X, shell_stride, species_stride, a, gam, bet, cons);
  return cudaGetLastError();
}

}  // namespace nuppn
