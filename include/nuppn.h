/*
 * nuppn.h -- C ABI of the B200 reaction-network solver.
 *
 * Drop-in boundary for NuPPN's per-zone network integration. The reference's Fortran frames call
 *   evaluate_all_rates(ye, nvar, nvrel, rho, t9, yps, nu)                 physics/source/evaluate_rates.F90:14
 *   integrate_network(nvar, yps, t9_0, t9_1, rho_0, rho_1, ye, dtwant, nvrel, nu, ierr)
 *                                                                          solver/source/solver.F90:53
 * once per zone (ppn.F90:298-301, mppnp.F90:719-724, tppnp.F90:152-154). Those routines read the
 * network from module globals (rates::v, k1..k8, nuc_data masks, /cnetw/ A and Z, the REACLIB and
 * weak-rate tables, jac_rhs::dns2csr_map). Here the network is handed over once, as a descriptor of
 * plain arrays in the reference's slot layout, and every entry point is batched over zones.
 *
 * Conventions
 *   - Species and reaction slots keep the reference's order; indices are 0-based (Fortran index - 1).
 *   - The library owns device memory; the caller owns every host buffer passed in.
 *   - No entry point exits or stops: problems come back as a nuppn_status, per-zone solver outcomes as
 *     the reference's error codes (utils/source/errors.F90:5-21) in ierr[].
 *   - Abundance arrays are zone-major: X[z * ldx + i] is species i of zone z (ldx >= nsp).
 *   - Entry points are not re-entrant on the same nuppn_net (one host thread per handle), like the
 *     reference's module state.
 */
#ifndef NUPPN_H
#define NUPPN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NUPPN_ABI_VERSION 3

typedef enum {
  NUPPN_OK = 0,
  NUPPN_ERR_ARG = -1,      /* bad argument or descriptor                                 */
  NUPPN_ERR_CUDA = -2,     /* a CUDA runtime call failed                                 */
  NUPPN_ERR_NOMEM = -3,    /* device or host allocation failed                           */
  NUPPN_ERR_NET = -4,      /* network inconsistent (e.g. k index out of range)           */
  NUPPN_ERR_LIMIT = -5,    /* size beyond a compiled limit                               */
  NUPPN_ERR_NODEV = -6,    /* no usable sm_100 device                                    */
  NUPPN_ERR_TIMEOUT = -7   /* a bounded device wait ran out                              */
} nuppn_status;

/* Per-zone solver outcome codes: utils/source/errors.F90:5-21 (0 = success). */
#define NUPPN_SLV_CNVRG    1
#define NUPPN_MAX_SUBSTEPS 2
#define NUPPN_BAD_STEP     3
#define NUPPN_NEG_ABUNDS   4
#define NUPPN_HUGE_ABUNDS  5
#define NUPPN_SUM_X        6
#define NUPPN_GOT_NAN      7
#define NUPPN_BAD_YE       8
#define NUPPN_NSE_CNVRG    9
#define NUPPN_NSE_WEAK     10
#define NUPPN_SMALL_DT     11
#define NUPPN_BAD_INPUT    20  /* T9/rho not finite or not positive (the reference would stop) */

/* Rate sources of a reaction slot (the label lab(nre) of reaction_info.F90:53-56, reduced to what
 * decides how the rate is computed; ppn_physics.F90:550-589 gathers by the same label). */
enum {
  NUPPN_SRC_NONE = 0,      /* rate 0 (slot unused)                                        */
  NUPPN_SRC_VITAL = 1,     /* analytic template (vital.F90:239-2209)                      */
  NUPPN_SRC_REACLIB = 2,   /* REACLIB rate (reaclib.F90:431-582)                          */
  NUPPN_SRC_NETGEN = 3,    /* NETGEN table (netgen.F90:179-310)                           */
  NUPPN_SRC_FULLER = 4,    /* FFN 2-D table (fuller.F90:92-122)                           */
  NUPPN_SRC_KADONIS = 5,   /* KADoNiS (n,g) table, Akima in kT (kadonis.F90:150-187)      */
  NUPPN_SRC_CONST = 6      /* constant rate (alpha decays, alpha_decays.F90)              */
};

/* Solver and physics knobs on the path: &ppn_solver defaults of solver_knobs.F90:43-57 and the
 * physics_knobs.F90 switches that evaluate_all_rates reads. */
typedef struct nuppn_knobs {
  int32_t ittd;                /* max Newton iterations (6)                                   */
  int32_t integration_method;  /* 0 = backward Euler + Newton, 1 = Bader-Deuflhard           */
  int32_t max_sub_steps;       /* 4000                                                        */
  int32_t interpolate_temp;    /* 1                                                           */
  int32_t interpolate_dens;    /* 1                                                           */
  int32_t screen_option;       /* 0 none, 2 Chugunov-DeWitt-Yakovlev 2007                     */
  int32_t detailed_balance;    /* 1                                                           */
  int32_t weak_rates;          /* 1                                                           */
  int32_t strong_rates;        /* 1                                                           */
  int32_t decay;               /* 0                                                           */
  int32_t i_nse;               /* 0                                                           */
  int32_t nse_weak_method;     /* 1 = Cash-Karp RK, 0 = Euler                                 */
  double dgrd;                 /* 1e-3                                                        */
  double grdthreshold;         /* 1e-15                                                       */
  double cyminformal;          /* 1e-30                                                       */
  double min_rate_ov_dt;       /* 1e-99                                                       */
  double min_t9_for_slv;       /* 0.01                                                        */
  double delta_state_max;      /* 1e99                                                        */
  double nse_min_t9;           /* 6                                                           */
  /* device-only choices (no reference counterpart) */
  int32_t lu_precision;        /* 0 = FP64 factor, 1 = FP32 factor + FP64 iterative refinement */
  int32_t ir_max_iters;        /* refinement sweeps per solve in mode 1 (default 3)           */
  double ir_rtol;              /* refinement stops when |dx| <= ir_rtol*|x| (default 1e-14)   */
  int32_t threads_per_zone;    /* threads that integrate one zone: 32 = one warp per zone, with
                                  zones_per_cta zones in each CTA; 64..256 (a multiple of 32) =
                                  one CTA of that size per zone; 0 = one CTA of 256 per zone     */
  int32_t lu_onewarp_max;      /* active systems up to this size are factored/solved by one warp
                                  (0 = library default; larger ones use sync-free multi-warp)    */
  int32_t lu_tile_max;         /* active systems up to this size (at most 64) are factored in a
                                  dense tile and solved in registers (0 = 64, negative = never)  */
  int32_t zones_per_cta;       /* one warp per zone: warps (zones) per CTA, 1..8 (0 = 8)         */
  int32_t zone_smem;           /* shared-memory bytes for each zone's active subsystem (0 =
                                  library choice: 72 KB per CTA, or the CTA's 216 KB split evenly
                                  among its zones); a zone whose system does not fit uses its
                                  global workspace                                                */
  int32_t reserved[3];
} nuppn_knobs;

/* Network description in the reference's slot layout (what rnetw2007, reaclib_init, netgen_init,
 * fuller_init, kadonis_init and reverse_init leave in module state). Array extents in brackets. */
typedef struct nuppn_net_desc {
  int32_t nsp, nre;
  int32_t igamma;                    /* slot of 'OOOOO' (jac_rhs.F90:52-58)                      */
  const double *anetw, *znetw;       /* [nsp] A and Z, COMMON /cnetw/                            */
  const uint8_t *considerisotope;    /* [nsp]                                                    */
  const double *exmass;              /* [nsp] mass excess (MeV): masses/Q of nse_swj.F90:186-196 */
  const double *gspin;               /* [nsp] 2J+1                                               */
  const int32_t *spec_part;          /* [nsp] partition-function row or -1                       */
  const int32_t *k;                  /* [nre][8] k1..k8 (rates.F90:15)                           */
  const int32_t *ilabb;              /* [nre] reaction type 1..22 (reaction_info.F90:8-34)      */
  const uint8_t *considerreaction;   /* [nre]                                                    */
  const double *rfac;                /* [nre] rate factors (evaluate_rates.F90:195)              */
  const int32_t *src, *src_idx;      /* [nre] rate source and index in that source              */
  const int32_t *irev;               /* [nre] detailed-balance partner or -1 (reverse.F90:13)   */
  /* REACLIB: contributions (a0..a6) summed into rates (reaclib.F90:478-498) */
  int32_t rl_ncontrib, rl_nrate;
  const double *rl_a;                /* [ncontrib][7]                                            */
  const int32_t *rl_rate;            /* [ncontrib] rate index, non-decreasing                    */
  const int32_t *rl_chapter;         /* [nrate] 1..11                                            */
  const uint8_t *rl_vflag;           /* [nrate] rflag2 == 'v'                                    */
  const uint8_t *rl_ecflag;          /* [nrate] rrlreac == '  ec'                                */
  const int32_t *rl_nireac;          /* [nrate] reaction type used for the density factor       */
  const int32_t *rl_part;            /* [nrate][6] partition-function rows (-1 -> 1.0)           */
  int32_t npart;
  const double *part_t9;             /* [24] temperature grid                                    */
  const double *part_val;            /* [npart][24]                                              */
  /* VITAL analytic templates: v = rho^dpow * xfac * sum c*T9^p*exp(d*T9^(-1/3) + f/T9 + g*T9) */
  int32_t vt_nrate, vt_nterm;
  const int32_t *vt_first;           /* [nrate+1]                                                */
  const double *vt_terms;            /* [nterm][5] (c, p, d, f, g)                               */
  const double *vt_dpow;             /* [nrate]                                                  */
  const int32_t *vt_xfac;            /* [nrate] species for the 0.5*(1+X) factor, or -1          */
  /* NETGEN beta table (netgen.F90:179-310) */
  int32_t ng_kgrid, ng_nreac, ng_ndmax;
  const double *ng_t8;               /* [kgrid]                                                  */
  const double *ng_flag;             /* [nreac]                                                  */
  const int32_t *ng_ndata;           /* [nreac]                                                  */
  const double *ng_ane;              /* [nreac][ndmax]                                           */
  const double *ng_l10v;             /* [kgrid][nreac][ndmax]                                    */
  /* FFN table (fuller.F90:92-122) */
  int32_t ff_nv, ff_nt, ff_nr;
  const double *ff_t9coo, *ff_rhocoo;/* [nt], [nr] (log10 T9, log10 rho*Ye)                      */
  const double *ff_l10v;             /* [nv][nt][nr]                                             */
  /* KADoNiS (kadonis.F90:150-187) */
  int32_t kd_n, kd_ne;
  const double *kd_e;                /* [ne] keV                                                 */
  const double *kd_rate;             /* [n][ne]                                                  */
  /* constant rates */
  int32_t nconst;
  const double *const_rate;          /* [nconst]                                                 */
  /* per VITAL rate: 0 = the template above, k = the reference's own formula for VITAL slot k
   * (vital.F90:339-569; k in 1-9, 14-17, 73; slot 5 reads X of vt_xfac as XII(IPROT)); NULL: all 0 */
  const int32_t *vt_form;            /* [vt_nrate]                                               */
} nuppn_net_desc;

typedef struct nuppn_net nuppn_net;

typedef struct nuppn_net_info {
  int32_t nsp, nre;                  /* slots                                                    */
  int32_t nspec_active, nreac_active;/* considered species / reactions                           */
  int32_t nnz_jac;                   /* nonzeros of the static Jacobian (jac_rhs.F90:504)       */
  int32_t nnz_lu;                    /* nonzeros of the filled pattern after symbolic analysis   */
  int32_t n_solve;                   /* order of the device system (considered, non-gamma)       */
  int32_t levels_lower, levels_upper;/* dependency levels of the triangular solves               */
  int64_t lu_flops;                  /* multiply-adds of one numeric factorization              */
  int64_t device_bytes;              /* device memory held by the handle                        */
} nuppn_net_info;

/* Per-zone counters of one nuppn_integrate call (solver_diagnostics.F90) */
typedef struct nuppn_zone_stats {
  int32_t nsucc;          /* accepted sub-steps                                                   */
  int32_t nfail;          /* rejected sub-steps                                                   */
  int32_t newton_iters;   /* total Newton iterations (BE) or sub-steps (BD)                       */
  int32_t nfact;          /* numeric factorizations                                               */
  int32_t nsolve;         /* triangular solve pairs                                               */
  int32_t nvar1_last;     /* species in the last dynamic-network solve                            */
  int32_t ir_sweeps;      /* refinement sweeps (mixed precision)                                  */
  int32_t nvar1_max;      /* largest dynamic-network solve of the call                            */
} nuppn_zone_stats;

/* -- library --------------------------------------------------------------------------------- */
int32_t nuppn_abi_version(void);
void nuppn_default_knobs(nuppn_knobs *knobs);
const char *nuppn_status_string(nuppn_status s);
/* Device status of the last failing CUDA call (human-readable, static storage). */
const char *nuppn_last_error(void);

/* Network set-up: replaces the init chain of ppn.F90:80-209 that fills module state, plus makemap
 * (jac_rhs.F90:461-540) and the one-time symbolic analysis that takes the place of SuperLU's
 * per-call COLAMD/symbolic work (c_fortran_dgssv.c:110-119). */
nuppn_status nuppn_net_create(const nuppn_net_desc *desc, const nuppn_knobs *knobs, int32_t device,
                              nuppn_net **out);
nuppn_status nuppn_net_destroy(nuppn_net *net);
nuppn_status nuppn_net_info_get(const nuppn_net *net, nuppn_net_info *info);
/* Replaces the knobs for later calls. threads_per_zone sets the CTA size and the workspace layout at
 * nuppn_net_create and cannot change afterwards (NUPPN_ERR_ARG if it differs from the handle's). */
nuppn_status nuppn_set_knobs(nuppn_net *net, const nuppn_knobs *knobs);

/* read_isotopedatabase (physics/source/nuc_data.F90:50-95): the first nnn entries of an isotope
 * database file in the reference's format (physics/run_template/isotopedatabase.txt and
 * isotopedatabase_all.txt: three header lines, then Z, A, element symbol, a reference mass number and
 * a T/F flag per line). Host only, no device needed. For each entry i: z[i], a[i], consider[i] (1 for
 * T), elem[3*i .. 3*i+2] the symbol, NUL-padded. Any output pointer may be NULL. NUPPN_ERR_ARG if the
 * file cannot be opened or a line does not parse; NUPPN_ERR_LIMIT if the file has fewer than nnn
 * entries (where the reference stops the run). networkI (ppn_physics.F90:40-130) keeps the entries
 * flagged T, in file order, as the network's isotopes after the VITAL species. */
nuppn_status nuppn_isotopedatabase_read(const char *path, int32_t nnn, int32_t *z, int32_t *a, uint8_t *consider,
                                        char *elem);

/* The network of a networksetup.txt file (physics/source/networksetup.F90): what write_networksetup
 * (:55-115, output_network) writes and read_networksetup (:140-260) reads, in the reference's slot
 * order. Names and labels are 5 characters each, blank padded, without NUL. k holds k1..k8 per
 * reaction: k1, k3, k5, k7 are 0-based species indices (-1 for a name not in the list), k2, k4, k6,
 * k8 the counts. Arrays are the caller's: sized nsp (species) and nre (reactions). */
typedef struct nuppn_netsetup {
  int32_t nsp, nre;                   /* NGIS species, NGIR reactions                                 */
  int32_t nisomers, nreac_isomers;    /* inumer, inumerr                                              */
  double t9, rho;                     /* set-up temperature and density of the header                 */
  char *zis;                          /* [nsp][5] species names                                       */
  uint8_t *considerisotope;           /* [nsp]                                                        */
  double *anetw, *znetw;              /* [nsp]                                                        */
  int32_t *isomeric_state;            /* [nsp] 1 ground, 2 isomer                                     */
  uint8_t *considerreaction;          /* [nre]                                                        */
  int32_t *k;                         /* [nre][8]                                                     */
  double *v;                          /* [nre] rate at the set-up T9 and rho                          */
  char *lab, *labb;                   /* [nre][5] rate reference and reaction type labels             */
  int32_t *ilabb;                     /* [nre] reaction type 1..22                                    */
  double *rfac, *bind_energy_diff;    /* [nre]                                                        */
} nuppn_netsetup;

/* write_networksetup: the file in the reference's fixed-column format (the lines
 * read_networksetup reads with its formats '(7x,I5,16x,I5)', fmtspecies and fmtreactionread). */
nuppn_status nuppn_networksetup_write(const char *path, const nuppn_netsetup *ns);

/* read_networksetup: with every array pointer NULL, fills only nsp, nre, nisomers, nreac_isomers,
 * t9 and rho (to size the arrays); otherwise also the arrays, which must hold ns->nsp species and
 * ns->nre reactions as set by the first call. NUPPN_ERR_ARG if the file cannot be read or a line does
 * not parse. Like the reference (:226-240), reactions with a participant whose considerisotope is
 * false are marked not considered. */
nuppn_status nuppn_networksetup_read(const char *path, nuppn_netsetup *ns);

/* -- ppn's per-cycle output files (printonecycle, frames/ppn/source/ppn.F90:431-539), byte for byte,
 *    in the reference's fixed columns, so NuGrid tools read them unchanged. Host only. --------------- */

/* iso_massf<mmmmm>.DAT (ppn.F90:519-536): the header, the model line (model, dzeit, agej), T9 and rho,
 * the neutron, proton and alpha number densities (the reference writes X * rho * N_A for n and p and
 * X(He4) / 4 * rho * N_A for alpha), the total energy flux, then one line per species whose
 * consider[i] is nonzero (all when consider is NULL): index, Z, A, isomeric state (1 when the array is
 * NULL), max(X, 1e-99) and the 5-character name (names: [nsp][5], not terminated). */
nuppn_status nuppn_write_iso_massf(const char *path, int32_t model, double dzeit, double agej, double t9, double rho,
                                   double densn, double densp, double densa, double total_energy_flux, int32_t nsp,
                                   const double *z, const double *a, const int32_t *isomeric_state, const double *x,
                                   const char *names, const uint8_t *consider);

/* flux_<mmmmm>.DAT (ppn.F90:496-510): one line per network reaction i < nreac with Z and A of its
 * k1, k3, k5 and k7 species (k: [nreac][8] 0-based species indices in the k1..k8 slot order of the
 * network description), max(flux, 1e-99), max(energy, 1e-99) and max(timescale, 1e99), as the
 * reference prints them (energy = flux * bind_energy_diff, in erg/(g s)). */
nuppn_status nuppn_write_flux(const char *path, int32_t nreac, const int32_t *k, const double *z, const double *a,
                              const double *flux, const double *energy, const double *timescale);

/* -- mppnp's diffusive mixing between mass shells (do_mixing with idifmix = 1,
 *    frames/mppnp/source/mixing.F90:34-342) ------------------------------------------------------ */

/* mix_calculate_D_Lagrangian (mixing.F90:60-98): d_lagr[j] = d_eul[j] (4 pi Rsun^2 / Msun)^2 exp(2 (2 ln r + ln rho)),
 * with ln r and ln rho averaged over shells j-1 and j (j > 0); 0 where d_eul <= 0. Host only. */
nuppn_status nuppn_mix_d_lagrangian(int32_t m, const double *d_eul, const double *rho, const double *rad,
                                    double *d_lagr);

/* mixdiff08 (mixing.F90:104-146): one fully implicit diffusion step of length dzeit over m shells for
 * the abundances X, element (shell j, species s) at X[j * shell_stride + s * species_stride]: either
 * rows of species (species_stride 1, shell_stride >= nsp) or columns of shells (shell_stride 1,
 * species_stride >= m; mppnp's yps(msl, nsp) passes shell_stride 1, species_stride msl). Every species
 * 0 .. nsp-2 whose consider[] is nonzero is mixed (all when consider is NULL; the last slot is left
 * alone, as mixdiff08 loops to NSP-1). mesa = 0: matrixdiffus on the mass coordinates xm[m]
 * (code_source GNV / EVL); mesa = 1: matrixdiffus_mesa on the shell masses dq[m] (MES). d_lagr[m]
 * (host) is limited in place by sig_term_limit as those routines limit it. The matrix and its
 * factorization are built on the host; the substitutions run on the GPU, one thread per species, with
 * tridag's operations in its order (equal to the reference bit for bit). NUPPN_ERR_ARG for a zero
 * pivot, a zero shell width or another layout. */
nuppn_status nuppn_mix_diffusion(int32_t m, int32_t nsp, double *X, int64_t shell_stride, int64_t species_stride,
                                 const double *xm, const double *dq, double *d_lagr, double dzeit,
                                 double sig_term_limit, int32_t mesa, const uint8_t *consider);

/* The same on device-resident abundances d_X, ordered on `stream` (a cudaStream_t, NULL: the default
 * stream); returns when the step is done. */
nuppn_status nuppn_mix_diffusion_device(int32_t m, int32_t nsp, double *d_X, int64_t shell_stride,
                                        int64_t species_stride, const double *xm, const double *dq, double *d_lagr,
                                        double dzeit, double sig_term_limit, int32_t mesa, const uint8_t *consider,
                                        void *stream);

/* -- tppnp's binary trajectory input (traj_data_bin_init / read_bin_trajectory,
 *    frames/tppnp/source/traj_data.F90:73-168): a stream file of the machine's byte order. Host only. */

/* The header: number of tracers and the smallest and largest time-step counts. */
nuppn_status nuppn_tppnp_header(const char *path, int32_t *num_tracers, int32_t *nsteps_min, int32_t *nsteps_max);

/* The tracer record at byte offset *pos (0: the first). With any of time..x NULL, only pnum, nsteps,
 * niso, mass, posini[3] and posfin[3] are set (to size the arrays) and *pos is left alone; otherwise
 * also time[nsteps] (s), t9[nsteps] (the file's temperature / 1e9, as read_trajectory divides it),
 * rho[nsteps] (g/cm^3), the initial composition a[niso], z[niso], zis[niso][5] (not terminated) and
 * x[niso], and *pos moves to the next tracer. NUPPN_ERR_ARG if the file is short or malformed. */
nuppn_status nuppn_tppnp_next(const char *path, int64_t *pos, int32_t *pnum, int32_t *nsteps, int32_t *niso,
                              double *mass, double *posini, double *posfin, double *time, double *t9, double *rho,
                              int32_t *a, int32_t *z, char *zis, double *x);

/* Static Jacobian pattern of makemap (jac_rhs.F90:461-540): row/col (0-based) of each COO entry in
 * the reference's row-major numbering, and dns2csr_map[nre][8] (entry index per slot, -1 if the
 * reaction is not considered). Sizes: row/col [nnz_jac]. */
nuppn_status nuppn_jac_pattern(const nuppn_net *net, int32_t *row, int32_t *col, int32_t *dns2csr_map);

/* evaluate_all_rates (evaluate_rates.F90:14-174) for nz zones: v[z*nre + r]. Host buffers. */
nuppn_status nuppn_eval_rates(nuppn_net *net, int32_t nz, const double *t9, const double *rho,
                              const double *ye, const double *X, int32_t ldx, double *v);

/* calculate_dxdt (jac_rhs.F90:217-278) from given rates: dxdt[z*nsp + i]. */
nuppn_status nuppn_dxdt(nuppn_net *net, int32_t nz, const double *v, const double *X, int32_t ldx,
                        double *dxdt);

/* calculate_jacobian (jac_rhs.F90:282-455) from given rates at step dt: jac values [z*nnz_jac + e]
 * (before the -dt scaling), entry set flags (row(e) /= -1) and the dynamic-network mask [z*nsp+i]. */
nuppn_status nuppn_jacobian(nuppn_net *net, int32_t nz, const double *v, const double *X, int32_t ldx,
                            const double *dt, double *jac, uint8_t *entry_set, uint8_t *mask);

/* One linear solve per zone of the reduced system that newton_iteration builds
 * (backward_euler.F90:133-148): (I - dt*J) x = b restricted to the mask, with the entry set flags
 * of nuppn_jacobian; x[z*nsp+i] = 0 for unmasked species. jac as returned by nuppn_jacobian. */
nuppn_status nuppn_solve_reduced(nuppn_net *net, int32_t nz, const double *jac,
                                 const uint8_t *entry_set, const uint8_t *mask, const double *dt,
                                 const double *b, double *x);

/* compute_nse (physics/source/nse_swj.F90:272-384) for nz zones from a fresh solver state (guess:
 * X(Ni56) = 1): the NSE mass fractions X[z*nsp + i] (1e-99 off the NSE set), the proton and neutron
 * chemical potentials (MeV), Newton iterations and the outcome code (0, BAD_YE, BAD_STEP or
 * NSE_CNVRG, where the reference stops the run). Host buffers. NUPPN_ERR_NET without protons or Ni56. */
nuppn_status nuppn_nse(nuppn_net *net, int32_t nz, const double *t9, const double *rho, const double *ye, double *X,
                       double *mu_p, double *mu_n, int32_t *iters, int32_t *ierr);

/* integrate_network (solver.F90:53-238), batched: every zone z advances X[z*ldx + :] over
 * dtwant[z] with its own sub-steps; ye[z] is updated; ierr[z] gets the reference's code. Rates are
 * evaluated at entry (the frames call evaluate_all_rates right before integrate_network) and again
 * whenever the interval-mean T9 or rho changes (solver.F90:146-150). stats may be NULL.
 * bd_state[z] carries what the reference keeps in saved module variables between calls of one
 * process: the Bader-Deuflhard optimal column kopt (bader_deuflhard.F90:32) and the first-call flag
 * frst (solver.F90:80). 0 = a fresh zone (frst true for its first sub-step, kopt from
 * bader_deuflhard_init); the call writes back the value to pass next time. May be NULL (all fresh). */
nuppn_status nuppn_integrate(nuppn_net *net, int32_t nz, double *X, int32_t ldx, const double *t9_0,
                             const double *t9_1, const double *rho_0, const double *rho_1, double *ye,
                             const double *dtwant, int32_t *ierr, nuppn_zone_stats *stats,
                             int32_t *bd_state);

/* Same on device-resident buffers (pointers from cudaMalloc in the caller's context) on the given
 * cudaStream_t (passed as void*; NULL = legacy default stream). Asynchronous: returns after launch. */
nuppn_status nuppn_integrate_device(nuppn_net *net, int32_t nz, double *d_X, int32_t ldx,
                                    const double *d_t9_0, const double *d_t9_1, const double *d_rho_0,
                                    const double *d_rho_1, double *d_ye, const double *d_dtwant,
                                    int32_t *d_ierr, nuppn_zone_stats *d_stats, int32_t *d_bd_state,
                                    void *stream);

/* integrate_network for zones of several networks in one launch: zone z uses nets[net_of_zone[z]]
 * (all handles on one device, at most 16), with that network's knobs; X rows have ldx >= the largest
 * nsp and zone z uses its first nsp entries. No counterpart routine in the reference, whose frames
 * run one network per process (NNN in ppn_physics.input); this is the uneven-size batch in which
 * zones of ~200-, ~1100- and ~2500-species networks advance together: one persistent launch of one
 * zone per CTA, every CTA's workspace sized for the largest network, zones taken hottest first, so
 * small and large systems share the GPU instead of running as separate waves. Other arguments and
 * outputs as for nuppn_integrate; a zone whose network index is out of range gets NUPPN_BAD_INPUT
 * (the host-buffer form rejects the call instead). */
nuppn_status nuppn_integrate_multi(nuppn_net *const *nets, int32_t nnets, int32_t nz, const int32_t *net_of_zone,
                                   double *X, int32_t ldx, const double *t9_0, const double *t9_1,
                                   const double *rho_0, const double *rho_1, double *ye, const double *dtwant,
                                   int32_t *ierr, nuppn_zone_stats *stats, int32_t *bd_state);

/* Same on device-resident buffers (d_net_of_zone included), asynchronous on the given stream. */
nuppn_status nuppn_integrate_multi_device(nuppn_net *const *nets, int32_t nnets, int32_t nz,
                                          const int32_t *d_net_of_zone, double *d_X, int32_t ldx,
                                          const double *d_t9_0, const double *d_t9_1, const double *d_rho_0,
                                          const double *d_rho_1, double *d_ye, const double *d_dtwant,
                                          int32_t *d_ierr, nuppn_zone_stats *d_stats, int32_t *d_bd_state,
                                          void *stream);

/* The trajectory loop of tppnp (frames/tppnp/source/tppnp.F90:131-168), batched: every zone z follows
 * its own trajectory of npts points time[z*npts + i], t9[...], rho[...]. The starting composition is
 * renormalised (Kahan sum) if |1 - sum X| > 1e-8; then for each interval i: Ye from the composition
 * (calculate_ye), integrate_network from point i to i+1, stop at the first interval with a non-zero
 * outcome (ierr[z] = that code, fail[z] = i; fail[z] = -1 when all succeed), and renormalise if
 * |1 - sum X| > 5e-7. Each zone carries its Bader-Deuflhard column and first-call flag between its
 * intervals (fresh for every trajectory). One launch for all intervals of all zones: zones with
 * few and many sub-steps share the GPU instead of waiting for each other interval by interval.
 * stats sum over the intervals (nvar1_max: maximum). fail and stats may be NULL. Host buffers. */
nuppn_status nuppn_integrate_trajectories(nuppn_net *net, int32_t nz, int32_t npts, double *X, int32_t ldx,
                                         const double *time, const double *t9, const double *rho, double *ye,
                                         int32_t *ierr, int32_t *fail, nuppn_zone_stats *stats);

/* Same on device-resident buffers, asynchronous on the given stream; bd_state as for
 * nuppn_integrate_device (0 = fresh). */
nuppn_status nuppn_integrate_trajectories_device(nuppn_net *net, int32_t nz, int32_t npts, double *d_X, int32_t ldx,
                                                const double *d_time, const double *d_t9, const double *d_rho,
                                                double *d_ye, int32_t *d_ierr, int32_t *d_fail,
                                                nuppn_zone_stats *d_stats, int32_t *d_bd_state, void *stream);

/* Same as nuppn_integrate_device, but this call allocates no device memory. It has no counterpart
 * in the reference (whose solver allocates through SuperLU on every call); it is for callers that
 * cannot call cudaMalloc while they step: programs that hand all of the GPU's memory to their own
 * allocator at start-up, or that keep cudaMalloc/cudaFree (which can synchronize the whole device)
 * out of their time-step loop. The handle itself is still made by nuppn_net_create at set-up.
 *
 * The per-CTA workspace and the zone counter live in one static device array of
 * NUPPN_NOALLOC_SCRATCH_BYTES (64 MiB), held on every GPU the library is used on until the process
 * exits. The call runs as many CTAs as whole workspace slabs fit in it (nuppn_net_info_get's
 * device_bytes does not count it); if one slab of this network does not fit it returns
 * NUPPN_ERR_LIMIT. The zone counter is cleared on the stream before each launch; the rest of the
 * array keeps the previous call's contents, which the kernel never reads before writing. Every call
 * on a device shares the array, so calls whose kernels overlap on the GPU (other streams, other
 * handles, other host threads) race: order them on one stream or synchronize between them.
 * The first call on a device looks up the array's address on that device (which may load the
 * library's device code); make that first call before any stream capture. The address is kept for
 * the life of the process: after cudaDeviceReset (which also frees every handle's device memory, so
 * the handles themselves are no longer usable) create new handles in a new process, not this one. */
#define NUPPN_NOALLOC_SCRATCH_BYTES (64u * 1024u * 1024u)
nuppn_status nuppn_integrate_device_noalloc(nuppn_net *net, int32_t nz, double *d_X, int32_t ldx,
                                            const double *d_t9_0, const double *d_t9_1,
                                            const double *d_rho_0, const double *d_rho_1, double *d_ye,
                                            const double *d_dtwant, int32_t *d_ierr,
                                            nuppn_zone_stats *d_stats, int32_t *d_bd_state, void *stream);

/* Number of kernel launches issued by the library since the handle was created (server launches
 * are counted by nuppn_serve_info). */
int64_t nuppn_launch_count(const nuppn_net *net);

/* ---- Autotuning of the integration kernel's shape ---------------------------------------------
 * No counterpart in the reference (one zone per MPI rank, no kernel to shape). The integration
 * kernel runs either one zone per CTA (every warp of the CTA shares the zone's wide phases, one warp
 * walks its dependency chains) or one zone per warp (each warp does all of its zone's work; several
 * zones per CTA). Which is faster depends on the network, on how many zones a call carries and on
 * how uneven their costs are, so nuppn_autotune measures it: it integrates the caller's batch (or
 * its first `sample` zones, 0 = all) once with each candidate shape from the same inputs, timed
 * with CUDA events, and keeps the shape with the most accepted zone sub-steps per second. Host
 * buffers as for nuppn_integrate; the inputs are not modified. The chosen shape is applied to the
 * handle (as nuppn_set_knobs would; the other knobs are unchanged). If `report` is not NULL, up to
 * `ncand` candidates are written there and *nreport gets their number. */
typedef struct nuppn_tune_result {
  int32_t threads_per_zone, zones_per_cta, zone_smem; /* the candidate's shape knobs                */
  int32_t zones_per_sm;                               /* zones resident per SM with that shape      */
  double ms;                                          /* one call over the sample                    */
  double zone_steps_per_s;                            /* accepted sub-steps per second               */
  int32_t chosen, reserved;
} nuppn_tune_result;
nuppn_status nuppn_autotune(nuppn_net *net, int32_t nz, const double *X, int32_t ldx, const double *t9_0,
                            const double *t9_1, const double *rho_0, const double *rho_1, const double *ye,
                            const double *dtwant, int32_t sample, nuppn_tune_result *report, int32_t ncand,
                            int32_t *nreport);

/* ---- Serving: a device-resident request loop ----------------------------------------------------
 * Each request is one call of integrate_network (solver.F90:53) for one zone, or one tppnp
 * trajectory (tppnp.F90:131-168), as the frames issue them one at a time; the server runs them on
 * the GPU as they arrive. The server keeps a persistent launch of the integration kernel on its own
 * stream. Its zone groups (the kernel shape of `net`: a CTA or a warp per zone) take requests one at
 * a time, in submission order, from a queue in device memory and write each result to host-mapped
 * memory as soon as that zone is done: a request that arrives while others are on the GPU starts
 * when any group is free, with no batch to wait for (continuous batching at zone granularity). A
 * host worker thread copies submitted requests into free queue slots, collects finished ones, and
 * relaunches the loop if it has left after staying idle (its groups leave after a few tens of
 * milliseconds without requests; every device wait is bounded). A request's result is the one
 * nuppn_integrate / nuppn_integrate_trajectories gives for it alone: zones never read one another's
 * state. The knobs are those of `net` when the server is opened; do not call nuppn_set_knobs or
 * destroy `net` while a server on it is open. Submit, poll and close from one host thread. Servers on
 * several handles (networks of different sizes) share the GPU: give each a share of the zone slots,
 * since a persistent loop holds its CTAs while it has work. */
typedef struct nuppn_server nuppn_server;

/* slots: zones integrated at once (0 = every zone slot the GPU holds for this kernel shape), rounded
 * down to whole CTAs and limited by admission: the workspace slabs (one per zone slot) must fit in
 * half of the free device memory (NUPPN_ERR_NOMEM if not even one CTA's worth fits). queue: requests
 * that can be on the device at once, waiting or running (0 = 4 x slots; at least slots). Trajectory
 * requests have at most 512 points (NUPPN_ERR_LIMIT beyond). */
nuppn_status nuppn_serve_open(nuppn_net *net, int32_t slots, int32_t queue, nuppn_server **out);

/* One zone: X[nsp] (copied at submit), interval T9/rho end points, Ye, dtwant, bd_state (0 = fresh,
 * as for nuppn_integrate). *id identifies the request in nuppn_serve_poll. */
nuppn_status nuppn_serve_submit(nuppn_server *srv, const double *X, double t9_0, double t9_1, double rho_0,
                                double rho_1, double ye, double dtwant, int32_t bd_state, int64_t *id);

/* One trajectory of npts points (time, t9, rho copied at submit), as for
 * nuppn_integrate_trajectories. */
nuppn_status nuppn_serve_submit_trajectory(nuppn_server *srv, const double *X, int32_t npts, const double *time,
                                           const double *t9, const double *rho, int64_t *id);

/* *done = 1 and the outputs filled (X[nsp], Ye, ierr, stats, bd_state, fail = failed interval or -1
 * for a trajectory) once the request has finished, after which its id is released; *done = 0 while
 * it is pending or on the GPU. Output pointers may be NULL. NUPPN_ERR_ARG for an unknown id;
 * NUPPN_ERR_CUDA if a CUDA call of the server failed (every request then fails). */
nuppn_status nuppn_serve_poll(nuppn_server *srv, int64_t id, int32_t *done, double *X, double *ye, int32_t *ierr,
                              nuppn_zone_stats *stats, int32_t *bd_state, int32_t *fail);

typedef struct {
  int32_t slots;            /* zones integrated at once                                   */
  int32_t queue;            /* queue slots on the device                                  */
  int32_t ctas;             /* CTAs of the persistent loop                                */
  int32_t pending;          /* submitted, waiting for a queue slot                        */
  int32_t in_flight;        /* in the device queue or running                             */
  int64_t launches;         /* launches of the persistent loop                            */
  int64_t published;        /* requests handed to the device                              */
  int64_t completed;        /* requests finished                                          */
  int64_t device_bytes;     /* device memory held by the server                           */
} nuppn_serve_stats;
nuppn_status nuppn_serve_info(nuppn_server *srv, nuppn_serve_stats *out);

/* Waits for the requests on the device, drops those still waiting for a queue slot, stops the loop
 * and frees everything. */
nuppn_status nuppn_serve_close(nuppn_server *srv);

#ifdef __cplusplus
}
#endif
#endif /* NUPPN_H */
