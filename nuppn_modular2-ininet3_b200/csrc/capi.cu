// capi.cu -- implementation of the C ABI declared in include/nuppn.h.
//
// The handle owns: the host analysis (HostNet), one device arena with every zone-shared network
// array (DevNet points into it), and a workspace of one slab per resident CTA. Host-buffer entry
// points stage their arguments through device buffers owned by the handle.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "net_host.h"
#include "nuppn_internal.h"

namespace nuppn {
namespace cta {  // solver.cu with one zone per CTA
cudaError_t launch_integrate(const DevNet &N, const WsLayout &L, char *ws, int grid, int block, int act_smem,
                             const IntegrateArgs &A, cudaStream_t st);
cudaError_t launch_phase(const DevNet &N, const WsLayout &L, char *ws, int grid, int block, int act_smem,
                         const PhaseArgs &A, cudaStream_t st);
cudaError_t configure_kernels(int dyn_smem);
cudaError_t launch_zone_order(const double *key, const double *key_b, int stride, int nz, int *order,
                              cudaStream_t st);
cudaError_t occupancy_integrate(int block, int act_smem, int *per_sm);
}  // namespace cta
namespace warp {  // solver.cu with one zone per warp
cudaError_t launch_integrate(const DevNet &N, const WsLayout &L, char *ws, int grid, int block, int act_smem,
                             const IntegrateArgs &A, cudaStream_t st);
cudaError_t configure_kernels(int dyn_smem);
cudaError_t occupancy_integrate(int block, int act_smem, int *per_sm);
}  // namespace warp
namespace cta {
cudaError_t launch_integrate_multi(const IntegrateArgs &A, char *ws, int grid, int act_smem, cudaStream_t st);
cudaError_t occupancy_integrate_multi(int act_smem, int *per_sm);
}  // namespace cta
using cta::launch_phase;
using cta::launch_zone_order;
}  // namespace nuppn

using namespace nuppn;

namespace {
std::mutex g_err_mu;
std::string g_last_error;

void set_error(const std::string &s) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  g_last_error = s;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

struct DevBuf {  // grow-only device buffer
  void *p = nullptr;
  size_t n = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= n) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaSuccess) n = bytes;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};
}  // namespace

struct nuppn_net {
  HostNet H;
  DevNet D;
  void *arena = nullptr;
  size_t arena_bytes = 0;
  WsLayout L;
  DevBuf ws, stage, counter, order;  // order: the zone schedule of the allocating entry points
  DevBuf multi;                      // networks' DevNet and WsLayout for nuppn_integrate_multi_device
  char *multi_host = nullptr;        // their pinned staging
  int ws_slots = 0;
  // integration kernel: one zone per CTA of `block` threads (warp_zones = 0), or one zone per warp
  // with `block` / 32 zones per CTA (warp_zones = 1); act_smem = shared memory of each zone's group
  int warp_zones = 0;
  int block = 256;
  int act_smem = 72 * 1024;  // CTA per zone: shared-memory budget per CTA for the active subsystem (3 CTAs per SM)
  int phase_block = 256;     // the parity entry points always run one zone per CTA of 256 threads
  int phase_smem = 72 * 1024;
  int device = 0;
  int nsm = 0;
  int64_t launches = 0;
};

#define CK(call)                                                                                  \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess) {                                                                      \
      set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                              \
      return NUPPN_ERR_CUDA;                                                                      \
    }                                                                                             \
  } while (0)

namespace {

// ---- arena upload ------------------------------------------------------------------------------
struct Arena {
  std::vector<std::pair<const void *, size_t>> items;
  std::vector<size_t> offs;
  size_t total = 0;
  template <class T>
  size_t add(const std::vector<T> &v) {
    size_t off = total;
    items.push_back({v.data(), v.size() * sizeof(T)});
    offs.push_back(off);
    total = align256(total + std::max<size_t>(v.size() * sizeof(T), 1));
    return off;
  }
};

nuppn_status upload(nuppn_net *net) {
  HostNet &H = net->H;
  DevNet &D = net->D;
  Arena A;
  // record offsets in a fixed sequence, then resolve to pointers
  std::vector<size_t> o;
  auto P = [&](auto &vec) { o.push_back(A.add(vec)); };
  P(H.an); P(H.zn); P(H.ciso); P(H.spart); P(H.gspin_nse);
  P(H.src); P(H.sidx); P(H.rfac); P(H.crea); P(H.rev_target); P(H.ilabb); P(H.scr_mode); P(H.scr_z1); P(H.scr_z2);
  P(H.irev); P(H.rev_sp); P(H.rev_kind); P(H.rev_mc); P(H.rev_Q);
  P(H.act_slot); P(H.act_k); P(H.act_ice);
  P(H.rl_first); P(H.rl_a); P(H.rl_info); P(H.rl_part); P(H.pt9); P(H.pval);
  P(H.vfirst); P(H.vxfac); P(H.vterms); P(H.vdpow); P(H.vform);
  P(H.ngt8); P(H.ngl10t8); P(H.ngflag); P(H.ngane); P(H.ngl10v); P(H.ngndata);
  P(H.fft9); P(H.ffrho); P(H.ffl10v); P(H.kdE); P(H.kdcoef); P(H.constr);
  P(H.jrow); P(H.jcol); P(H.jdiag); P(H.jg_ptr); P(H.jg_item); P(H.dg_ptr); P(H.dg_item); P(H.dg_coef);
  P(H.jg_long); P(H.dg_long); P(H.jg_oth);
  P(H.sys_of_sp); P(H.sp_of_sys); P(H.pos_of_entry); P(H.lu_src); P(H.lu_rowptr); P(H.lu_diag); P(H.lu_col); P(H.upd_start);
  P(H.upd_off); P(H.lvL_ptr); P(H.lvL_rows); P(H.lvL_grp); P(H.lvU_ptr); P(H.lvU_rows); P(H.lvU_grp);
  P(H.k1_ptr); P(H.k1_list);
  P(H.nse_idx); P(H.nse_part); P(H.nse_m); P(H.nse_q); P(H.nse_g); P(H.nse_z); P(H.nse_n); P(H.nse_zoa);
  CK(cudaMalloc(&net->arena, A.total));
  net->arena_bytes = A.total;
  std::vector<char> host(A.total, 0);
  for (size_t i = 0; i < A.items.size(); ++i)
    if (A.items[i].second) memcpy(host.data() + A.offs[i], A.items[i].first, A.items[i].second);
  CK(cudaMemcpy(net->arena, host.data(), A.total, cudaMemcpyHostToDevice));
  char *b = (char *)net->arena;
  size_t q = 0;
  auto nx = [&]() { return (void *)(b + o[q++]); };
  memset(&D, 0, sizeof(D));
  D.an = (const double *)nx(); D.zn = (const double *)nx(); D.ciso = (const uint8_t *)nx(); D.spart = (const int *)nx();
  D.gspin_nse = (const double *)nx();
  D.src = (const int *)nx(); D.sidx = (const int *)nx(); D.rfac = (const double *)nx(); D.crea = (const uint8_t *)nx();
  D.rev_target = (const uint8_t *)nx(); D.ilabb = (const int *)nx(); D.scr_mode = (const int *)nx();
  D.scr_z1 = (const double *)nx(); D.scr_z2 = (const double *)nx();
  D.irev = (const int *)nx(); D.rev_sp = (const int *)nx(); D.rev_kind = (const int *)nx();
  D.rev_mc = (const double *)nx(); D.rev_Q = (const double *)nx();
  D.act_slot = (const int *)nx(); D.act_k = (const int *)nx(); D.act_ice = (const int *)nx();
  D.rl_first = (const int *)nx(); D.rl_a = (const double *)nx(); D.rl_info = (const int *)nx();
  D.rl_part = (const int *)nx(); D.pt9 = (const double *)nx(); D.pval = (const double *)nx();
  D.vfirst = (const int *)nx(); D.vxfac = (const int *)nx(); D.vterms = (const double *)nx(); D.vdpow = (const double *)nx();
  D.vform = (const int *)nx();
  D.ngt8 = (const double *)nx(); D.ngl10t8 = (const double *)nx(); D.ngflag = (const double *)nx();
  D.ngane = (const double *)nx(); D.ngl10v = (const double *)nx(); D.ngndata = (const int *)nx();
  D.fft9 = (const double *)nx(); D.ffrho = (const double *)nx(); D.ffl10v = (const double *)nx();
  D.kdE = (const double *)nx(); D.kdcoef = (const double *)nx(); D.constr = (const double *)nx();
  D.jrow = (const int *)nx(); D.jcol = (const int *)nx(); D.jdiag = (const int *)nx();
  D.jg_ptr = (const int *)nx(); D.jg_item = (const int *)nx(); D.dg_ptr = (const int *)nx();
  D.dg_item = (const int *)nx(); D.dg_coef = (const double *)nx();
  D.jg_long = (const int *)nx(); D.dg_long = (const int *)nx(); D.jg_oth = (const int *)nx();
  D.sys_of_sp = (const int *)nx(); D.sp_of_sys = (const int *)nx(); D.pos_of_entry = (const int *)nx();
  D.lu_src = (const int *)nx();
  D.lu_rowptr = (const int *)nx(); D.lu_diag = (const int *)nx(); D.lu_col = (const int *)nx();
  D.upd_start = (const int *)nx(); D.upd_off = (const uint16_t *)nx();
  D.lvL_ptr = (const int *)nx(); D.lvL_rows = (const int *)nx(); D.lvL_grp = (const int *)nx();
  D.lvU_ptr = (const int *)nx(); D.lvU_rows = (const int *)nx(); D.lvU_grp = (const int *)nx();
  D.k1_ptr = (const int *)nx(); D.k1_list = (const int *)nx();
  D.nse_idx = (const int *)nx(); D.nse_part = (const int *)nx(); D.nse_m = (const double *)nx();
  D.nse_q = (const double *)nx(); D.nse_g = (const double *)nx(); D.nse_z = (const double *)nx();
  D.nse_n = (const double *)nx(); D.nse_zoa = (const double *)nx();
  D.nse_num = (int)H.nse_idx.size(); D.nse_iprot = H.nse_iprot; D.nse_ini56 = H.nse_ini56; D.nse_p2 = H.nse_p2;
  // scalars
  D.nsp = H.nsp; D.nre = H.nre; D.nact = H.nact; D.ig = H.ig; D.nsys = H.nsys; D.nnzJ = H.nnzJ; D.nnzLU = H.nnzLU;
  D.ihe4 = H.ihe4; D.ibe8 = H.ibe8;
  D.nc = H.nc; D.nr = H.nr; D.npart = H.npart; D.nv = H.nv;
  D.ngk = H.ngk; D.ngn = H.ngn; D.ngd = H.ngd; D.ffv = H.ffv; D.fft = H.fft; D.ffr = H.ffr;
  D.kdn = H.kdn; D.kde = H.kde;
  D.njg_long = (int)H.jg_long.size(); D.ndg_long = (int)H.dg_long.size(); D.ndg_item = (int)H.dg_item.size();
  D.nlvL = (int)H.lvL_ptr.size() - 1; D.nlvU = (int)H.lvU_ptr.size() - 1;
  memcpy(D.nseq, H.nseq, sizeof(D.nseq));
  memcpy(D.bd_a, H.bd_a, sizeof(D.bd_a));
  memcpy(D.alf, H.alf, sizeof(D.alf));
  D.kmax = H.kmax; D.kopt0 = H.kopt0;
  D.kn = H.kn;
  D.nvar = H.nvar;
  return NUPPN_OK;
}

WsLayout layout(const HostNet &H) {
  WsLayout L;
  size_t t = 0;
  auto take = [&](size_t bytes) { size_t o = t; t = align256(t + std::max<size_t>(bytes, 8)); return o; };
  const size_t d = sizeof(double);
  L.v = take(H.nre * d); L.rv = take(H.nr * d); L.ngv = take(H.ngn * d); L.ffv = take(H.ffv * d);
  L.kdv = take(H.kdn * d); L.partinter = take(H.npart * d); L.G = take(H.nsp * d); L.flux = take(H.nact * d);
  L.contrib = take(std::max<size_t>((size_t)H.nact * 8, H.nre) * d); L.first_l = take(H.nsp * sizeof(int));
  L.eset = take(H.nnzJ); L.jac = take(H.nnzJ * d); L.mask = take(H.nsp); L.xn = take(H.nsp * d);
  L.dxdt = take(H.nsp * d); L.y = take(H.nsp * d); L.y_old = take(H.nsp * d); L.y_cur = take(H.nsp * d);
  L.y_new = take(H.nsp * d); L.y_k = take(H.nsp * d); L.delta_k = take(H.nsp * d); L.y_ext = take(H.nsp * d);
  L.yscal = take(H.nsp * d); L.qcol = take((size_t)(kMaxLevels + 1) * H.nsp * d);
  L.yerr = take((size_t)(kMaxLevels + 1) * H.nsp * d); L.lu = take((size_t)H.nnzLU * d);
  L.bsys = take(H.nsys * d); L.xsys = take(H.nsys * d); L.rhs = take(H.nsp * d);
  L.act_tmp = take((size_t)4 * (H.nsys + 1) * sizeof(int));
  L.act = take(act_bytes_max(H.nsys, H.nnzLU, 8));
  {
    size_t ngi = H.dg_item.size();
    L.act_r = take(rhs_bytes(H.nsys, (int)ngi));
    size_t njg = H.jg_item.size();
    L.act_otmp = take(((size_t)H.nnzLU + 1) * sizeof(int));
    L.act_dtmp = take(njg * sizeof(double));
    L.act_btmp = take(njg);
    L.bd = take((size_t)(2 * kMaxLevels + 8) * H.nsys * sizeof(double));
  }
  {
    const size_t ngi = H.dg_item.size();
    L.rhs_key = take(ngi * sizeof(int));
    L.rhs_val = take(ngi * sizeof(double));
    const size_t npmax = ((size_t)H.nsys + 1) + ngi / kRhsPiece + 1;  // pieces of the active rows, at most
    L.rhs_piece = take(((size_t)H.nsys + 1 + 4 * npmax) * sizeof(int));
    const size_t keys = (size_t)kRhsWarps * kRhsKeysPerRow * ((size_t)H.nsys + 1);
    L.rhs_acc = take(keys * sizeof(double));
    L.rhs_tag = take(keys * sizeof(int));
    L.rhs_list = take(keys * sizeof(int));
    L.rhs_spc = take((size_t)H.nsp * sizeof(int));
    L.cache_mask = take((size_t)H.nsp);
    L.cache_xn = take((size_t)H.nsp * sizeof(double));
    L.rhs_rkey = take((size_t)H.nact * sizeof(int));
    L.rhs_rcf = take((size_t)H.nact * sizeof(double));
    L.rhs_rpk = take((size_t)H.nact * sizeof(uint32_t));
    L.jac_long = take(3 * ((size_t)H.nnzLU + 1) * sizeof(int));
  }
  L.nse = take((5 * (size_t)H.nsp + (size_t)H.nse_p2) * sizeof(double));
  L.nse_stride = (size_t)H.nsp;
  L.bytes = t;
  return L;
}

nuppn_status ensure_ws(nuppn_net *net, int slots) {
  if (slots <= net->ws_slots) return NUPPN_OK;
  CK(net->ws.ensure((size_t)slots * net->L.bytes));
  net->ws_slots = slots;
  return NUPPN_OK;
}

int zones_per_cta(const nuppn_net *net) { return net->warp_zones ? net->block / 32 : 1; }

// CTAs of the integration kernel resident on the whole GPU
int resident_ctas(const nuppn_net *net) {
  int per = 0;
  cudaError_t e = net->warp_zones ? warp::occupancy_integrate(net->block, net->act_smem, &per)
                                  : cta::occupancy_integrate(net->block, net->act_smem, &per);
  if (e != cudaSuccess || per <= 0) per = 1;
  return per * net->nsm;
}

// zones in flight at once (one workspace slab each)
int resident_slots(const nuppn_net *net) { return resident_ctas(net) * zones_per_cta(net); }

// CTAs of the parity kernel (one zone per CTA of phase_block threads)
int phase_slots(const nuppn_net *net) {
  int per = 0;
  if (cta::occupancy_integrate(net->phase_block, net->phase_smem, &per) != cudaSuccess || per <= 0) per = 1;
  return per * net->nsm;
}

// CTAs for nz zones: whole CTAs' worth of zones, at most the resident CTAs and `slabs` workspace slabs
int integrate_grid(const nuppn_net *net, int nz, int slabs) {
  const int zpc = zones_per_cta(net);
  int grid = std::min((nz + zpc - 1) / zpc, resident_ctas(net));
  return std::max(1, std::min(grid, slabs / zpc));
}

cudaError_t launch_integrate_net(const nuppn_net *net, char *ws, int grid, const IntegrateArgs &A, cudaStream_t s) {
  return net->warp_zones ? warp::launch_integrate(net->D, net->L, ws, grid, net->block, net->act_smem, A, s)
                         : cta::launch_integrate(net->D, net->L, ws, grid, net->block, net->act_smem, A, s);
}

// Largest dynamic shared memory of one CTA of the warp-per-zone kernel: the 227 KB opt-in limit
// per CTA less the kernel's ~7 KB of static arrays (per-warp reduction and scan scratch, long-entry
// lists) and a margin.
constexpr int kWarpCtaSmem = 216 * 1024;

nuppn_status check_shape(const nuppn_knobs &kn) {
  const int t = kn.threads_per_zone;
  if (t < 0 || t % 32 || t > 256) {
    set_error("threads_per_zone must be 0 or a multiple of 32 up to 256");
    return NUPPN_ERR_ARG;
  }
  if (kn.zones_per_cta < 0 || kn.zones_per_cta > 8) {
    set_error("zones_per_cta must be 0..8");
    return NUPPN_ERR_ARG;
  }
  if (kn.zone_smem < 0 || kn.zone_smem > kWarpCtaSmem) {
    set_error("zone_smem must be 0..216 KB");
    return NUPPN_ERR_ARG;
  }
  return NUPPN_OK;
}

// Kernel shape from the knobs: one zone per warp (threads_per_zone = 32) or one per CTA, the CTA
// size and each zone's shared memory; sets the kernels' dynamic shared-memory limits to match.
nuppn_status apply_shape(nuppn_net *net, const nuppn_knobs &kn) {
  net->warp_zones = kn.threads_per_zone == 32 ? 1 : 0;
  if (net->warp_zones) {
    const int zpc = kn.zones_per_cta > 0 ? kn.zones_per_cta : 8;
    net->block = 32 * zpc;
    const int share = (kWarpCtaSmem / zpc) & ~15;
    net->act_smem = kn.zone_smem > 0 ? std::min(kn.zone_smem & ~15, share) : share;
    net->phase_block = 256;
  } else {
    net->block = kn.threads_per_zone > 0 ? kn.threads_per_zone : 256;
    net->act_smem = kn.zone_smem > 0 ? (kn.zone_smem & ~15) : 72 * 1024;
    net->phase_block = net->block;
  }
  net->phase_smem = net->warp_zones ? 72 * 1024 : net->act_smem;
  cudaError_t e = cta::configure_kernels(std::max(net->phase_smem, net->warp_zones ? 0 : net->act_smem));
  if (e == cudaSuccess && net->warp_zones) e = warp::configure_kernels(net->act_smem * zones_per_cta(net));
  if (e != cudaSuccess) {
    set_error(std::string("cannot configure dynamic shared memory: ") + cudaGetErrorString(e));
    return NUPPN_ERR_CUDA;
  }
  return NUPPN_OK;
}

nuppn_status check_zone_args(nuppn_net *net, int nz, int ldx) {
  if (!net) { set_error("null handle"); return NUPPN_ERR_ARG; }
  if (nz < 0) { set_error("nz < 0"); return NUPPN_ERR_ARG; }
  if (ldx < net->H.nsp) { set_error("ldx < nsp"); return NUPPN_ERR_ARG; }
  return NUPPN_OK;
}

// stage host arrays into the handle's device staging buffer
struct Stager {
  std::vector<std::pair<size_t, size_t>> parts;  // (offset, bytes)
  size_t total = 0;
  size_t add(size_t bytes) {
    size_t o = total;
    total = align256(total + std::max<size_t>(bytes, 8));
    return o;
  }
};

}  // namespace

// ---- scratch for nuppn_integrate_device_noalloc -------------------------------------------------
// One fixed device array holds that entry point's zone counter (first 256 bytes) and its per-CTA
// workspace slabs, so the call needs no cudaMalloc. In host code the name g_noalloc_scratch is
// only a host-side stand-in for the symbol: kernels get the address cudaGetSymbolAddress returns,
// looked up on every call with the device current, so neither a device reset nor another context
// made current on that device leaves a stale address behind.
static __device__ __align__(256) char g_noalloc_scratch[NUPPN_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr size_t kNoAllocCounterBytes = 256;

// Device address of the scratch array in the current context (on `device`, which must be current).
cudaError_t noalloc_scratch(int device, void **out) {
  if (device < 0) return cudaErrorInvalidDevice;
  return cudaGetSymbolAddress(out, g_noalloc_scratch);
}
}  // namespace

extern "C" {

int32_t nuppn_abi_version(void) { return NUPPN_ABI_VERSION; }

void nuppn_default_knobs(nuppn_knobs *k) {
  if (!k) return;
  memset(k, 0, sizeof(*k));
  k->ittd = 6; k->integration_method = 0; k->max_sub_steps = 4000;
  k->interpolate_temp = 1; k->interpolate_dens = 1; k->screen_option = 2; k->detailed_balance = 1;
  k->weak_rates = 1; k->strong_rates = 1; k->decay = 0; k->i_nse = 0; k->nse_weak_method = 1;
  k->dgrd = 1.e-3; k->grdthreshold = 1.e-15; k->cyminformal = 1.0e-30; k->min_rate_ov_dt = 1.e-99;
  k->min_t9_for_slv = 0.01; k->delta_state_max = 1.e99; k->nse_min_t9 = 6.0;
  k->lu_precision = 0; k->ir_max_iters = 3; k->ir_rtol = 1e-14; k->threads_per_zone = 0;
}

const char *nuppn_status_string(nuppn_status s) {
  switch (s) {
    case NUPPN_OK: return "ok";
    case NUPPN_ERR_ARG: return "bad argument";
    case NUPPN_ERR_CUDA: return "CUDA error";
    case NUPPN_ERR_NOMEM: return "out of memory";
    case NUPPN_ERR_NET: return "inconsistent network";
    case NUPPN_ERR_LIMIT: return "size limit";
    case NUPPN_ERR_NODEV: return "no sm_100 device";
    case NUPPN_ERR_TIMEOUT: return "device wait timed out";
  }
  return "unknown";
}

const char *nuppn_last_error(void) {
  static thread_local std::string copy;
  std::lock_guard<std::mutex> lk(g_err_mu);
  copy = g_last_error;
  return copy.c_str();
}

nuppn_status nuppn_net_create(const nuppn_net_desc *desc, const nuppn_knobs *knobs, int32_t device, nuppn_net **out) {
  if (!desc || !out) { set_error("null argument"); return NUPPN_ERR_ARG; }
  *out = nullptr;
  nuppn_knobs kn;
  if (knobs) kn = *knobs; else nuppn_default_knobs(&kn);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0) {
    set_error("no CUDA device");
    return NUPPN_ERR_NODEV;
  }
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) { set_error("device is not sm_100 or newer"); return NUPPN_ERR_NODEV; }
  CK(cudaSetDevice(device));
  nuppn_net *net = new (std::nothrow) nuppn_net();
  if (!net) return NUPPN_ERR_NOMEM;
  std::string msg = build_host_net(*desc, kn, net->H);
  if (!msg.empty()) {
    set_error(msg);
    delete net;
    return NUPPN_ERR_NET;
  }
  net->device = device;
  net->nsm = prop.multiProcessorCount;
  if (kn.lu_precision != 0 && kn.lu_precision != 1) {
    delete net;
    set_error("lu_precision must be 0 (FP64) or 1 (FP32 factor + FP64 refinement)");
    return NUPPN_ERR_ARG;
  }
  nuppn_status st = check_shape(kn);
  if (st != NUPPN_OK) { delete net; return st; }
  st = upload(net);
  if (st != NUPPN_OK) { delete net; return st; }
  st = apply_shape(net, kn);
  if (st != NUPPN_OK) { nuppn_net_destroy(net); return st; }
  net->L = layout(net->H);
  if (net->counter.ensure(256) != cudaSuccess) { delete net; set_error("counter alloc"); return NUPPN_ERR_NOMEM; }
  *out = net;
  return NUPPN_OK;
}

nuppn_status nuppn_net_destroy(nuppn_net *net) {
  if (!net) return NUPPN_OK;
  cudaSetDevice(net->device);
  if (net->arena) cudaFree(net->arena);
  net->ws.release();
  net->stage.release();
  net->counter.release();
  net->order.release();
  net->multi.release();
  if (net->multi_host) cudaFreeHost(net->multi_host);
  delete net;
  return NUPPN_OK;
}

nuppn_status nuppn_net_info_get(const nuppn_net *net, nuppn_net_info *info) {
  if (!net || !info) return NUPPN_ERR_ARG;
  const HostNet &H = net->H;
  info->nsp = H.nsp; info->nre = H.nre; info->nspec_active = H.nvar; info->nreac_active = H.nact;
  info->nnz_jac = H.nnzJ; info->nnz_lu = H.nnzLU; info->n_solve = H.nsys;
  info->levels_lower = (int)H.lvL_ptr.size() - 1; info->levels_upper = (int)H.lvU_ptr.size() - 1;
  info->lu_flops = H.lu_flops;
  info->device_bytes = (int64_t)(net->arena_bytes + net->ws.n + net->stage.n + net->counter.n + net->order.n);
  return NUPPN_OK;
}

nuppn_status nuppn_set_knobs(nuppn_net *net, const nuppn_knobs *knobs) {
  if (!net || !knobs) return NUPPN_ERR_ARG;
  if (knobs->lu_precision != 0 && knobs->lu_precision != 1) {
    set_error("lu_precision must be 0 (FP64) or 1 (FP32 factor + FP64 refinement)");
    return NUPPN_ERR_ARG;
  }
  if (knobs->i_nse == 1 && (net->H.nse_iprot < 0 || net->H.nse_ini56 < 0)) {
    set_error("i_nse = 1 needs protons and Ni56 among the considered species");
    return NUPPN_ERR_NET;
  }
  nuppn_status sh = check_shape(*knobs);
  if (sh != NUPPN_OK) return sh;
  sh = apply_shape(net, *knobs);  // the workspace grows on the next call if the shape needs more slabs
  if (sh != NUPPN_OK) return sh;
  double old_dgrd = net->H.kn.dgrd;
  net->H.kn = *knobs;
  if (knobs->dgrd != old_dgrd) bd_constants(net->H);
  memcpy(net->D.nseq, net->H.nseq, sizeof(net->D.nseq));
  memcpy(net->D.bd_a, net->H.bd_a, sizeof(net->D.bd_a));
  memcpy(net->D.alf, net->H.alf, sizeof(net->D.alf));
  net->D.kmax = net->H.kmax; net->D.kopt0 = net->H.kopt0;
  net->D.kn = *knobs;
  return NUPPN_OK;
}

nuppn_status nuppn_isotopedatabase_read(const char *path, int32_t nnn, int32_t *z, int32_t *a, uint8_t *consider,
                                        char *elem) {
  std::vector<IsotopeEntry> e;
  const std::string err = read_isotope_database(path, nnn, e);
  if (!err.empty()) {
    set_error(err);
    return err.find("fewer than") != std::string::npos ? NUPPN_ERR_LIMIT : NUPPN_ERR_ARG;
  }
  for (size_t i = 0; i < e.size(); ++i) {
    if (z) z[i] = e[i].z;
    if (a) a[i] = e[i].a;
    if (consider) consider[i] = e[i].consider ? 1 : 0;
    if (elem) memcpy(elem + 3 * i, e[i].elem, 3);
  }
  return NUPPN_OK;
}

nuppn_status nuppn_networksetup_write(const char *path, const nuppn_netsetup *ns) {
  if (!ns) { set_error("null argument"); return NUPPN_ERR_ARG; }
  const std::string err = write_networksetup(path, *ns);
  if (!err.empty()) { set_error(err); return NUPPN_ERR_ARG; }
  return NUPPN_OK;
}

nuppn_status nuppn_networksetup_read(const char *path, nuppn_netsetup *ns) {
  if (!ns) { set_error("null argument"); return NUPPN_ERR_ARG; }
  const std::string err = read_networksetup(path, *ns);
  if (!err.empty()) { set_error(err); return NUPPN_ERR_ARG; }
  return NUPPN_OK;
}

nuppn_status nuppn_write_iso_massf(const char *path, int32_t model, double dzeit, double agej, double t9, double rho,
                                   double densn, double densp, double densa, double total_energy_flux, int32_t nsp,
                                   const double *z, const double *a, const int32_t *isomeric_state, const double *x,
                                   const char *names, const uint8_t *consider) {
  if (!path || nsp < 0 || (nsp > 0 && (!z || !a || !x || !names))) { set_error("null argument"); return NUPPN_ERR_ARG; }
  if (!write_iso_massf(path, model, dzeit, agej, t9, rho, densn, densp, densa, total_energy_flux, nsp, z, a,
                       isomeric_state, x, names, consider)) {
    set_error(std::string("cannot write ") + path);
    return NUPPN_ERR_ARG;
  }
  return NUPPN_OK;
}

nuppn_status nuppn_write_flux(const char *path, int32_t nreac, const int32_t *k, const double *z, const double *a,
                              const double *flux, const double *energy, const double *timescale) {
  if (!path || nreac < 0 || (nreac > 0 && (!k || !z || !a || !flux || !energy || !timescale))) {
    set_error("null argument");
    return NUPPN_ERR_ARG;
  }
  if (!write_flux(path, nreac, k, z, a, flux, energy, timescale)) {
    set_error(std::string("cannot write ") + path);
    return NUPPN_ERR_ARG;
  }
  return NUPPN_OK;
}

}  // extern "C"

namespace nuppn {
cudaError_t launch_mix_columns(int m, int ncol, double *X, long long shell_stride, long long species_stride,
                               const double *a, const double *gam, const double *bet, const unsigned char *cons,
                               cudaStream_t stream);
}

namespace {

// The step's matrix and factorization for nuppn_mix_diffusion*; d_lagr is limited in place as
// matrixdiffus limits it. The abundances are either rows of species (species_stride 1, shell_stride >=
// nsp) or columns of shells (shell_stride 1, species_stride >= m, mppnp's yps(msl, nsp)); *extent is the
// elements the array spans.
nuppn_status mix_prepare(int32_t m, int32_t nsp, int64_t shell_stride, int64_t species_stride, const double *xm,
                         const double *dq, double *d_lagr, double dzeit, double sig, int32_t mesa,
                         std::vector<double> &a, std::vector<double> &gam, std::vector<double> &bet,
                         int64_t *extent) {
  const bool rows = species_stride == 1 && shell_stride >= nsp;
  const bool cols = shell_stride == 1 && species_stride >= m;
  if (m < 2 || nsp < 1 || !(rows || cols) || !d_lagr || (mesa ? !dq : !xm)) {
    set_error("nuppn_mix_diffusion: m >= 2, nsp >= 1, rows of species (species_stride 1, shell_stride >= nsp) "
              "or columns of shells (shell_stride 1, species_stride >= m), d_lagr and xm (or dq with mesa) "
              "required");
    return NUPPN_ERR_ARG;
  }
  *extent = (int64_t)(m - 1) * shell_stride + (int64_t)(nsp - 1) * species_stride + 1;
  std::vector<double> b, c;
  std::string err = mix_matrix(m, xm, dq, d_lagr, dzeit, sig, mesa != 0, a, b, c);
  if (err.empty()) err = tridag_factor(m, a, b, c, gam, bet);
  if (!err.empty()) {
    set_error("nuppn_mix_diffusion: " + err);
    return NUPPN_ERR_ARG;
  }
  return NUPPN_OK;
}

}  // namespace

extern "C" {

nuppn_status nuppn_mix_d_lagrangian(int32_t m, const double *d_eul, const double *rho, const double *rad,
                                    double *d_lagr) {
  if (m < 1 || !d_eul || !rho || !rad || !d_lagr) { set_error("null argument"); return NUPPN_ERR_ARG; }
  mix_d_lagrangian(m, d_eul, rho, rad, d_lagr);
  return NUPPN_OK;
}

nuppn_status nuppn_mix_diffusion_device(int32_t m, int32_t nsp, double *d_X, int64_t shell_stride,
                                        int64_t species_stride, const double *xm, const double *dq, double *d_lagr,
                                        double dzeit, double sig_term_limit, int32_t mesa, const uint8_t *consider,
                                        void *stream) {
  if (!d_X) { set_error("null argument"); return NUPPN_ERR_ARG; }
  std::vector<double> a, gam, bet;
  int64_t extent = 0;
  const nuppn_status st = mix_prepare(m, nsp, shell_stride, species_stride, xm, dq, d_lagr, dzeit, sig_term_limit,
                                      mesa, a, gam, bet, &extent);
  if (st != NUPPN_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t vb = (size_t)m * sizeof(double);
  char *buf = nullptr;
  CK(cudaMallocAsync((void **)&buf, 3 * vb + (size_t)nsp, s));
  double *da = (double *)buf, *dg = da + m, *db = dg + m;
  unsigned char *dc = consider ? (unsigned char *)(buf + 3 * vb) : nullptr;
  cudaError_t e = cudaMemcpyAsync(da, a.data(), vb, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dg, gam.data(), vb, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(db, bet.data(), vb, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && dc) e = cudaMemcpyAsync(dc, consider, (size_t)nsp, cudaMemcpyHostToDevice, s);
  // mixdiff08 (mixing.F90:131-140) mixes species 1 .. NSP-1: the last slot is left alone
  if (e == cudaSuccess)
    e = nuppn::launch_mix_columns(m, nsp - 1, d_X, shell_stride, species_stride, da, dg, db, dc, s);
  const cudaError_t f = cudaFreeAsync(buf, s);
  if (e == cudaSuccess) e = f;
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the host vectors of the copies go out of scope
  if (e != cudaSuccess) {
    set_error(std::string("nuppn_mix_diffusion: ") + cudaGetErrorString(e));
    return NUPPN_ERR_CUDA;
  }
  return NUPPN_OK;
}

nuppn_status nuppn_mix_diffusion(int32_t m, int32_t nsp, double *X, int64_t shell_stride, int64_t species_stride,
                                 const double *xm, const double *dq, double *d_lagr, double dzeit,
                                 double sig_term_limit, int32_t mesa, const uint8_t *consider) {
  if (!X) { set_error("null argument"); return NUPPN_ERR_ARG; }
  int64_t extent = 0;
  {  // the matrix and its factorization first, on a copy of d_lagr: argument errors need no GPU
    std::vector<double> a, gam, bet, dcopy(d_lagr ? d_lagr : nullptr, d_lagr ? d_lagr + std::max(m, 0) : nullptr);
    const nuppn_status st = mix_prepare(m, nsp, shell_stride, species_stride, xm, dq, d_lagr ? dcopy.data() : nullptr,
                                        dzeit, sig_term_limit, mesa, a, gam, bet, &extent);
    if (st != NUPPN_OK) return st;
  }
  const size_t bytes = (size_t)extent * sizeof(double);
  double *dX = nullptr;
  CK(cudaMalloc((void **)&dX, bytes));
  cudaError_t e = cudaMemcpy(dX, X, bytes, cudaMemcpyHostToDevice);
  nuppn_status st = NUPPN_ERR_CUDA;
  if (e == cudaSuccess) {
    st = nuppn_mix_diffusion_device(m, nsp, dX, shell_stride, species_stride, xm, dq, d_lagr, dzeit, sig_term_limit,
                                    mesa, consider, nullptr);
    if (st == NUPPN_OK) {
      e = cudaMemcpy(X, dX, bytes, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) {
        set_error(std::string("nuppn_mix_diffusion: ") + cudaGetErrorString(e));
        st = NUPPN_ERR_CUDA;
      }
    }
  } else {
    set_error(std::string("nuppn_mix_diffusion: ") + cudaGetErrorString(e));
  }
  cudaFree(dX);
  return st;
}

nuppn_status nuppn_tppnp_header(const char *path, int32_t *num_tracers, int32_t *nsteps_min, int32_t *nsteps_max) {
  if (!path || !num_tracers || !nsteps_min || !nsteps_max) { set_error("null argument"); return NUPPN_ERR_ARG; }
  int n = 0, lo = 0, hi = 0;
  const std::string err = tppnp_header(path, &n, &lo, &hi);
  if (!err.empty()) { set_error(err); return NUPPN_ERR_ARG; }
  *num_tracers = n; *nsteps_min = lo; *nsteps_max = hi;
  return NUPPN_OK;
}

nuppn_status nuppn_tppnp_next(const char *path, int64_t *pos, int32_t *pnum, int32_t *nsteps, int32_t *niso,
                              double *mass, double *posini, double *posfin, double *time, double *t9, double *rho,
                              int32_t *a, int32_t *z, char *zis, double *x) {
  if (!path || !pos || !pnum || !nsteps || !niso) { set_error("null argument"); return NUPPN_ERR_ARG; }
  int pn = 0, nt = 0, ni = 0;
  const std::string err = tppnp_next(path, pos, &pn, &nt, &ni, mass, posini, posfin, time, t9, rho, a, z, zis, x);
  if (!err.empty()) { set_error(err); return NUPPN_ERR_ARG; }
  *pnum = pn; *nsteps = nt; *niso = ni;
  return NUPPN_OK;
}

nuppn_status nuppn_jac_pattern(const nuppn_net *net, int32_t *row, int32_t *col, int32_t *map) {
  if (!net) return NUPPN_ERR_ARG;
  const HostNet &H = net->H;
  if (row) memcpy(row, H.jrow.data(), H.jrow.size() * sizeof(int));
  if (col) memcpy(col, H.jcol.data(), H.jcol.size() * sizeof(int));
  if (map) memcpy(map, H.dmap_all.data(), H.dmap_all.size() * sizeof(int));
  return NUPPN_OK;
}

int64_t nuppn_launch_count(const nuppn_net *net) { return net ? net->launches : 0; }

nuppn_status nuppn_integrate_device_noalloc(nuppn_net *net, int32_t nz, double *d_X, int32_t ldx,
                                            const double *d_t9_0, const double *d_t9_1, const double *d_rho_0,
                                            const double *d_rho_1, double *d_ye, const double *d_dtwant,
                                            int32_t *d_ierr, nuppn_zone_stats *d_stats, int32_t *d_bd_state,
                                            void *stream) {
  nuppn_status st = check_zone_args(net, nz, ldx);
  if (st != NUPPN_OK) return st;
  if (nz == 0) return NUPPN_OK;
  if (!d_X || !d_t9_0 || !d_t9_1 || !d_rho_0 || !d_rho_1 || !d_ye || !d_dtwant || !d_ierr) {
    set_error("null device argument");
    return NUPPN_ERR_ARG;
  }
  const size_t slab = net->L.bytes;
  if (kNoAllocCounterBytes + slab > (size_t)NUPPN_NOALLOC_SCRATCH_BYTES) {
    set_error("nuppn_integrate_device_noalloc: this network needs " + std::to_string(slab) +
              " bytes of workspace per CTA, more than the static scratch of " +
              std::to_string((size_t)NUPPN_NOALLOC_SCRATCH_BYTES) + " bytes; use nuppn_integrate_device");
    return NUPPN_ERR_LIMIT;
  }
  CK(cudaSetDevice(net->device));
  void *base = nullptr;
  CK(noalloc_scratch(net->device, &base));
  const int slabs = (int)(((size_t)NUPPN_NOALLOC_SCRATCH_BYTES - kNoAllocCounterBytes) / slab);
  if (slabs < zones_per_cta(net)) {
    set_error("nuppn_integrate_device_noalloc: the static scratch holds " + std::to_string(slabs) +
              " workspace slabs of this network, fewer than the zones of one CTA (" +
              std::to_string(zones_per_cta(net)) + "); use fewer zones_per_cta or nuppn_integrate_device");
    return NUPPN_ERR_LIMIT;
  }
  const int grid = integrate_grid(net, nz, slabs);
  cudaStream_t s = (cudaStream_t)stream;
  CK(cudaMemsetAsync(base, 0, sizeof(int), s));  // the zone counter starts at zero every call
  IntegrateArgs A = {};
  A.nz = nz; A.ldx = ldx; A.X = d_X; A.t9_0 = d_t9_0; A.t9_1 = d_t9_1; A.rho_0 = d_rho_0; A.rho_1 = d_rho_1;
  A.dtwant = d_dtwant; A.ye = d_ye; A.ierr = d_ierr; A.stats = d_stats; A.bd_state = d_bd_state;
  A.counter = (int *)base;
  CK(launch_integrate_net(net, (char *)base + kNoAllocCounterBytes, grid, A, s));
  net->launches++;
  return NUPPN_OK;
}

// ---- phase entry points (host buffers) ----------------------------------------------------------
static nuppn_status run_phase(nuppn_net *net, int nz, int op, const double *X, int ldx, const double *t9,
                              const double *rho, const double *ye, const double *v, const double *dt,
                              const double *jac, const uint8_t *eset, const uint8_t *mask, const double *b,
                              double *out_v, double *out_dxdt, double *out_jac, uint8_t *out_eset, uint8_t *out_mask,
                              double *out_x) {
  nuppn_status st = check_zone_args(net, nz, X ? ldx : net ? net->H.nsp : 0);
  if (st != NUPPN_OK) return st;
  if (nz == 0) return NUPPN_OK;
  CK(cudaSetDevice(net->device));
  const HostNet &H = net->H;
  Stager S;
  size_t oX = X ? S.add((size_t)nz * ldx * 8) : 0, ot9 = t9 ? S.add(nz * 8) : 0, orho = rho ? S.add(nz * 8) : 0;
  size_t oye = ye ? S.add(nz * 8) : 0, ov = v ? S.add((size_t)nz * H.nre * 8) : 0, odt = dt ? S.add(nz * 8) : 0;
  size_t ojac = jac ? S.add((size_t)nz * H.nnzJ * 8) : 0, oes = eset ? S.add((size_t)nz * H.nnzJ) : 0;
  size_t omk = mask ? S.add((size_t)nz * H.nsp) : 0, ob = b ? S.add((size_t)nz * H.nsp * 8) : 0;
  size_t oov = out_v ? S.add((size_t)nz * H.nre * 8) : 0, ood = out_dxdt ? S.add((size_t)nz * H.nsp * 8) : 0;
  size_t ooj = out_jac ? S.add((size_t)nz * H.nnzJ * 8) : 0, ooe = out_eset ? S.add((size_t)nz * H.nnzJ) : 0;
  size_t oom = out_mask ? S.add((size_t)nz * H.nsp) : 0, oox = out_x ? S.add((size_t)nz * H.nsp * 8) : 0;
  CK(net->stage.ensure(S.total));
  char *sb = (char *)net->stage.p;
  auto up = [&](size_t off, const void *src, size_t bytes) -> cudaError_t {
    return src ? cudaMemcpy(sb + off, src, bytes, cudaMemcpyHostToDevice) : cudaSuccess;
  };
  CK(up(oX, X, (size_t)nz * ldx * 8)); CK(up(ot9, t9, nz * 8)); CK(up(orho, rho, nz * 8)); CK(up(oye, ye, nz * 8));
  CK(up(ov, v, (size_t)nz * H.nre * 8)); CK(up(odt, dt, nz * 8)); CK(up(ojac, jac, (size_t)nz * H.nnzJ * 8));
  CK(up(oes, eset, (size_t)nz * H.nnzJ)); CK(up(omk, mask, (size_t)nz * H.nsp)); CK(up(ob, b, (size_t)nz * H.nsp * 8));
  int grid = std::min(nz, phase_slots(net));
  st = ensure_ws(net, grid);
  if (st != NUPPN_OK) return st;
  PhaseArgs A;
  memset(&A, 0, sizeof(A));
  A.nz = nz; A.ldx = ldx; A.op = op;
  A.X = X ? (const double *)(sb + oX) : nullptr; A.t9 = t9 ? (const double *)(sb + ot9) : nullptr;
  A.rho = rho ? (const double *)(sb + orho) : nullptr; A.ye = ye ? (const double *)(sb + oye) : nullptr;
  A.v_in = v ? (const double *)(sb + ov) : nullptr; A.dt = dt ? (const double *)(sb + odt) : nullptr;
  A.jac_in = jac ? (const double *)(sb + ojac) : nullptr; A.eset_in = eset ? (const uint8_t *)(sb + oes) : nullptr;
  A.mask_in = mask ? (const uint8_t *)(sb + omk) : nullptr; A.b = b ? (const double *)(sb + ob) : nullptr;
  A.out_v = out_v ? (double *)(sb + oov) : nullptr; A.out_dxdt = out_dxdt ? (double *)(sb + ood) : nullptr;
  A.out_jac = out_jac ? (double *)(sb + ooj) : nullptr; A.out_eset = out_eset ? (uint8_t *)(sb + ooe) : nullptr;
  A.out_mask = out_mask ? (uint8_t *)(sb + oom) : nullptr; A.out_x = out_x ? (double *)(sb + oox) : nullptr;
  CK(launch_phase(net->D, net->L, (char *)net->ws.p, grid, net->phase_block, net->phase_smem, A, 0));
  net->launches++;
  CK(cudaDeviceSynchronize());
  auto down = [&](void *dst, size_t off, size_t bytes) -> cudaError_t {
    return dst ? cudaMemcpy(dst, sb + off, bytes, cudaMemcpyDeviceToHost) : cudaSuccess;
  };
  CK(down(out_v, oov, (size_t)nz * H.nre * 8)); CK(down(out_dxdt, ood, (size_t)nz * H.nsp * 8));
  CK(down(out_jac, ooj, (size_t)nz * H.nnzJ * 8)); CK(down(out_eset, ooe, (size_t)nz * H.nnzJ));
  CK(down(out_mask, oom, (size_t)nz * H.nsp)); CK(down(out_x, oox, (size_t)nz * H.nsp * 8));
  return NUPPN_OK;
}

nuppn_status nuppn_nse(nuppn_net *net, int32_t nz, const double *t9, const double *rho, const double *ye, double *X,
                       double *mu_p, double *mu_n, int32_t *iters, int32_t *ierr) {
  if (!net) { set_error("null handle"); return NUPPN_ERR_ARG; }
  if (nz < 0) { set_error("nz < 0"); return NUPPN_ERR_ARG; }
  if (!t9 || !rho || !ye || !X || !mu_p || !mu_n || !iters || !ierr) { set_error("null argument"); return NUPPN_ERR_ARG; }
  if (net->H.nse_iprot < 0 || net->H.nse_ini56 < 0) {
    set_error("NSE needs protons and Ni56 among the considered species");
    return NUPPN_ERR_NET;
  }
  if (nz == 0) return NUPPN_OK;
  CK(cudaSetDevice(net->device));
  const int nsp = net->H.nsp;
  Stager S;
  size_t o1 = S.add(nz * 8), o2 = S.add(nz * 8), o3 = S.add(nz * 8), oX = S.add((size_t)nz * nsp * 8);
  size_t op = S.add(nz * 8), on = S.add(nz * 8), oi = S.add(nz * 4), oe = S.add(nz * 4);
  CK(net->stage.ensure(S.total));
  char *sb = (char *)net->stage.p;
  CK(cudaMemcpy(sb + o1, t9, nz * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sb + o2, rho, nz * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sb + o3, ye, nz * 8, cudaMemcpyHostToDevice));
  int grid = std::min(nz, phase_slots(net));
  nuppn_status st = ensure_ws(net, grid);
  if (st != NUPPN_OK) return st;
  PhaseArgs A;
  memset(&A, 0, sizeof(A));
  A.nz = nz; A.ldx = nsp; A.op = 4;
  A.t9 = (const double *)(sb + o1); A.rho = (const double *)(sb + o2); A.ye = (const double *)(sb + o3);
  A.out_x = (double *)(sb + oX); A.out_mu_p = (double *)(sb + op); A.out_mu_n = (double *)(sb + on);
  A.out_iters = (int *)(sb + oi); A.out_ierr = (int *)(sb + oe);
  CK(launch_phase(net->D, net->L, (char *)net->ws.p, grid, net->phase_block, net->phase_smem, A, 0));
  net->launches++;
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(X, sb + oX, (size_t)nz * nsp * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(mu_p, sb + op, nz * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(mu_n, sb + on, nz * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(iters, sb + oi, nz * 4, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(ierr, sb + oe, nz * 4, cudaMemcpyDeviceToHost));
  return NUPPN_OK;
}

nuppn_status nuppn_eval_rates(nuppn_net *net, int32_t nz, const double *t9, const double *rho, const double *ye,
                              const double *X, int32_t ldx, double *v) {
  if (!t9 || !rho || !ye || !X || !v) { set_error("null argument"); return NUPPN_ERR_ARG; }
  return run_phase(net, nz, 0, X, ldx, t9, rho, ye, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, v, nullptr,
                   nullptr, nullptr, nullptr, nullptr);
}

nuppn_status nuppn_dxdt(nuppn_net *net, int32_t nz, const double *v, const double *X, int32_t ldx, double *dxdt) {
  if (!v || !X || !dxdt) { set_error("null argument"); return NUPPN_ERR_ARG; }
  return run_phase(net, nz, 1, X, ldx, nullptr, nullptr, nullptr, v, nullptr, nullptr, nullptr, nullptr, nullptr,
                   nullptr, dxdt, nullptr, nullptr, nullptr, nullptr);
}

nuppn_status nuppn_jacobian(nuppn_net *net, int32_t nz, const double *v, const double *X, int32_t ldx, const double *dt,
                            double *jac, uint8_t *entry_set, uint8_t *mask) {
  if (!v || !X || !dt || !jac || !entry_set || !mask) { set_error("null argument"); return NUPPN_ERR_ARG; }
  return run_phase(net, nz, 2, X, ldx, nullptr, nullptr, nullptr, v, dt, nullptr, nullptr, nullptr, nullptr, nullptr,
                   nullptr, jac, entry_set, mask, nullptr);
}

nuppn_status nuppn_solve_reduced(nuppn_net *net, int32_t nz, const double *jac, const uint8_t *entry_set,
                                 const uint8_t *mask, const double *dt, const double *b, double *x) {
  if (!jac || !entry_set || !mask || !dt || !b || !x) { set_error("null argument"); return NUPPN_ERR_ARG; }
  return run_phase(net, nz, 3, nullptr, net ? net->H.nsp : 0, nullptr, nullptr, nullptr, nullptr, dt, jac, entry_set,
                   mask, b, nullptr, nullptr, nullptr, nullptr, nullptr, x);
}

// ---- integration -------------------------------------------------------------------------------
nuppn_status nuppn_integrate_device(nuppn_net *net, int32_t nz, double *d_X, int32_t ldx, const double *d_t9_0,
                                    const double *d_t9_1, const double *d_rho_0, const double *d_rho_1, double *d_ye,
                                    const double *d_dtwant, int32_t *d_ierr, nuppn_zone_stats *d_stats,
                                    int32_t *d_bd_state, void *stream) {
  nuppn_status st = check_zone_args(net, nz, ldx);
  if (st != NUPPN_OK) return st;
  if (nz == 0) return NUPPN_OK;
  if (!d_X || !d_t9_0 || !d_t9_1 || !d_rho_0 || !d_rho_1 || !d_ye || !d_dtwant || !d_ierr) {
    set_error("null device argument");
    return NUPPN_ERR_ARG;
  }
  CK(cudaSetDevice(net->device));
  const int grid = integrate_grid(net, nz, resident_slots(net));
  st = ensure_ws(net, grid * zones_per_cta(net));
  if (st != NUPPN_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  CK(net->order.ensure((size_t)nz * 4));
  CK(cudaMemsetAsync(net->counter.p, 0, sizeof(int), s));
  CK(launch_zone_order(d_t9_0, d_t9_1, 1, nz, (int *)net->order.p, s));
  IntegrateArgs A = {};
  A.nz = nz; A.ldx = ldx; A.X = d_X; A.t9_0 = d_t9_0; A.t9_1 = d_t9_1; A.rho_0 = d_rho_0; A.rho_1 = d_rho_1;
  A.dtwant = d_dtwant; A.ye = d_ye; A.ierr = d_ierr; A.stats = d_stats; A.bd_state = d_bd_state;
  A.counter = (int *)net->counter.p;
  A.order = (const int *)net->order.p;
  CK(launch_integrate_net(net, (char *)net->ws.p, grid, A, s));
  net->launches += 2;  // k_zone_order, k_integrate
  return NUPPN_OK;
}

nuppn_status nuppn_integrate(nuppn_net *net, int32_t nz, double *X, int32_t ldx, const double *t9_0,
                             const double *t9_1, const double *rho_0, const double *rho_1, double *ye,
                             const double *dtwant, int32_t *ierr, nuppn_zone_stats *stats, int32_t *bd_state) {
  nuppn_status st = check_zone_args(net, nz, ldx);
  if (st != NUPPN_OK) return st;
  if (nz == 0) return NUPPN_OK;
  if (!X || !t9_0 || !t9_1 || !rho_0 || !rho_1 || !ye || !dtwant || !ierr) {
    set_error("null argument");
    return NUPPN_ERR_ARG;
  }
  CK(cudaSetDevice(net->device));
  Stager S;
  size_t oX = S.add((size_t)nz * ldx * 8), o1 = S.add(nz * 8), o2 = S.add(nz * 8), o3 = S.add(nz * 8);
  size_t o4 = S.add(nz * 8), o5 = S.add(nz * 8), o6 = S.add(nz * 8), oi = S.add(nz * 4);
  size_t os = S.add((size_t)nz * sizeof(nuppn_zone_stats)), ob = S.add(nz * 4);
  CK(net->stage.ensure(S.total));
  char *sb = (char *)net->stage.p;
  CK(cudaMemcpy(sb + oX, X, (size_t)nz * ldx * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sb + o1, t9_0, nz * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sb + o2, t9_1, nz * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sb + o3, rho_0, nz * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sb + o4, rho_1, nz * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sb + o5, ye, nz * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sb + o6, dtwant, nz * 8, cudaMemcpyHostToDevice));
  if (bd_state) CK(cudaMemcpy(sb + ob, bd_state, nz * 4, cudaMemcpyHostToDevice));
  else CK(cudaMemset(sb + ob, 0, nz * 4));
  st = nuppn_integrate_device(net, nz, (double *)(sb + oX), ldx, (double *)(sb + o1), (double *)(sb + o2),
                              (double *)(sb + o3), (double *)(sb + o4), (double *)(sb + o5), (double *)(sb + o6),
                              (int *)(sb + oi), (nuppn_zone_stats *)(sb + os), (int *)(sb + ob), nullptr);
  if (st != NUPPN_OK) return st;
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(X, sb + oX, (size_t)nz * ldx * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(ye, sb + o5, nz * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(ierr, sb + oi, nz * 4, cudaMemcpyDeviceToHost));
  if (stats) CK(cudaMemcpy(stats, sb + os, (size_t)nz * sizeof(nuppn_zone_stats), cudaMemcpyDeviceToHost));
  if (bd_state) CK(cudaMemcpy(bd_state, sb + ob, nz * 4, cudaMemcpyDeviceToHost));
  return NUPPN_OK;
}

// ---- autotuning of the kernel shape -------------------------------------------------------------
nuppn_status nuppn_autotune(nuppn_net *net, int32_t nz, const double *X, int32_t ldx, const double *t9_0,
                            const double *t9_1, const double *rho_0, const double *rho_1, const double *ye,
                            const double *dtwant, int32_t sample, nuppn_tune_result *report, int32_t ncand,
                            int32_t *nreport) {
  nuppn_status st = check_zone_args(net, nz, ldx);
  if (st != NUPPN_OK) return st;
  if (!X || !t9_0 || !t9_1 || !rho_0 || !rho_1 || !ye || !dtwant || sample < 0 || (report && ncand < 0)) {
    set_error("null or negative argument");
    return NUPPN_ERR_ARG;
  }
  if (nreport) *nreport = 0;
  const int n = sample > 0 ? std::min(sample, nz) : nz;
  if (n == 0) return NUPPN_OK;
  CK(cudaSetDevice(net->device));
  // inputs (kept) and one call's working copies
  Stager S;
  const size_t xb = (size_t)n * ldx * 8, vb = (size_t)n * 8;
  size_t oX0 = S.add(xb), oX = S.add(xb), o1 = S.add(vb), o2 = S.add(vb), o3 = S.add(vb), o4 = S.add(vb);
  size_t oy0 = S.add(vb), oy = S.add(vb), odt = S.add(vb), oi = S.add((size_t)n * 4), ob = S.add((size_t)n * 4);
  size_t os = S.add((size_t)n * sizeof(nuppn_zone_stats));
  DevBuf buf;
  struct Release {
    DevBuf &b;
    ~Release() { b.release(); }
  } release_buf{buf};
  CK(buf.ensure(S.total));
  char *b = (char *)buf.p;
  CK(cudaMemcpy(b + oX0, X, xb, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b + o1, t9_0, vb, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b + o2, t9_1, vb, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b + o3, rho_0, vb, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b + o4, rho_1, vb, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b + oy0, ye, vb, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b + odt, dtwant, vb, cudaMemcpyHostToDevice));
  // candidates: one zone per CTA of 256 threads and 72 KB (3 per SM), of 128 threads and 36 KB (6 per
  // SM) and of 64 threads and 24 KB (9 per SM): fewer threads for the wide phases, more zones whose
  // one-warp dependency chains share the SM; one zone per warp with 8 zones per CTA, 4 per CTA at the
  // same share of shared memory (two CTAs per SM), and 4 per CTA with twice the share (64-row tiles
  // of the hottest zones fit in shared memory, one CTA per SM)
  struct Cand { int tpz, zpc, smem; };
  const Cand cands[] = {{0, 0, 0}, {128, 0, 36864}, {64, 0, 24576}, {32, 8, 0}, {32, 4, 27648}, {32, 4, 0}};
  const int nc = (int)(sizeof(cands) / sizeof(cands[0]));
  const nuppn_knobs base = net->H.kn;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  std::vector<nuppn_zone_stats> stv(n);
  std::vector<double> rate(nc, -1.0), ms(nc, 0.0);
  std::vector<int> zsm(nc, 0);
  nuppn_status out = NUPPN_OK;
  for (int c = 0; c < nc && out == NUPPN_OK; ++c) {
    nuppn_knobs kn = base;
    kn.threads_per_zone = cands[c].tpz;
    kn.zones_per_cta = cands[c].zpc;
    kn.zone_smem = cands[c].smem;
    if (apply_shape(net, kn) != NUPPN_OK) continue;  // a shape this device cannot run is skipped
    zsm[c] = resident_slots(net) / std::max(net->nsm, 1);
    for (int rep = 0; rep < 2 && out == NUPPN_OK; ++rep) {  // the first call grows the workspace
      cudaError_t e = cudaMemcpyAsync(b + oX, b + oX0, xb, cudaMemcpyDeviceToDevice, 0);
      if (e == cudaSuccess) e = cudaMemcpyAsync(b + oy, b + oy0, vb, cudaMemcpyDeviceToDevice, 0);
      if (e == cudaSuccess) e = cudaMemsetAsync(b + ob, 0, (size_t)n * 4, 0);
      if (e == cudaSuccess) e = cudaEventRecord(e0, 0);
      if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); out = NUPPN_ERR_CUDA; break; }
      out = nuppn_integrate_device(net, n, (double *)(b + oX), ldx, (double *)(b + o1), (double *)(b + o2),
                                   (double *)(b + o3), (double *)(b + o4), (double *)(b + oy), (double *)(b + odt),
                                   (int *)(b + oi), (nuppn_zone_stats *)(b + os), (int *)(b + ob), nullptr);
      if (out != NUPPN_OK) break;
      e = cudaEventRecord(e1, 0);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float t = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
      if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); out = NUPPN_ERR_CUDA; break; }
      ms[c] = t;
    }
    if (out != NUPPN_OK) break;
    if (cudaMemcpy(stv.data(), b + os, (size_t)n * sizeof(nuppn_zone_stats), cudaMemcpyDeviceToHost) != cudaSuccess) {
      set_error("autotune: stats copy");
      out = NUPPN_ERR_CUDA;
      break;
    }
    int64_t steps = 0;
    for (const nuppn_zone_stats &z : stv) steps += z.nsucc;
    rate[c] = ms[c] > 0.0 ? (double)steps / (ms[c] * 1e-3) : 0.0;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int best = -1;
  for (int c = 0; c < nc; ++c)
    if (rate[c] > 0.0 && (best < 0 || rate[c] > rate[best])) best = c;
  nuppn_knobs kn = base;
  if (out == NUPPN_OK && best >= 0) {
    kn.threads_per_zone = cands[best].tpz;
    kn.zones_per_cta = cands[best].zpc;
    kn.zone_smem = cands[best].smem;
  }
  const nuppn_status st2 = apply_shape(net, kn);  // the winner, or the shape the handle had
  net->H.kn = kn;
  net->D.kn = kn;
  if (out == NUPPN_OK && st2 != NUPPN_OK) out = st2;
  if (report) {
    int k = 0;
    for (int c = 0; c < nc && k < ncand; ++c, ++k) {
      nuppn_tune_result &r = report[k];
      memset(&r, 0, sizeof(r));
      r.threads_per_zone = cands[c].tpz;
      r.zones_per_cta = cands[c].zpc;
      r.zone_smem = cands[c].smem;
      r.zones_per_sm = zsm[c];
      r.ms = ms[c];
      r.zone_steps_per_s = rate[c];
      r.chosen = c == best;
    }
    if (nreport) *nreport = k;
  }
  return out;
}

// ---- several networks in one launch ------------------------------------------------------------
constexpr int kMaxMultiNets = 16;

nuppn_status nuppn_integrate_multi_device(nuppn_net *const *nets, int32_t nnets, int32_t nz, const int32_t *d_net_of,
                                          double *d_X, int32_t ldx, const double *d_t9_0, const double *d_t9_1,
                                          const double *d_rho_0, const double *d_rho_1, double *d_ye,
                                          const double *d_dtwant, int32_t *d_ierr, nuppn_zone_stats *d_stats,
                                          int32_t *d_bd_state, void *stream) {
  if (!nets || nnets < 1 || nnets > kMaxMultiNets) {
    set_error("nnets must be 1.." + std::to_string(kMaxMultiNets));
    return NUPPN_ERR_ARG;
  }
  nuppn_net *net = nets[0];
  size_t slab = 0;
  int nsp_max = 0;
  for (int i = 0; i < nnets; ++i) {
    if (!nets[i]) { set_error("null network handle"); return NUPPN_ERR_ARG; }
    if (nets[i]->device != net->device) { set_error("the networks are on different devices"); return NUPPN_ERR_ARG; }
    slab = std::max(slab, nets[i]->L.bytes);
    nsp_max = std::max(nsp_max, nets[i]->H.nsp);
  }
  if (nz < 0) { set_error("nz < 0"); return NUPPN_ERR_ARG; }
  if (ldx < nsp_max) { set_error("ldx < the largest network's nsp"); return NUPPN_ERR_ARG; }
  if (nz == 0) return NUPPN_OK;
  if (!d_net_of || !d_X || !d_t9_0 || !d_t9_1 || !d_rho_0 || !d_rho_1 || !d_ye || !d_dtwant || !d_ierr) {
    set_error("null device argument");
    return NUPPN_ERR_ARG;
  }
  CK(cudaSetDevice(net->device));
  cudaStream_t s = (cudaStream_t)stream;
  // one zone per CTA of 256 threads, 72 KB of shared memory each (3 CTAs per SM)
  const int act_smem = 72 * 1024;
  CK(cta::configure_kernels(std::max(act_smem, net->phase_smem)));
  int per = 0;
  if (cta::occupancy_integrate_multi(act_smem, &per) != cudaSuccess || per <= 0) per = 1;
  const int grid = std::min(nz, per * net->nsm);
  CK(net->ws.ensure((size_t)grid * slab));
  net->ws_slots = (int)(net->ws.n / std::max<size_t>(net->L.bytes, 1));
  const size_t desc = a16(sizeof(DevNet)) * kMaxMultiNets, lay = a16(sizeof(WsLayout)) * kMaxMultiNets;
  CK(net->multi.ensure(desc + lay));
  if (!net->multi_host) CK(cudaHostAlloc((void **)&net->multi_host, desc + lay, cudaHostAllocPortable));
  CK(cudaStreamSynchronize(s));  // the staging buffer may still feed the previous call's copy
  DevNet *hn = (DevNet *)net->multi_host;
  WsLayout *hl = (WsLayout *)(net->multi_host + desc);
  for (int i = 0; i < nnets; ++i) { hn[i] = nets[i]->D; hl[i] = nets[i]->L; }
  CK(cudaMemcpyAsync(net->multi.p, net->multi_host, desc + lay, cudaMemcpyHostToDevice, s));
  CK(net->order.ensure((size_t)nz * 4));
  CK(cudaMemsetAsync(net->counter.p, 0, sizeof(int), s));
  CK(launch_zone_order(d_t9_0, d_t9_1, 1, nz, (int *)net->order.p, s));
  IntegrateArgs A = {};
  A.nz = nz; A.ldx = ldx; A.X = d_X; A.t9_0 = d_t9_0; A.t9_1 = d_t9_1; A.rho_0 = d_rho_0; A.rho_1 = d_rho_1;
  A.dtwant = d_dtwant; A.ye = d_ye; A.ierr = d_ierr; A.stats = d_stats; A.bd_state = d_bd_state;
  A.counter = (int *)net->counter.p;
  A.order = (const int *)net->order.p;
  A.nets = (const DevNet *)net->multi.p;
  A.lays = (const WsLayout *)((char *)net->multi.p + desc);
  A.net_of = d_net_of;
  A.nnets = nnets;
  A.slab = slab;
  CK(cta::launch_integrate_multi(A, (char *)net->ws.p, grid, act_smem, s));
  net->launches += 2;  // k_zone_order, k_integrate_multi
  return NUPPN_OK;
}

nuppn_status nuppn_integrate_multi(nuppn_net *const *nets, int32_t nnets, int32_t nz, const int32_t *net_of, double *X,
                                   int32_t ldx, const double *t9_0, const double *t9_1, const double *rho_0,
                                   const double *rho_1, double *ye, const double *dtwant, int32_t *ierr,
                                   nuppn_zone_stats *stats, int32_t *bd_state) {
  if (!nets || nnets < 1 || nnets > kMaxMultiNets || !nets[0]) { set_error("bad network list"); return NUPPN_ERR_ARG; }
  if (nz < 0) { set_error("nz < 0"); return NUPPN_ERR_ARG; }
  if (nz == 0) return NUPPN_OK;
  if (!net_of || !X || !t9_0 || !t9_1 || !rho_0 || !rho_1 || !ye || !dtwant || !ierr) {
    set_error("null argument");
    return NUPPN_ERR_ARG;
  }
  for (int z = 0; z < nz; ++z)
    if (net_of[z] < 0 || net_of[z] >= nnets) { set_error("net_of[" + std::to_string(z) + "] out of range"); return NUPPN_ERR_ARG; }
  nuppn_net *net = nets[0];
  CK(cudaSetDevice(net->device));
  Stager S;
  size_t oX = S.add((size_t)nz * ldx * 8), o1 = S.add(nz * 8), o2 = S.add(nz * 8), o3 = S.add(nz * 8);
  size_t o4 = S.add(nz * 8), o5 = S.add(nz * 8), o6 = S.add(nz * 8), oi = S.add(nz * 4), on = S.add(nz * 4);
  size_t os = S.add((size_t)nz * sizeof(nuppn_zone_stats)), ob = S.add(nz * 4);
  CK(net->stage.ensure(S.total));
  char *sb = (char *)net->stage.p;
  CK(cudaMemcpy(sb + oX, X, (size_t)nz * ldx * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sb + o1, t9_0, nz * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sb + o2, t9_1, nz * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sb + o3, rho_0, nz * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sb + o4, rho_1, nz * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sb + o5, ye, nz * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sb + o6, dtwant, nz * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sb + on, net_of, nz * 4, cudaMemcpyHostToDevice));
  if (bd_state) CK(cudaMemcpy(sb + ob, bd_state, nz * 4, cudaMemcpyHostToDevice));
  else CK(cudaMemset(sb + ob, 0, nz * 4));
  nuppn_status st = nuppn_integrate_multi_device(nets, nnets, nz, (const int *)(sb + on), (double *)(sb + oX), ldx,
                                                 (double *)(sb + o1), (double *)(sb + o2), (double *)(sb + o3),
                                                 (double *)(sb + o4), (double *)(sb + o5), (double *)(sb + o6),
                                                 (int *)(sb + oi), (nuppn_zone_stats *)(sb + os), (int *)(sb + ob),
                                                 nullptr);
  if (st != NUPPN_OK) return st;
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(X, sb + oX, (size_t)nz * ldx * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(ye, sb + o5, nz * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(ierr, sb + oi, nz * 4, cudaMemcpyDeviceToHost));
  if (stats) CK(cudaMemcpy(stats, sb + os, (size_t)nz * sizeof(nuppn_zone_stats), cudaMemcpyDeviceToHost));
  if (bd_state) CK(cudaMemcpy(bd_state, sb + ob, nz * 4, cudaMemcpyDeviceToHost));
  return NUPPN_OK;
}

nuppn_status nuppn_integrate_trajectories_device(nuppn_net *net, int32_t nz, int32_t npts, double *d_X, int32_t ldx,
                                                const double *d_time, const double *d_t9, const double *d_rho,
                                                double *d_ye, int32_t *d_ierr, int32_t *d_fail,
                                                nuppn_zone_stats *d_stats, int32_t *d_bd_state, void *stream) {
  nuppn_status st = check_zone_args(net, nz, ldx);
  if (st != NUPPN_OK) return st;
  if (npts < 2) { set_error("npts < 2"); return NUPPN_ERR_ARG; }
  if (nz == 0) return NUPPN_OK;
  if (!d_X || !d_time || !d_t9 || !d_rho || !d_ye || !d_ierr) {
    set_error("null device argument");
    return NUPPN_ERR_ARG;
  }
  CK(cudaSetDevice(net->device));
  const int grid = integrate_grid(net, nz, resident_slots(net));
  st = ensure_ws(net, grid * zones_per_cta(net));
  if (st != NUPPN_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  CK(net->order.ensure((size_t)nz * 4));
  CK(cudaMemsetAsync(net->counter.p, 0, sizeof(int), s));
  CK(launch_zone_order(d_t9, nullptr, npts, nz, (int *)net->order.p, s));
  IntegrateArgs A = {};
  A.nz = nz; A.ldx = ldx; A.X = d_X; A.ye = d_ye; A.ierr = d_ierr; A.stats = d_stats; A.bd_state = d_bd_state;
  A.counter = (int *)net->counter.p;
  A.order = (const int *)net->order.p;
  A.npts = npts; A.tr_time = d_time; A.tr_t9 = d_t9; A.tr_rho = d_rho; A.tr_fail = d_fail;
  CK(launch_integrate_net(net, (char *)net->ws.p, grid, A, s));
  net->launches += 2;  // k_zone_order, k_integrate
  return NUPPN_OK;
}

nuppn_status nuppn_integrate_trajectories(nuppn_net *net, int32_t nz, int32_t npts, double *X, int32_t ldx,
                                         const double *time, const double *t9, const double *rho, double *ye,
                                         int32_t *ierr, int32_t *fail, nuppn_zone_stats *stats) {
  nuppn_status st = check_zone_args(net, nz, ldx);
  if (st != NUPPN_OK) return st;
  if (npts < 2) { set_error("npts < 2"); return NUPPN_ERR_ARG; }
  if (nz == 0) return NUPPN_OK;
  if (!X || !time || !t9 || !rho || !ye || !ierr) {
    set_error("null argument");
    return NUPPN_ERR_ARG;
  }
  CK(cudaSetDevice(net->device));
  const size_t np = (size_t)nz * npts * 8;
  Stager S;
  size_t oX = S.add((size_t)nz * ldx * 8), ot = S.add(np), o9 = S.add(np), orh = S.add(np), oy = S.add(nz * 8);
  size_t oi = S.add(nz * 4), of = S.add(nz * 4), os = S.add((size_t)nz * sizeof(nuppn_zone_stats)), ob = S.add(nz * 4);
  CK(net->stage.ensure(S.total));
  char *sb = (char *)net->stage.p;
  CK(cudaMemcpy(sb + oX, X, (size_t)nz * ldx * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sb + ot, time, np, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sb + o9, t9, np, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sb + orh, rho, np, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sb + oy, ye, nz * 8, cudaMemcpyHostToDevice));
  CK(cudaMemset(sb + ob, 0, nz * 4));
  st = nuppn_integrate_trajectories_device(net, nz, npts, (double *)(sb + oX), ldx, (double *)(sb + ot),
                                           (double *)(sb + o9), (double *)(sb + orh), (double *)(sb + oy),
                                           (int *)(sb + oi), (int *)(sb + of), (nuppn_zone_stats *)(sb + os),
                                           (int *)(sb + ob), nullptr);
  if (st != NUPPN_OK) return st;
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(X, sb + oX, (size_t)nz * ldx * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(ye, sb + oy, nz * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(ierr, sb + oi, nz * 4, cudaMemcpyDeviceToHost));
  if (fail) CK(cudaMemcpy(fail, sb + of, nz * 4, cudaMemcpyDeviceToHost));
  if (stats) CK(cudaMemcpy(stats, sb + os, (size_t)nz * sizeof(nuppn_zone_stats), cudaMemcpyDeviceToHost));
  return NUPPN_OK;
}

}  // extern "C"

// ---- serving: a device-resident request loop -----------------------------------------------------
// The server keeps one persistent launch of the integration kernel (trajectory instantiation, queue
// mode) on its own stream. Its groups claim published requests one at a time from a queue in device
// memory and write each result to host-mapped memory as soon as that zone is done, so requests that
// arrive while others are on the GPU start as soon as a group is free, with no batch to wait for. A
// host worker thread publishes submitted requests (asynchronous copies of their inputs, then of the
// published count, on a second stream), collects finished ones, and relaunches the loop when it has
// left after staying idle. Request seq uses queue slot seq % cap; a slot is reused only once its
// previous request has finished.
namespace {

constexpr int kServeMaxPoints = 512;   // points of a trajectory request
constexpr int kServeIdlePolls = 4000;  // empty polls (sleeps growing to 8 us) before a group leaves

struct ServeReq {
  int64_t id = 0;
  int kind = 0;  // 0: one zone, 1: one trajectory
  int npts = 0;
  std::vector<double> X, time, t9, rho;
  double t9_0 = 0, t9_1 = 0, rho_0 = 0, rho_1 = 0, ye = 0, dtwant = 0;
  int bd = 0, ierr = 0, fail = -1;
  nuppn_zone_stats st{};
  long long seq = -1;
  int status = 0;  // 0 pending or on the GPU, 1 done, 2 failed
  std::string err;
};

}  // namespace

struct nuppn_server {
  nuppn_net *net = nullptr;
  int slots = 0;      // zones integrated at once (workspace slabs)
  int grid = 0;       // CTAs of the loop
  int cap = 0;        // queue slots
  DevBuf ws, dq;      // workspace slabs; device queue
  char *hmap = nullptr;    // host-mapped results: RingOut[cap], x_out[cap][nsp]
  char *hstage = nullptr;  // pinned staging: per slot RingIn + X + grid, then published counts [cap], stop
  size_t stage_slot = 0;
  RingIn *d_in = nullptr;
  double *d_xin = nullptr, *d_grid = nullptr;
  long long *d_pub = nullptr;
  unsigned long long *d_claimed = nullptr;
  int *d_stop = nullptr, *h_stop = nullptr;
  RingOut *h_out = nullptr, *d_out = nullptr;
  double *h_xout = nullptr, *d_xout = nullptr;
  cudaStream_t sk = nullptr, sc = nullptr;
  cudaEvent_t kdone = nullptr;
  bool running = false;
  long long published = 0, claimed = 0;
  std::vector<ServeReq *> in_slot;  // request in each queue slot, or null
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<ServeReq *> pending;
  std::unordered_map<int64_t, ServeReq *> reqs;
  int64_t next_id = 1;
  std::atomic<bool> stop{false};
  std::atomic<int64_t> launches{0}, completed{0};
  std::atomic<int> in_flight{0}, queued{0};
  int64_t device_bytes = 0;
  std::string fatal;  // a failed CUDA call of the worker: every later request fails with it
};

namespace {

// Free everything the server holds (the loop has left).
void serve_free(nuppn_server *S) {
  if (S->sk) cudaStreamSynchronize(S->sk);
  if (S->sc) cudaStreamSynchronize(S->sc);
  S->ws.release();
  S->dq.release();
  if (S->hmap) cudaFreeHost(S->hmap);
  if (S->hstage) cudaFreeHost(S->hstage);
  if (S->kdone) cudaEventDestroy(S->kdone);
  if (S->sk) cudaStreamDestroy(S->sk);
  if (S->sc) cudaStreamDestroy(S->sc);
  S->hmap = S->hstage = nullptr;
  S->kdone = nullptr;
  S->sk = S->sc = nullptr;
}

cudaError_t serve_launch(nuppn_server *S) {
  IntegrateArgs A = {};
  ServeQueue &Q = A.queue;
  Q.in = S->d_in; Q.out = S->d_out; Q.x_in = S->d_xin; Q.x_out = S->d_xout; Q.grid = S->d_grid;
  Q.published = S->d_pub; Q.claimed = S->d_claimed; Q.stop = S->d_stop;
  Q.nslots = S->cap; Q.npts_max = kServeMaxPoints; Q.idle_polls = kServeIdlePolls;
  A.npts = 1;  // selects the trajectory instantiation, which runs the queue loop
  cudaError_t e = launch_integrate_net(S->net, (char *)S->ws.p, S->grid, A, S->sk);
  if (e == cudaSuccess) e = cudaEventRecord(S->kdone, S->sk);
  if (e == cudaSuccess) {
    S->running = true;
    S->launches++;
  }
  return e;
}

// Publish request r in queue slot r->seq % cap: its inputs, then the new published count.
cudaError_t serve_publish(nuppn_server *S, ServeReq *r) {
  const int nsp = S->net->H.nsp, slot = (int)(r->seq % S->cap);
  char *st = S->hstage + (size_t)slot * S->stage_slot;
  RingIn *in = (RingIn *)st;
  double *x = (double *)(st + a16(sizeof(RingIn)));
  double *g = x + nsp;
  memset(in, 0, sizeof(*in));
  in->seq = r->seq; in->kind = r->kind; in->npts = r->npts; in->bd = r->bd;
  in->t9_0 = r->t9_0; in->t9_1 = r->t9_1; in->rho_0 = r->rho_0; in->rho_1 = r->rho_1; in->ye = r->ye;
  in->dtwant = r->dtwant;
  memcpy(x, r->X.data(), (size_t)nsp * 8);
  cudaError_t e = cudaMemcpyAsync(S->d_xin + (size_t)slot * nsp, x, (size_t)nsp * 8, cudaMemcpyHostToDevice, S->sc);
  if (e == cudaSuccess && r->kind == 1) {
    memcpy(g, r->time.data(), (size_t)r->npts * 8);
    memcpy(g + kServeMaxPoints, r->t9.data(), (size_t)r->npts * 8);
    memcpy(g + 2 * kServeMaxPoints, r->rho.data(), (size_t)r->npts * 8);
    e = cudaMemcpyAsync(S->d_grid + (size_t)slot * 3 * kServeMaxPoints, g, (size_t)3 * kServeMaxPoints * 8,
                        cudaMemcpyHostToDevice, S->sc);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(S->d_in + slot, in, sizeof(RingIn), cudaMemcpyHostToDevice, S->sc);
  long long *pub = (long long *)(S->hstage + (size_t)S->cap * S->stage_slot) + slot;
  *pub = r->seq + 1;
  if (e == cudaSuccess) e = cudaMemcpyAsync(S->d_pub, pub, sizeof(long long), cudaMemcpyHostToDevice, S->sc);
  return e;
}

void serve_fail_all(nuppn_server *S, const std::string &why) {
  std::lock_guard<std::mutex> lk(S->mu);
  S->fatal = why;
  for (ServeReq *r : S->pending) { r->status = 2; r->err = why; S->completed++; S->queued--; }
  S->pending.clear();
  for (ServeReq *&r : S->in_slot)
    if (r) { r->status = 2; r->err = why; S->completed++; S->in_flight--; r = nullptr; }
}

void serve_loop(nuppn_server *S) {
  cudaSetDevice(S->net->device);
  const int nsp = S->net->H.nsp;
  for (;;) {
    bool did = false;
    // finished requests: RingOut::done = seq + 1 (written after the results)
    for (int slot = 0; slot < S->cap; ++slot) {
      ServeReq *r = S->in_slot[slot];
      if (!r) continue;
      const volatile long long *done = &S->h_out[slot].done;
      if (*done != r->seq + 1) continue;
      std::atomic_thread_fence(std::memory_order_acquire);
      const RingOut &o = S->h_out[slot];
      std::lock_guard<std::mutex> lk(S->mu);
      memcpy(r->X.data(), S->h_xout + (size_t)slot * nsp, (size_t)nsp * 8);
      r->ye = o.ye; r->bd = o.bd; r->ierr = o.ierr; r->st = o.st; r->fail = r->kind == 1 ? o.fail : -1;
      r->status = 1;
      S->in_slot[slot] = nullptr;
      S->in_flight--;
      S->completed++;
      did = true;
    }
    // publish pending requests in order while their queue slot is free
    if (!S->stop.load() && S->fatal.empty()) {
      for (;;) {
        ServeReq *r = nullptr;
        {
          std::lock_guard<std::mutex> lk(S->mu);
          if (S->pending.empty() || S->in_slot[(int)(S->published % S->cap)]) break;
          r = S->pending.front();
          S->pending.pop_front();
          r->seq = S->published++;
          S->in_slot[(int)(r->seq % S->cap)] = r;
          S->queued--;
          S->in_flight++;
        }
        const cudaError_t e = serve_publish(S, r);
        if (e != cudaSuccess) {
          serve_fail_all(S, std::string("serve: ") + cudaGetErrorString(e));
          break;
        }
        did = true;
      }
    }
    // the loop on the device: note when it has left, relaunch it while published requests wait
    if (S->running) {
      const cudaError_t q = cudaEventQuery(S->kdone);
      if (q == cudaSuccess) {
        S->running = false;
        unsigned long long c = 0;
        if (cudaMemcpy(&c, S->d_claimed, sizeof(c), cudaMemcpyDeviceToHost) == cudaSuccess) S->claimed = (long long)c;
      } else if (q != cudaErrorNotReady) {
        S->running = false;
        serve_fail_all(S, std::string("serve loop: ") + cudaGetErrorString(q));
      }
    }
    if (!S->running && S->published > S->claimed && S->fatal.empty()) {  // published requests always run
      const cudaError_t e = serve_launch(S);
      if (e != cudaSuccess) serve_fail_all(S, std::string("serve launch: ") + cudaGetErrorString(e));
      did = true;
    }
    if (S->stop.load()) {
      bool busy = false;
      for (ServeReq *r : S->in_slot) busy |= r != nullptr;
      if (!busy || !S->fatal.empty()) break;  // what was on the GPU has finished; pending requests are dropped
    }
    if (!did) {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv.wait_for(lk, std::chrono::microseconds(50));
    }
  }
  // ask the loop to leave and wait for it
  *S->h_stop = 1;
  cudaMemcpyAsync(S->d_stop, S->h_stop, sizeof(int), cudaMemcpyHostToDevice, S->sc);
  cudaStreamSynchronize(S->sc);
  cudaStreamSynchronize(S->sk);
}

}  // namespace

extern "C" {

nuppn_status nuppn_serve_open(nuppn_net *net, int32_t slots, int32_t queue, nuppn_server **out) {
  if (!net || !out) { set_error("null argument"); return NUPPN_ERR_ARG; }
  if (slots < 0 || queue < 0) { set_error("slots and queue must be >= 0"); return NUPPN_ERR_ARG; }
  *out = nullptr;
  CK(cudaSetDevice(net->device));
  size_t free_b = 0, total_b = 0;
  CK(cudaMemGetInfo(&free_b, &total_b));
  nuppn_server *S = new (std::nothrow) nuppn_server();
  if (!S) return NUPPN_ERR_NOMEM;
  S->net = net;
  // zones in flight: whole CTAs of the kernel shape, at most the GPU's resident ones and the slabs
  // that fit in half of the free device memory (admission by free HBM)
  const int zpc = zones_per_cta(net), resident = resident_slots(net);
  const int by_mem = (int)std::min<size_t>((size_t)resident, (free_b / 2) / std::max<size_t>(net->L.bytes, 1));
  int want = slots > 0 ? std::min<int>(slots, resident) : resident;
  want = std::min(want, by_mem);
  S->grid = want / zpc;
  S->slots = S->grid * zpc;
  if (S->grid < 1) {
    delete S;
    set_error("nuppn_serve_open: not even one CTA of workspace slabs (" + std::to_string((size_t)zpc * net->L.bytes) +
              " bytes) fits in half of the " + std::to_string(free_b) + " bytes free, or slots < zones per CTA");
    return NUPPN_ERR_NOMEM;
  }
  S->cap = queue > 0 ? std::max<int>(queue, S->slots) : 4 * S->slots;
  const int nsp = net->H.nsp, cap = S->cap;
  // device queue: RingIn[cap], x_in[cap][nsp], grid[cap][3][max points], published, claimed, stop
  const size_t o_in = 0, o_x = align256((size_t)cap * sizeof(RingIn)), o_g = o_x + align256((size_t)cap * nsp * 8);
  const size_t o_pub = o_g + align256((size_t)cap * 3 * kServeMaxPoints * 8), o_cl = o_pub + 256, o_st = o_cl + 256;
  const size_t dq_bytes = o_st + 256;
  const size_t map_bytes = align256((size_t)cap * sizeof(RingOut)) + (size_t)cap * nsp * 8;
  S->stage_slot = a16(sizeof(RingIn)) + (size_t)nsp * 8 + (size_t)3 * kServeMaxPoints * 8;
  const size_t stage_bytes = (size_t)cap * S->stage_slot + (size_t)cap * sizeof(long long) + 64;
  cudaError_t e = cudaStreamCreateWithFlags(&S->sk, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->sc, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S->kdone, cudaEventDisableTiming);
  if (e == cudaSuccess) e = S->ws.ensure((size_t)S->slots * net->L.bytes);
  if (e == cudaSuccess) e = S->dq.ensure(dq_bytes);
  if (e == cudaSuccess) e = cudaHostAlloc((void **)&S->hmap, map_bytes, cudaHostAllocMapped | cudaHostAllocPortable);
  if (e == cudaSuccess) e = cudaHostAlloc((void **)&S->hstage, stage_bytes, cudaHostAllocPortable);
  if (e == cudaSuccess) e = cudaMemset(S->dq.p, 0, dq_bytes);
  if (e == cudaSuccess) {
    memset(S->hmap, 0, map_bytes);
    memset(S->hstage, 0, stage_bytes);
    char *dq = (char *)S->dq.p;
    S->d_in = (RingIn *)(dq + o_in);
    S->d_xin = (double *)(dq + o_x);
    S->d_grid = (double *)(dq + o_g);
    S->d_pub = (long long *)(dq + o_pub);
    S->d_claimed = (unsigned long long *)(dq + o_cl);
    S->d_stop = (int *)(dq + o_st);
    S->h_out = (RingOut *)S->hmap;
    S->h_xout = (double *)(S->hmap + align256((size_t)cap * sizeof(RingOut)));
    S->h_stop = (int *)(S->hstage + (size_t)cap * S->stage_slot + (size_t)cap * sizeof(long long));
    void *dp = nullptr;
    e = cudaHostGetDevicePointer(&dp, S->hmap, 0);
    if (e == cudaSuccess) {
      S->d_out = (RingOut *)dp;
      S->d_xout = (double *)((char *)dp + align256((size_t)cap * sizeof(RingOut)));
    }
  }
  if (e != cudaSuccess) {
    serve_free(S);
    delete S;
    set_error(std::string("nuppn_serve_open: ") + cudaGetErrorString(e));
    return NUPPN_ERR_NOMEM;
  }
  S->in_slot.assign(cap, nullptr);
  S->device_bytes = (int64_t)(S->ws.n + S->dq.n);
  S->worker = std::thread(serve_loop, S);
  *out = S;
  return NUPPN_OK;
}

static nuppn_status serve_enqueue(nuppn_server *S, ServeReq *r, int64_t *id) {
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (!S->fatal.empty()) {
      set_error(S->fatal);
      delete r;
      return NUPPN_ERR_CUDA;
    }
    r->id = S->next_id++;
    S->reqs[r->id] = r;
    S->pending.push_back(r);
    S->queued++;
  }
  S->cv.notify_one();
  *id = r->id;
  return NUPPN_OK;
}

nuppn_status nuppn_serve_submit(nuppn_server *srv, const double *X, double t9_0, double t9_1, double rho_0,
                                double rho_1, double ye, double dtwant, int32_t bd_state, int64_t *id) {
  if (!srv || !X || !id) { set_error("null argument"); return NUPPN_ERR_ARG; }
  ServeReq *r = new (std::nothrow) ServeReq();
  if (!r) return NUPPN_ERR_NOMEM;
  r->kind = 0;
  r->X.assign(X, X + srv->net->H.nsp);
  r->t9_0 = t9_0; r->t9_1 = t9_1; r->rho_0 = rho_0; r->rho_1 = rho_1; r->ye = ye; r->dtwant = dtwant;
  r->bd = bd_state;
  return serve_enqueue(srv, r, id);
}

nuppn_status nuppn_serve_submit_trajectory(nuppn_server *srv, const double *X, int32_t npts, const double *time,
                                           const double *t9, const double *rho, int64_t *id) {
  if (!srv || !X || !time || !t9 || !rho || !id) { set_error("null argument"); return NUPPN_ERR_ARG; }
  if (npts < 2) { set_error("npts < 2"); return NUPPN_ERR_ARG; }
  if (npts > kServeMaxPoints) {
    set_error("a served trajectory has at most " + std::to_string(kServeMaxPoints) + " points");
    return NUPPN_ERR_LIMIT;
  }
  ServeReq *r = new (std::nothrow) ServeReq();
  if (!r) return NUPPN_ERR_NOMEM;
  r->kind = 1;
  r->npts = npts;
  r->X.assign(X, X + srv->net->H.nsp);
  r->time.assign(time, time + npts);
  r->t9.assign(t9, t9 + npts);
  r->rho.assign(rho, rho + npts);
  return serve_enqueue(srv, r, id);
}

nuppn_status nuppn_serve_poll(nuppn_server *srv, int64_t id, int32_t *done, double *X, double *ye, int32_t *ierr,
                              nuppn_zone_stats *stats, int32_t *bd_state, int32_t *fail) {
  if (!srv || !done) { set_error("null argument"); return NUPPN_ERR_ARG; }
  ServeReq *r = nullptr;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->reqs.find(id);
    if (it == srv->reqs.end()) { set_error("unknown request id"); return NUPPN_ERR_ARG; }
    if (it->second->status == 0) { *done = 0; return NUPPN_OK; }
    r = it->second;
    srv->reqs.erase(it);
  }
  *done = 1;
  const int st = r->status;
  const std::string err = r->err;
  if (st == 1) {
    if (X) memcpy(X, r->X.data(), r->X.size() * 8);
    if (ye) *ye = r->ye;
    if (ierr) *ierr = r->ierr;
    if (stats) *stats = r->st;
    if (bd_state) *bd_state = r->bd;
    if (fail) *fail = r->fail;
  }
  delete r;
  if (st != 1) { set_error(err); return NUPPN_ERR_CUDA; }
  return NUPPN_OK;
}

nuppn_status nuppn_serve_info(nuppn_server *srv, nuppn_serve_stats *out) {
  if (!srv || !out) { set_error("null argument"); return NUPPN_ERR_ARG; }
  std::lock_guard<std::mutex> lk(srv->mu);
  out->slots = srv->slots;
  out->queue = srv->cap;
  out->ctas = srv->grid;
  out->pending = srv->queued.load();
  out->in_flight = srv->in_flight.load();
  out->launches = srv->launches.load();
  out->published = srv->published;
  out->completed = srv->completed.load();
  out->device_bytes = srv->device_bytes;
  return NUPPN_OK;
}

nuppn_status nuppn_serve_close(nuppn_server *srv) {
  if (!srv) return NUPPN_OK;
  srv->stop = true;
  srv->cv.notify_all();
  if (srv->worker.joinable()) srv->worker.join();
  cudaSetDevice(srv->net->device);
  serve_free(srv);
  for (auto &kv : srv->reqs) delete kv.second;
  delete srv;
  return NUPPN_OK;
}

}  // extern "C"
