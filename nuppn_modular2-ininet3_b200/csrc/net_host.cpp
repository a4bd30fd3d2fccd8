// net_host.cpp -- one-time host analysis of a network description (see net_host.h).
#include "net_host.h"

#include <algorithm>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <numeric>
#include <set>
#include <unordered_map>

namespace nuppn {

namespace {

// physical constants of utils/source/constants.F90
const double ev2erg = 1.602177e-12, mev2erg = ev2erg * 1.0e6, erg2mev = 1.0 / mev2erg;
const double pi = 3.141592653589793238462643383279502884;
const double clight = 2.99792458e10, clight2 = clight * clight;
const double planck_erg = 4.135667662e-21 * mev2erg;
const double amu = 1.6605402e-24, mp_mev = 938.27231, mn_mev = 939.56563, me_g = 9.10938356e-28;

enum { i_ng = 1, i_gn, i_np, i_na, i_pg, i_gp, i_pn, i_pa, i_ag };

template <class T>
std::vector<T> cp(const T *p, size_t n) {
  return (p && n) ? std::vector<T>(p, p + n) : std::vector<T>(n, T(0));
}

// Akima coefficients, the construction of utils/source/akima.F90:78-132 (abs_smooth delta 0.1)
void akima_coefs(int n, const double *x, const double *y, double *out /*[(n-1)*4]*/) {
  const double eps = 1e-30, dlt = 0.1;
  std::vector<double> mm(n + 3), t(n + 1);
  auto m = [&](int i) -> double & { return mm[i + 1]; };
  for (int i = 1; i <= n - 1; ++i) m(i) = (y[i] - y[i - 1]) / (x[i] - x[i - 1]);
  m(0) = 2.0 * m(1) - m(2);
  m(-1) = 2.0 * m(0) - m(1);
  m(n) = 2.0 * m(n - 1) - m(n - 2);
  m(n + 1) = 2.0 * m(n) - m(n - 1);
  auto sm = [&](double v) { return v >= dlt ? v : (v <= -dlt ? -v : v * v / (2.0 * dlt) + dlt / 2.0); };
  for (int i = 1; i <= n; ++i) {
    double m1 = m(i - 2), m2 = m(i - 1), m3 = m(i), m4 = m(i + 1);
    double w1 = sm(m4 - m3), w2 = sm(m2 - m1);
    t[i] = (w1 < eps && w2 < eps) ? 0.5 * (m2 + m3) : (w1 * m2 + w2 * m3) / (w1 + w2);
  }
  for (int i = 1; i <= n - 1; ++i) {
    double dx = x[i] - x[i - 1], t1 = t[i], t2 = t[i + 1];
    out[(i - 1) * 4 + 0] = y[i - 1];
    out[(i - 1) * 4 + 1] = t1;
    out[(i - 1) * 4 + 2] = (3.0 * m(i) - 2.0 * t1 - t2) / dx;
    out[(i - 1) * 4 + 3] = (t1 + t2 - 2.0 * m(i)) / (dx * dx);
  }
}

// Minimum-degree order on the symmetrised pattern (elimination graph), nodes in `last` kept for the
// end (in the given order). Ties go to the lower index, so the order is deterministic.
std::vector<int> min_degree(int n, const std::vector<std::vector<int>> &adj0, const std::vector<int> &last) {
  std::vector<std::set<int>> adj(n);
  for (int i = 0; i < n; ++i) adj[i] = std::set<int>(adj0[i].begin(), adj0[i].end());
  std::vector<char> alive(n, 1), islast(n, 0);
  for (int v : last) islast[v] = 1;
  std::set<std::pair<int, int>> pq;  // (degree, node); deg[] holds the key stored for each node
  std::vector<int> deg(n);
  for (int i = 0; i < n; ++i) {
    deg[i] = (int)adj[i].size();
    if (!islast[i]) pq.insert({deg[i], i});
  }
  std::vector<int> order;
  order.reserve(n);
  while (!pq.empty()) {
    int v = pq.begin()->second;
    pq.erase(pq.begin());
    order.push_back(v);
    alive[v] = 0;
    std::vector<int> nb(adj[v].begin(), adj[v].end());
    for (int a : nb) adj[a].erase(v);
    for (size_t x = 0; x < nb.size(); ++x)
      for (size_t y = 0; y < nb.size(); ++y)
        if (x != y) adj[nb[x]].insert(nb[y]);
    for (int a : nb) {
      if (islast[a] || (int)adj[a].size() == deg[a]) continue;
      pq.erase({deg[a], a});
      deg[a] = (int)adj[a].size();
      pq.insert({deg[a], a});
    }
    adj[v].clear();
  }
  for (int v : last) order.push_back(v);
  return order;
}

int group_for(double avg) {
  int g = 1;
  while (g < 32 && g < avg) g *= 2;
  return g;
}

}  // namespace

std::string read_isotope_database(const char *path, int nnn, std::vector<IsotopeEntry> &out) {
  out.clear();
  if (!path || nnn < 0) return "isotope database: bad argument";
  FILE *f = std::fopen(path, "r");
  if (!f) return std::string("isotope database: cannot open ") + path;
  char line[512];
  int header = 0, lineno = 0;
  std::string err;
  while ((int)out.size() < nnn && std::fgets(line, sizeof line, f)) {
    ++lineno;
    if (header < 3) {  // the reference skips three lines (nuc_data.F90:60-62)
      ++header;
      continue;
    }
    IsotopeEntry e;
    char el[16] = {0}, fl[16] = {0};
    if (std::sscanf(line, "%d %d %15s %lf %15s", &e.z, &e.a, el, &e.amin, fl) != 5) {
      // a blank line ends the list as an end of file would (nuc_data.F90:64-65, end=98778)
      bool blank = true;
      for (const char *c = line; *c; ++c) blank &= (*c == ' ' || *c == '\t' || *c == '\n' || *c == '\r');
      if (!blank) err = "isotope database: cannot parse line " + std::to_string(lineno);
      break;
    }
    if (std::strlen(el) > 2) {
      err = "isotope database: element symbol longer than 2 characters on line " + std::to_string(lineno);
      break;
    }
    std::memcpy(e.elem, el, std::strlen(el));
    const char c = fl[0];
    if (c == 'T' || c == 't') e.consider = true;
    else if (c == 'F' || c == 'f') e.consider = false;
    else {
      err = "isotope database: flag is not T or F on line " + std::to_string(lineno);
      break;
    }
    out.push_back(e);
  }
  std::fclose(f);
  if (!err.empty()) return err;
  if ((int)out.size() < nnn)
    return "isotope database: " + std::to_string(out.size()) + " entries, fewer than the " + std::to_string(nnn) +
           " requested";
  return "";
}

void bd_constants(HostNet &H) {  // bader_deuflhard.F90:66-124
  const double cf = 1, cj = 0.0, cs = 10, clr = cj, safe1 = 0.25, alpha = 5.0 / 7.0;
  const int nl = kMaxLevels;
  std::memset(H.nseq, 0, sizeof(H.nseq));
  std::memset(H.bd_a, 0, sizeof(H.bd_a));
  std::memset(H.alf, 0, sizeof(H.alf));
  H.nseq[1] = 2; H.nseq[2] = 6; H.nseq[3] = 10;
  for (int i = 4; i <= nl + 1; ++i) H.nseq[i] = (int)std::lround((double)H.nseq[i - 1] / alpha);
  H.bd_a[1] = cj + clr + (H.nseq[1] + 1) * (cf + cs);
  for (int i = 2; i <= nl; ++i) H.bd_a[i] = H.bd_a[i - 1] + H.nseq[i] * (cf + cs) + clr + cs;
  for (int iq = 2; iq <= nl; ++iq)
    for (int k = 1; k <= iq - 1; ++k)
      H.alf[k][iq] = std::pow(H.kn.dgrd * safe1,
                              (H.bd_a[k + 1] - H.bd_a[iq + 1]) / ((H.bd_a[iq + 1] - H.bd_a[1] + 1.0) * (2.0 * k + 1)));
  int kopt;
  H.kmax = 0;
  for (kopt = 2; kopt <= nl - 1; ++kopt)
    if (H.bd_a[kopt + 1] > H.bd_a[kopt] * H.alf[kopt - 1][kopt]) { H.kmax = kopt; break; }
  H.kopt0 = kopt;
}

std::string build_host_net(const nuppn_net_desc &d, const nuppn_knobs &kn, HostNet &H) {
  H.kn = kn;
  const int nsp = d.nsp, nre = d.nre;
  if (nsp <= 0 || nre < 0 || !d.anetw || !d.znetw || !d.considerisotope || !d.k || !d.considerreaction ||
      !d.ilabb || !d.src || !d.src_idx)
    return "descriptor: missing species or reaction arrays";
  if (d.igamma < 0 || d.igamma >= nsp) return "descriptor: igamma out of range";
  H.nsp = nsp; H.nre = nre; H.ig = d.igamma;
  H.an = cp(d.anetw, nsp); H.zn = cp(d.znetw, nsp); H.ciso = cp(d.considerisotope, nsp);
  H.spart = d.spec_part ? cp(d.spec_part, nsp) : std::vector<int>(nsp, -1);
  H.crea = cp(d.considerreaction, nre); H.ilabb = cp(d.ilabb, nre);
  H.src = cp(d.src, nre); H.sidx = cp(d.src_idx, nre);
  H.rfac = d.rfac ? cp(d.rfac, nre) : std::vector<double>(nre, 1.0);
  H.irev = d.irev ? cp(d.irev, nre) : std::vector<int>(nre, -1);
  H.k_all = cp(d.k, (size_t)nre * 8);
  H.nvar = 0;
  for (int i = 0; i < nsp; ++i) H.nvar += H.ciso[i] ? 1 : 0;
  for (int i = 0; i < nsp; ++i) {
    if (H.zn[i] == 2 && H.an[i] == 4) H.ihe4 = i;
    if (H.zn[i] == 4 && H.an[i] == 8) H.ibe8 = i;
  }
  // ---- validation of the reaction slots
  for (int l = 0; l < nre; ++l) {
    if (!H.crea[l]) continue;
    const int *k = &H.k_all[(size_t)l * 8];
    for (int s = 0; s < 8; s += 2)
      if (k[s] < 0 || k[s] >= nsp) return "descriptor: k index out of range in reaction " + std::to_string(l);
    if (k[1] < 0 || k[1] > 4 || k[3] < 0 || k[3] > 4) return "descriptor: reactant count outside 0..4";
    if (k[0] == H.ig || k[6] == H.ig) return "descriptor: k1/k7 is the gamma slot";
    for (int s = 0; s < 8; s += 2)
      if (k[s] != H.ig && !H.ciso[k[s]])
        return "descriptor: considered reaction " + std::to_string(l) + " has a species that is not considered";
    if (H.irev[l] >= nre) return "descriptor: irev out of range";
  }
  // ---- nuclear data (nse_swj.F90:186-196)
  std::vector<double> ex = cp(d.exmass, nsp), gs = d.gspin ? cp(d.gspin, nsp) : std::vector<double>(nsp, 1.0);
  std::vector<double> ppn_m(nsp, 0.0), ppn_q(nsp, 0.0);
  H.gspin_nse.assign(nsp, 0.0);
  for (int i = 0; i < nsp; ++i) {
    if (i == H.ig) continue;
    double z = H.zn[i], n = H.an[i] - H.zn[i];
    ppn_m[i] = ex[i] * mev2erg / clight2 + H.an[i] * amu;
    ppn_m[i] = ppn_m[i] - z * me_g;
    ppn_q[i] = z * mp_mev + n * mn_mev - ppn_m[i] * clight2 * erg2mev;
    if (H.an[i] == 1.0 && (z == 0.0 || z == 1.0)) ppn_q[i] = 0.0;
    if (H.ciso[i] && H.an[i] != 0 && gs[i] != 0 && ppn_m[i] != 0) H.gspin_nse[i] = gs[i];
  }
  for (int i = 0; i < nsp; ++i) {
    if (H.gspin_nse[i] == 0.0) continue;
    const int j = (int)H.nse_idx.size();
    if (H.zn[i] == 1 && H.an[i] == 1) H.nse_iprot = j;
    if (H.zn[i] == 28 && H.an[i] == 56) H.nse_ini56 = j;
    H.nse_idx.push_back(i);
    H.nse_part.push_back(H.spart[i]);
    H.nse_m.push_back(ppn_m[i]);
    H.nse_q.push_back(ppn_q[i]);
    H.nse_g.push_back(gs[i]);
    H.nse_z.push_back(H.zn[i]);
    H.nse_n.push_back(H.an[i] - H.zn[i]);
    H.nse_zoa.push_back(H.zn[i] / H.an[i]);
  }
  while (H.nse_p2 < nsp) H.nse_p2 *= 2;
  if (kn.i_nse == 1 && (H.nse_iprot < 0 || H.nse_ini56 < 0))
    return "i_nse = 1 needs protons and Ni56 among the considered species (compute_nse's guess and Coulomb terms)";
  // ---- rate slots: screening, reverse constants, 'RVRSE' targets
  H.scr_mode.assign(nre, 0); H.scr_z1.assign(nre, 0.0); H.scr_z2.assign(nre, 0.0);
  H.rev_target.assign(nre, 0);
  H.rev_sp.assign((size_t)nre * 4, -1); H.rev_kind.assign(nre, 0);
  H.rev_mc.assign(nre, 0.0); H.rev_Q.assign(nre, 0.0);
  for (int l = 0; l < nre; ++l) {
    const int *k = &H.k_all[(size_t)l * 8];
    int slot = l + 1;  // reference numbering (evaluate_rates.F90:69-121)
    if (slot == 43) H.scr_mode[l] = 1;
    else if (slot == 109) H.scr_mode[l] = 2;
    else if (!H.crea[l] && slot > 110) H.scr_mode[l] = 3;
    else {
      bool ok = k[0] >= 0 && k[0] < nsp && k[2] >= 0 && k[2] < nsp;
      H.scr_z1[l] = ok ? H.zn[k[0]] : 0.0;
      H.scr_z2[l] = ok ? (k[1] == 2 ? H.zn[k[0]] : H.zn[k[2]]) : 0.0;
    }
    if (H.crea[l] && H.irev[l] >= 0) {
      H.rev_target[H.irev[l]] = 1;
      int a1 = k[0], a2 = k[2], b1 = k[4], b2 = k[6], na1 = k[1], nb1 = k[5], nb2 = k[7];
      if ((na1 != 1 && na1 != 2) || (nb2 != 1 && nb2 != 2)) continue;  // reverse_rate ierr = 1
      int a2e = na1 == 1 ? a2 : a1;
      int b1e = nb2 == 2 ? b2 : (nb1 == 1 ? b1 : -1);
      double m_a1 = ppn_m[a1], m_a2 = ppn_m[a2e], m_b2 = ppn_m[b2], m_b1 = b1e >= 0 ? ppn_m[b1e] : 0.0;
      int *rs = &H.rev_sp[(size_t)l * 4];
      rs[0] = a1; rs[1] = a2e; rs[2] = b1e; rs[3] = b2;
      int t = H.ilabb[l];
      if (t == i_ng || t == i_pg || t == i_ag) {
        H.rev_kind[l] = 1;
        H.rev_mc[l] = m_a1 * m_a2 / m_b2 * 2.0 * pi / planck_erg / planck_erg;
        H.rev_Q[l] = -ppn_q[a1] - ppn_q[a2] + ppn_q[b2];
      } else {
        H.rev_kind[l] = 2;
        H.rev_mc[l] = std::pow(m_a1 * m_a2 / m_b1 / m_b2, 1.5);
        H.rev_Q[l] = -ppn_q[a1] - ppn_q[a2] + ppn_q[b1] + ppn_q[b2];
      }
    }
  }
  // ---- rate tables
  H.nc = d.rl_ncontrib; H.nr = d.rl_nrate;
  if (H.nc > 0 && (!d.rl_a || !d.rl_rate)) return "descriptor: REACLIB arrays missing";
  H.rl_a = cp(d.rl_a, (size_t)H.nc * 7);
  std::vector<int> rr = cp(d.rl_rate, H.nc);
  H.rl_first.assign(H.nr + 1, 0);
  for (int i = 0; i < H.nc; ++i) {
    if (rr[i] < 0 || rr[i] >= H.nr) return "descriptor: rl_rate out of range";
    if (i > 0 && rr[i] < rr[i - 1]) return "descriptor: rl_rate must be non-decreasing";
    H.rl_first[rr[i] + 1]++;
  }
  for (int r = 0; r < H.nr; ++r) H.rl_first[r + 1] += H.rl_first[r];
  std::vector<int> ch = cp(d.rl_chapter, H.nr), nir = cp(d.rl_nireac, H.nr);
  std::vector<uint8_t> vf = cp(d.rl_vflag, H.nr), ecf = cp(d.rl_ecflag, H.nr);
  H.rl_info.resize(H.nr);
  for (int r = 0; r < H.nr; ++r) H.rl_info[r] = (ch[r] & 0xff) | ((vf[r] ? 1 : 0) << 8) | ((ecf[r] ? 1 : 0) << 9) | (nir[r] << 16);
  H.rl_part = cp(d.rl_part, (size_t)H.nr * 6);
  H.npart = d.npart;
  H.pt9 = cp(d.part_t9, kPartDim);
  H.pval = cp(d.part_val, (size_t)H.npart * kPartDim);
  for (int r = 0; r < H.nr * 6; ++r)
    if (H.rl_part[r] >= H.npart) return "descriptor: rl_part out of range";
  H.nv = d.vt_nrate;
  H.vfirst = cp(d.vt_first, H.nv + 1); H.vterms = cp(d.vt_terms, (size_t)d.vt_nterm * 5);
  H.vdpow = cp(d.vt_dpow, H.nv); H.vxfac = cp(d.vt_xfac, H.nv);
  H.vform = d.vt_form ? cp(d.vt_form, H.nv) : std::vector<int>(H.nv, 0);
  for (int i = 0; i < H.nv; ++i) {
    const int f = H.vform[i];
    const bool known = f == 0 || (f >= 1 && f <= 9) || (f >= 14 && f <= 17) || f == 73;
    if (!known) return "descriptor: vt_form names a VITAL slot without a formula here (1-9, 14-17, 73)";
    if (f == 5 && (H.vxfac[i] < 0 || H.vxfac[i] >= d.nsp)) return "descriptor: VITAL slot 5 needs vt_xfac = protons";
  }
  H.ngk = d.ng_kgrid; H.ngn = d.ng_nreac; H.ngd = std::max(1, d.ng_ndmax);
  H.ngt8 = cp(d.ng_t8, H.ngk); H.ngflag = cp(d.ng_flag, H.ngn); H.ngndata = cp(d.ng_ndata, H.ngn);
  H.ngane = cp(d.ng_ane, (size_t)H.ngn * H.ngd); H.ngl10v = cp(d.ng_l10v, (size_t)H.ngk * H.ngn * H.ngd);
  H.ngl10t8.resize(H.ngk);
  for (int i = 0; i < H.ngk; ++i) H.ngl10t8[i] = std::log10(H.ngt8[i]);
  if (H.ngn > 0 && H.ngk < 2) return "descriptor: NETGEN temperature grid needs >= 2 points";
  for (int i = 0; i < H.ngn; ++i)
    if (H.ngflag[i] > 0.0 && (H.ngndata[i] < 2 || H.ngndata[i] > H.ngd))
      return "descriptor: density-tabulated NETGEN rate needs 2..ndmax density points";
  for (int i = 0; i < nsp; ++i)
    if (H.spart[i] >= d.npart) return "descriptor: spec_part out of range";
  if (d.npart > 0 && !d.part_t9) return "descriptor: partition grid missing";
  H.ffv = d.ff_nv; H.fft = d.ff_nt; H.ffr = d.ff_nr;
  H.fft9 = cp(d.ff_t9coo, H.fft); H.ffrho = cp(d.ff_rhocoo, H.ffr);
  H.ffl10v = cp(d.ff_l10v, (size_t)H.ffv * H.fft * H.ffr);
  H.kdn = d.kd_n; H.kde = d.kd_ne;
  if (H.ffv > 0 && (H.fft < 2 || H.ffr < 2)) return "descriptor: FFN grid needs >= 2 points per axis";
  if (H.kdn > 0 && (H.kde < 3 || !d.kd_rate || !d.kd_e)) return "descriptor: KADoNiS table needs >= 3 energies";
  H.kdE = cp(d.kd_e, H.kde);
  H.kdcoef.assign((size_t)H.kdn * std::max(0, H.kde - 1) * 4, 0.0);
  for (int i = 0; i < H.kdn; ++i)
    akima_coefs(H.kde, H.kdE.data(), d.kd_rate + (size_t)i * H.kde, &H.kdcoef[(size_t)i * (H.kde - 1) * 4]);
  H.constr = d.nconst > 0 ? cp(d.const_rate, d.nconst) : std::vector<double>(1, 0.0);
  for (int l = 0; l < nre; ++l) {
    int s = H.src[l], i = H.sidx[l];
    int lim = s == NUPPN_SRC_VITAL ? H.nv : s == NUPPN_SRC_REACLIB ? H.nr : s == NUPPN_SRC_NETGEN ? H.ngn
            : s == NUPPN_SRC_FULLER ? H.ffv : s == NUPPN_SRC_KADONIS ? H.kdn : s == NUPPN_SRC_CONST ? d.nconst : 1 << 30;
    if (s != NUPPN_SRC_NONE && (i < 0 || i >= lim)) return "descriptor: src_idx out of range in slot " + std::to_string(l);
  }
  // ---- active reactions
  for (int l = 0; l < nre; ++l)
    if (H.crea[l]) H.act_slot.push_back(l);
  H.nact = (int)H.act_slot.size();
  // ---- makemap (jac_rhs.F90:461-540): pattern numbered row-major
  std::vector<std::vector<int>> rowsets(nsp);
  for (int l : H.act_slot) {
    const int *k = &H.k_all[(size_t)l * 8];
    int in1 = k[0], in2 = k[2], out1 = k[4], out2 = k[6];
    for (int c : {in1, in2})
      for (int r : {in1, in2, out1, out2}) rowsets[r].push_back(c);
  }
  for (int i = 0; i < nsp; ++i)
    if (H.ciso[i]) rowsets[i].push_back(i);
  std::vector<int> jrowptr(nsp + 1, 0);
  for (int i = 0; i < nsp; ++i) {
    auto &v = rowsets[i];
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    jrowptr[i + 1] = jrowptr[i] + (int)v.size();
    for (int c : v) { H.jrow.push_back(i); H.jcol.push_back(c); }
  }
  H.nnzJ = (int)H.jrow.size();
  auto entry = [&](int r, int c) -> int {
    auto &v = rowsets[r];
    auto it = std::lower_bound(v.begin(), v.end(), c);
    return (it != v.end() && *it == c) ? jrowptr[r] + (int)(it - v.begin()) : -1;
  };
  H.jdiag.assign(nsp, -1);
  for (int i = 0; i < nsp; ++i) H.jdiag[i] = entry(i, i);
  H.dmap_all.assign((size_t)nre * 8, -1);
  H.act_k.resize((size_t)H.nact * 8);
  H.act_ice.resize((size_t)H.nact * 8);
  for (int a = 0; a < H.nact; ++a) {
    int l = H.act_slot[a];
    const int *k = &H.k_all[(size_t)l * 8];
    int in1 = k[0], in2 = k[2], out1 = k[4], out2 = k[6];
    int rws[8] = {in1, in2, out1, out2, in1, in2, out1, out2};
    int cls[8] = {in1, in1, in1, in1, in2, in2, in2, in2};
    for (int s = 0; s < 8; ++s) {
      int e = entry(rws[s], cls[s]);
      H.dmap_all[(size_t)l * 8 + s] = e;
      H.act_ice[(size_t)a * 8 + s] = e;
      H.act_k[(size_t)a * 8 + s] = k[s];
    }
  }
  // ---- reactions by their first reactant (every considered reaction once; k1 is never gamma)
  H.k1_ptr.assign(nsp + 1, 0);
  for (int a = 0; a < H.nact; ++a) H.k1_ptr[H.act_k[(size_t)a * 8] + 1]++;
  for (int i = 0; i < nsp; ++i) H.k1_ptr[i + 1] += H.k1_ptr[i];
  H.k1_list.assign(H.nact, 0);
  {
    std::vector<int> fill(H.k1_ptr.begin(), H.k1_ptr.end() - 1);
    for (int a = 0; a < H.nact; ++a) H.k1_list[fill[H.act_k[(size_t)a * 8]]++] = a;
  }
  // ---- gather lists in the reference's accumulation order
  {
    std::vector<std::vector<int>> lists(H.nnzJ);
    const int upd_order[8] = {0, 1, 4, 2, 3, 5, 6, 7};  // ice1..ice8 of jac_rhs.F90:365-392
    for (int a = 0; a < H.nact; ++a)
      for (int u = 0; u < 8; ++u) {
        int s = upd_order[u];
        lists[H.act_ice[(size_t)a * 8 + s]].push_back(a * 8 + s);
      }
    H.jg_ptr.assign(H.nnzJ + 1, 0);
    for (int e = 0; e < H.nnzJ; ++e) H.jg_ptr[e + 1] = H.jg_ptr[e] + (int)lists[e].size();
    H.jg_item.reserve(H.jg_ptr[H.nnzJ]);
    for (auto &L : lists) H.jg_item.insert(H.jg_item.end(), L.begin(), L.end());
    H.jg_oth.reserve(H.jg_item.size());
    for (int it : H.jg_item) {
      const int *k = &H.act_k[(size_t)(it >> 3) * 8];
      const int o = (it & 7) < 4 ? k[2] : k[0];  // slots 0-3: d/dy(k1), the other is k3; 4-7: d/dy(k3)
      H.jg_oth.push_back(o == H.ig ? -1 : o);
    }
  }
  {
    std::vector<std::vector<int>> lists(nsp);
    for (int a = 0; a < H.nact; ++a)
      for (int q = 0; q < 4; ++q) lists[H.act_k[(size_t)a * 8 + 2 * q]].push_back(a * 4 + q);
    H.dg_ptr.assign(nsp + 1, 0);
    for (int i = 0; i < nsp; ++i) H.dg_ptr[i + 1] = H.dg_ptr[i] + (int)lists[i].size();
    for (auto &L : lists) H.dg_item.insert(H.dg_item.end(), L.begin(), L.end());
    for (int it : H.dg_item) {
      int a = it >> 2, q = it & 3;
      const int *k = &H.act_k[(size_t)a * 8];
      H.dg_coef.push_back(q == 0 ? (double)(-k[1]) : q == 1 ? -1.0 : q == 2 ? (double)k[5] : (double)k[7]);
    }
    for (int i = 0; i < nsp; ++i)
      if (H.dg_ptr[i + 1] - H.dg_ptr[i] > 48) H.dg_long.push_back(i);
    for (int e = 0; e < H.nnzJ; ++e)
      if (H.jg_ptr[e + 1] - H.jg_ptr[e] > 48) H.jg_long.push_back(e);
  }
  // ---- linear system: considered species except gamma, fill-reducing order
  std::vector<int> sys0;
  for (int i = 0; i < nsp; ++i)
    if (H.ciso[i] && i != H.ig) sys0.push_back(i);
  int n = (int)sys0.size();
  if (n >= (1 << 14) - 1) return "more than 16382 species in the linear system";  // 14-bit compact indices
  H.nsys = n;
  std::vector<int> sidx0(nsp, -1);
  for (int q = 0; q < n; ++q) sidx0[sys0[q]] = q;
  std::vector<std::vector<int>> adj(n);
  for (int e = 0; e < H.nnzJ; ++e) {
    int r = sidx0[H.jrow[e]], c = sidx0[H.jcol[e]];
    if (r < 0 || c < 0 || r == c) continue;
    adj[r].push_back(c);
    adj[c].push_back(r);
  }
  for (auto &v : adj) { std::sort(v.begin(), v.end()); v.erase(std::unique(v.begin(), v.end()), v.end()); }
  // dense rows/columns (the light particles n, p, alpha, ...) are ordered last, by degree
  std::vector<int> last;
  for (int q = 0; q < n; ++q)
    if ((int)adj[q].size() > std::max(32, n / 10)) last.push_back(q);
  std::sort(last.begin(), last.end(), [&](int x, int y) {
    return adj[x].size() != adj[y].size() ? adj[x].size() < adj[y].size() : x < y;
  });
  std::vector<int> order = min_degree(n, adj, last);  // order[newpos] = old system index
  H.sp_of_sys.resize(n);
  H.sys_of_sp.assign(nsp, -1);
  std::vector<int> newpos(n);
  for (int p = 0; p < n; ++p) { newpos[order[p]] = p; H.sp_of_sys[p] = sys0[order[p]]; H.sys_of_sp[sys0[order[p]]] = p; }
  // ---- symbolic factorization, static diagonal pivots, row-wise (up-looking)
  std::vector<std::vector<int>> arow(n);
  for (int e = 0; e < H.nnzJ; ++e) {
    int r = H.sys_of_sp[H.jrow[e]], c = H.sys_of_sp[H.jcol[e]];
    if (r < 0 || c < 0) continue;
    arow[r].push_back(c);
  }
  std::vector<std::vector<int>> upat(n);  // U part (cols > i), sorted
  H.lu_rowptr.assign(n + 1, 0);
  H.lu_diag.assign(n, 0);
  std::vector<char> mark(n, 0);
  for (int i = 0; i < n; ++i) {
    std::set<int> lpend;
    std::vector<int> cols;
    arow[i].push_back(i);
    for (int c : arow[i])
      if (!mark[c]) { mark[c] = 1; cols.push_back(c); if (c < i) lpend.insert(c); }
    std::vector<int> lcols;
    while (!lpend.empty()) {
      int j = *lpend.begin();
      lpend.erase(lpend.begin());
      lcols.push_back(j);
      for (int c : upat[j])
        if (!mark[c]) { mark[c] = 1; cols.push_back(c); if (c < i) lpend.insert(c); }
    }
    for (int c : cols) mark[c] = 0;
    std::sort(cols.begin(), cols.end());
    for (int c : cols) {
      if (c == i) H.lu_diag[i] = (int)H.lu_col.size();
      if (c > i) upat[i].push_back(c);
      H.lu_col.push_back(c);
    }
    H.lu_rowptr[i + 1] = (int)H.lu_col.size();
  }
  H.nnzLU = (int)H.lu_col.size();
  // ---- update map: for each L entry (i,j), offsets in row i of the columns of U(j)
  H.upd_start.assign(H.nnzLU + 1, 0);
  {
    std::vector<int> posinrow(n, -1);
    std::vector<uint16_t> offs;
    for (int i = 0; i < n; ++i) {
      int rs = H.lu_rowptr[i], re = H.lu_rowptr[i + 1];
      if (re - rs > 65535) return "network too large for 16-bit row offsets";
      for (int p = rs; p < re; ++p) posinrow[H.lu_col[p]] = p - rs;
      for (int p = rs; p < re; ++p) {
        H.upd_start[p] = (int)offs.size();
        if (p < H.lu_diag[i]) {
          int j = H.lu_col[p];
          for (int q = H.lu_diag[j] + 1; q < H.lu_rowptr[j + 1]; ++q) {
            int o = posinrow[H.lu_col[q]];
            if (o < 0) return "symbolic factorization is not closed under fill";
            offs.push_back((uint16_t)o);
          }
          H.lu_flops += H.lu_rowptr[j + 1] - H.lu_diag[j] - 1;
        }
      }
      for (int p = rs; p < re; ++p) posinrow[H.lu_col[p]] = -1;
    }
    H.upd_start[H.nnzLU] = (int)offs.size();
    H.upd_off.swap(offs);
  }
  // ---- level schedules
  {
    std::vector<int> lvL(n, 0), lvU(n, 0);
    for (int i = 0; i < n; ++i)
      for (int p = H.lu_rowptr[i]; p < H.lu_diag[i]; ++p) lvL[i] = std::max(lvL[i], lvL[H.lu_col[p]] + 1);
    for (int i = n - 1; i >= 0; --i)
      for (int p = H.lu_diag[i] + 1; p < H.lu_rowptr[i + 1]; ++p) lvU[i] = std::max(lvU[i], lvU[H.lu_col[p]] + 1);
    auto build = [&](const std::vector<int> &lv, bool lower, std::vector<int> &ptr, std::vector<int> &rows,
                     std::vector<int> &grp) {
      int nl = n ? *std::max_element(lv.begin(), lv.end()) + 1 : 0;
      std::vector<std::vector<int>> b(nl);
      for (int i = 0; i < n; ++i) b[lv[i]].push_back(i);
      ptr.assign(nl + 1, 0);
      grp.assign(nl, 1);
      for (int l = 0; l < nl; ++l) {
        ptr[l + 1] = ptr[l] + (int)b[l].size();
        double tot = 0;
        for (int i : b[l]) {
          rows.push_back(i);
          tot += lower ? H.lu_diag[i] - H.lu_rowptr[i] : H.lu_rowptr[i + 1] - H.lu_diag[i] - 1;
        }
        grp[l] = group_for(b[l].empty() ? 1.0 : tot / b[l].size());
      }
    };
    build(lvL, true, H.lvL_ptr, H.lvL_rows, H.lvL_grp);
    build(lvU, false, H.lvU_ptr, H.lvU_rows, H.lvU_grp);
  }
  // ---- Jacobian entry -> LU position
  H.pos_of_entry.assign(H.nnzJ, -1);
  for (int e = 0; e < H.nnzJ; ++e) {
    int r = H.sys_of_sp[H.jrow[e]], c = H.sys_of_sp[H.jcol[e]];
    if (r < 0 || c < 0) continue;
    auto b = H.lu_col.begin() + H.lu_rowptr[r], en = H.lu_col.begin() + H.lu_rowptr[r + 1];
    auto it = std::lower_bound(b, en, c);
    H.pos_of_entry[e] = (int)(it - H.lu_col.begin());
  }
  H.lu_src.assign(H.nnzLU, -1);
  for (int e = 0; e < H.nnzJ; ++e)
    if (H.pos_of_entry[e] >= 0) H.lu_src[H.pos_of_entry[e]] = e;
  bd_constants(H);
  return "";
}

}  // namespace nuppn
