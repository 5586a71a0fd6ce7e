// Host-side CCD problem builder (see include/ccdhost.h for the contract).
//
// Builds, for the three reference models, exactly the inputs the reference's own host hands
// to its CCD loop: orbitals in the reference order, normal-ordered energies, regular and
// modified channels permuted by the 1-rank first-fit-decreasing balance, sorted channel and
// three-body maps, the eight remap tables and the V blocks.  Everything is derived directly
// from the channel structure in O(#T2) work instead of the reference's hash-table passes, and
// every matrix element is evaluated with the same floating-point expression as the reference,
// so the blocks are bit-identical.
#include "ccdhost.h"
#include "channel_order.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <string>
#include <vector>

namespace {

enum ModelKind { kPairing, kInfMatter, kElectronGas };

// Legendre's three-square theorem test and the integer ceil-sqrt used to turn shell counts
// into |n|^2 cut-offs (util.cpp:1-19).
bool sum_of_three_squares(unsigned n) {
  if (n == 0) return true;
  while (n % 4 == 0) n /= 4;
  return (n % 8) != 7;
}
unsigned ceil_sqrt(unsigned x) {
  unsigned r = 1;
  while (r * r < x) r++;
  return r;
}
// The reference advances its cut-off E until `shells` non-empty |n|^2 shells are covered
// (ElectronGasSPBasis.cpp:38-43, 69-74).
unsigned shell_cutoff(uint64_t shells) {
  unsigned e = 0;
  for (uint64_t i = 1; i < shells; e++)
    if (sum_of_three_squares(e + 1)) i++;
  return e;
}

struct Model {
  ModelKind kind;
  uint64_t nsp = 0, np = 0;
  int stride = 5;
  std::vector<int32_t> qn;      // SPBasis::indexMap rows
  std::vector<double> eps;      // bare single-particle energies
  int nmax = 0, tz_max = 1, chan_tz_max = -2, mod_chan_tz_max = 0;
  uint64_t nchan = 0;
  double L = 0, e_sq = 0, density = 0, g = 0, xi = 0;

  const int32_t *q(uint64_t p) const { return &qn[p * stride]; }

  // Unpermuted regular / modified channel index (ElectronGasSPBasis.cpp:572-624,
  // InfMatterSPBasis.cpp:458-510, PairingSPBasis.cpp:168-181).
  uint64_t chan0(uint64_t p, uint64_t r) const {
    const int32_t *a = q(p), *b = q(r);
    if (kind == kPairing) return (uint64_t)((a[1] + b[1] + 2) / 2);
    const uint64_t n = 4 * (uint64_t)nmax + 1, s = 3, t = 2 + chan_tz_max / 2;
    uint64_t nx = a[0] + b[0] + n / 2, ny = a[1] + b[1] + n / 2, nz = a[2] + b[2] + n / 2;
    uint64_t sz = (a[3] + b[3] + 2) / 2, tz = (a[4] + b[4] + 2) / 2;
    return nx * n * n * s * t + ny * n * s * t + nz * s * t + sz * t + tz;
  }
  uint64_t mod0(uint64_t p, uint64_t r) const {
    const int32_t *a = q(p), *b = q(r);
    if (kind == kPairing) return (uint64_t)((a[1] - b[1] + 2) / 2);
    const uint64_t n = 4 * (uint64_t)nmax + 1, s = 3, t = 1 + mod_chan_tz_max;
    uint64_t nx = a[0] - b[0] + n / 2, ny = a[1] - b[1] + n / 2, nz = a[2] - b[2] + n / 2;
    uint64_t sz = (a[3] - b[3] + 2) / 2, tz = (a[4] - b[4] + mod_chan_tz_max) / 2;
    return nx * n * n * s * t + ny * n * s * t + nz * s * t + sz * t + tz;
  }

  // Direct (not antisymmetrised) matrix elements, same expression order as the reference.
  double direct_eg(uint64_t p, uint64_t r, uint64_t s, uint64_t t) const {
    const int32_t *qi = q(p), *qj = q(r), *qk = q(s), *ql = q(t);
    double vout = 0.;
    if (qi[3] == qk[3] && qj[3] == ql[3]) {
      if (qi[0] + qj[0] == qk[0] + ql[0] && qi[1] + qj[1] == qk[1] + ql[1] &&
          qi[2] + qj[2] == qk[2] + ql[2]) {
        double prefactor = e_sq / (L * L * L);
        double rel = 0.0, mu = 0.0;
        for (int i = 0; i < 3; i++) {
          double term = 2 * M_PI * (qi[i] - qk[i]) / L;
          rel += term * term;
        }
        if (rel < 1.e-5) vout = 0.0;
        else vout = prefactor * 4 * M_PI / (rel + mu * mu);
      }
    }
    return vout;
  }
  double direct_pnm(uint64_t p, uint64_t r, uint64_t s, uint64_t t) const {
    const int32_t *qi = q(p), *qj = q(r), *qk = q(s), *ql = q(t);
    double vout = 0.;
    if (qi[0] + qj[0] == qk[0] + ql[0] && qi[1] + qj[1] == qk[1] + ql[1] &&
        qi[2] + qj[2] == qk[2] + ql[2]) {
      double Lb = pow(np / density, 1. / 3.);
      const double v0r = 200, v0t = 178, v0s = 91.85;
      const double kr = 1.487, kt = 0.639, ks = 0.465;
      double q2 = 0.;
      for (int i = 0; i < 3; i++) {
        double ki = 2 * M_PI * qi[i] / Lb, kj = 2 * M_PI * qj[i] / Lb;
        double kk = 2 * M_PI * qk[i] / Lb, kl = 2 * M_PI * ql[i] / Lb;
        double bra = 0.5 * (ki - kj), ket = 0.5 * (kk - kl);
        double tr = bra - ket;
        q2 += tr * tr;
      }
      double vr = v0r / (Lb * Lb * Lb) * pow(M_PI / kr, 1.5) * exp(-q2 / (4 * kr));
      double vt = -v0t / (Lb * Lb * Lb) * pow(M_PI / kt, 1.5) * exp(-q2 / (4 * kt));
      double vs = -v0s / (Lb * Lb * Lb) * pow(M_PI / ks, 1.5) * exp(-q2 / (4 * ks));
      double spin_ex = (qi[3] == ql[3] && qj[3] == qk[3]) ? 1 : 0;
      double iso_ex = (qi[4] == ql[4] && qj[4] == qk[4]) ? 1 : 0;
      int d_s = (qi[3] == qk[3]) * (qj[3] == ql[3]);
      int d_t = (qi[4] == qk[4]) * (qj[4] == ql[4]);
      double is_it = d_s * d_t;
      double ps_it = spin_ex * d_t;
      double ps_pt = spin_ex * iso_ex;
      double is_pt = d_s * iso_ex;
      vout = 0.5 * (vr + 0.5 * vt + 0.5 * vs) * is_it + 0.25 * (vt - vs) * ps_it -
             0.5 * (vr + 0.5 * vt + 0.5 * vs) * ps_pt - 0.25 * (vt - vs) * is_pt;
    }
    return vout;
  }
  // Antisymmetrised <pq|v|rs> (SPBasis::calcTBME of each model).
  double tbme(uint64_t p, uint64_t r, uint64_t s, uint64_t t) const {
    if (kind == kPairing) {
      const int32_t *a = q(p), *b = q(r), *c = q(s), *d = q(t);
      double vout = 0.;
      if (a[0] == b[0] && c[0] == d[0] && a[1] == -b[1] && -c[1] == d[1]) {
        vout = -0.5 * g;
        if (a[1] == -c[1]) vout = -vout;
      }
      return vout;
    }
    if (kind == kElectronGas) return direct_eg(p, r, s, t) - direct_eg(p, r, t, s);
    return direct_pnm(p, r, s, t) - direct_pnm(p, r, t, s);
  }
};

// Plane-wave orbitals: |n|^2 <= emax, ordered by |n|^2 then (nx, ny, nz, sz, tz) loop order
// (InfMatterSPBasis.cpp:13-161, ElectronGasSPBasis.cpp:14-170).
void plane_wave_orbitals(Model &m, uint64_t n_shells, uint64_t n_particle_shells) {
  unsigned emax = shell_cutoff(n_shells);
  int nmax = (int)ceil_sqrt(emax);
  int nmax_actual = 0;
  uint64_t nsp = 0;
  for (int nx = -nmax; nx <= nmax; nx++)
    for (int ny = -nmax; ny <= nmax; ny++)
      for (int nz = -nmax; nz <= nmax; nz++)
        if ((unsigned)(nx * nx + ny * ny + nz * nz) <= emax) {
          if (nx > nmax_actual) nmax_actual = nx;
          nsp += 2 * (uint64_t)m.tz_max;
        }
  m.nmax = nmax_actual;
  unsigned ef = shell_cutoff(n_particle_shells);
  int pmax = (int)ceil_sqrt(ef);
  uint64_t np = 0;
  for (int nx = -pmax; nx <= pmax; nx++)
    for (int ny = -pmax; ny <= pmax; ny++)
      for (int nz = -pmax; nz <= pmax; nz++)
        if ((unsigned)(nx * nx + ny * ny + nz * nz) <= ef) np += 2 * (uint64_t)m.tz_max;
  m.nsp = nsp;
  m.np = np;
  std::vector<uint64_t> start(emax + 2, 0);
  const int n = m.nmax;
  for (int nx = -n; nx <= n; nx++)
    for (int ny = -n; ny <= n; ny++)
      for (int nz = -n; nz <= n; nz++) {
        unsigned e = nx * nx + ny * ny + nz * nz;
        if (e <= emax) start[e + 1] += 2 * (uint64_t)m.tz_max;
      }
  for (unsigned e = 1; e <= emax; e++) start[e] += start[e - 1];
  m.stride = 5;
  m.qn.assign(nsp * 5, 0);
  for (int nx = -n; nx <= n; nx++)
    for (int ny = -n; ny <= n; ny++)
      for (int nz = -n; nz <= n; nz++) {
        unsigned e = nx * nx + ny * ny + nz * nz;
        if (e > emax) continue;
        for (int sz = -1; sz <= 1; sz += 2)
          for (int tz = -1; tz <= m.tz_max - 1; tz += 2) {
            int32_t *r = &m.qn[start[e]++ * 5];
            r[0] = nx; r[1] = ny; r[2] = nz; r[3] = sz; r[4] = tz;
          }
      }
  if (m.tz_max == 1) { m.chan_tz_max = -2; m.mod_chan_tz_max = 0; }
  else { m.chan_tz_max = 2; m.mod_chan_tz_max = 2; }
  uint64_t cn = 2 * (uint64_t)(2 * m.nmax) + 1;
  m.nchan = cn * cn * cn * (uint64_t)(3 * (2 + m.chan_tz_max / 2));
}

}  // namespace

struct ccdhost_system {
  Model m;
  double eref = 0, mbpt2 = 0;
  ccdgpu_problem prob;
  ccdgpu_model model;
  std::vector<double> eps;  // normal ordered
  std::vector<ccdgpu_channel_dims> dims, mdims;
  std::vector<ccdgpu_three_body_dims> tdims;
  std::vector<ccdgpu_pair> pp_all, hh_all, ph_all, hp_all, mpp_all, mhh_all, mhp_all, mph_all;
  std::vector<ccdgpu_channel_maps> maps, mmaps;
  std::vector<ccdgpu_triple> hpp_all, phh_all;
  std::vector<uint64_t> hpp_off_map, phh_off_map;  // start of each orbital's 3-body map
  std::vector<double> v[7];                         // hhhh, hhpp, pppp, hpph_mod, hphp_mod, h_hpp, phh_p
  std::vector<const double *> vptr[7];
  std::vector<ccdgpu_chain_index> tab[8];
  std::vector<const ccdgpu_chain_index *> tabptr[8];
};

namespace {

int finish(ccdhost_system *s, int32_t flags) {
  const bool vblocks = !(flags & CCDHOST_NO_V);
  const bool load_v_pppp = vblocks && (flags & CCDHOST_LOAD_V_PPPP);
  const bool tables = !(flags & CCDHOST_NO_TABLES);
  Model &m = s->m;
  const uint64_t nsp = m.nsp, np = m.np, nch = m.nchan;

  // E_ref with bare energies, then normal ordering (SPBasis.cpp:7-40).
  double eref = 0.;
  for (uint64_t i = 0; i < np; i++)
    for (uint64_t j = 0; j < np; j++) eref += 0.5 * m.tbme(i, j, i, j);
  for (uint64_t i = 0; i < np; i++) eref += m.eps[i];
  s->eref = eref;
  s->eps.resize(nsp);
  for (uint64_t p = 0; p < nsp; p++) {
    double e = m.eps[p];
    for (uint64_t j = 0; j < np; j++) e += m.tbme(p, j, p, j);
    s->eps[p] = e;
  }

  // Channels and their sorted maps (SPBasis.cpp:80-441), in the 1-rank first-fit-decreasing
  // order: on the device with CCDHOST_DEVICE_CHANNELS (ccdgpu_build_channels), else here.
  // pos[] = index of (p, q) inside its own list, chan[] = its permuted channel.
  const uint64_t npart = nsp - np;
  std::vector<uint32_t> pos(nsp * nsp), mpos(nsp * nsp), chan(nsp * nsp), mchan(nsp * nsp);
  s->dims.resize(nch);
  s->mdims.resize(nch);
  // List offsets of every channel from the (permuted) dimensions; the lists sized to match.
  std::vector<uint64_t> off_pp(nch + 1, 0), off_hh(nch + 1, 0), off_ph(nch + 1, 0),
      off_hp(nch + 1, 0);
  std::vector<uint64_t> moff_pp(nch + 1, 0), moff_hh(nch + 1, 0), moff_ph(nch + 1, 0),
      moff_hp(nch + 1, 0);
  auto set_offsets = [&]() {
    for (uint64_t c = 0; c < nch; c++) {
      off_pp[c + 1] = off_pp[c] + s->dims[c].pp; off_hh[c + 1] = off_hh[c] + s->dims[c].hh;
      off_ph[c + 1] = off_ph[c] + s->dims[c].ph; off_hp[c + 1] = off_hp[c] + s->dims[c].hp;
      moff_pp[c + 1] = moff_pp[c] + s->mdims[c].pp; moff_hh[c + 1] = moff_hh[c] + s->mdims[c].hh;
      moff_ph[c + 1] = moff_ph[c] + s->mdims[c].ph; moff_hp[c + 1] = moff_hp[c] + s->mdims[c].hp;
    }
    s->pp_all.resize(off_pp[nch]); s->hh_all.resize(off_hh[nch]);
    s->ph_all.resize(off_ph[nch]); s->hp_all.resize(off_hp[nch]);
    s->mpp_all.resize(moff_pp[nch]); s->mhh_all.resize(moff_hh[nch]);
    s->mph_all.resize(moff_ph[nch]); s->mhp_all.resize(moff_hp[nch]);
  };
  if (flags & CCDHOST_DEVICE_CHANNELS) {
    for (auto *v : {&s->pp_all, &s->mpp_all}) v->resize(npart * npart);
    for (auto *v : {&s->hh_all, &s->mhh_all}) v->resize(np * np);
    for (auto *v : {&s->hp_all, &s->mhp_all, &s->ph_all, &s->mph_all}) v->resize(np * npart);
    ccdgpu_channel_rule rule{};
    rule.kind = m.kind == kPairing ? CCDGPU_MODEL_PAIRING
                : m.kind == kInfMatter ? CCDGPU_MODEL_INF_MATTER
                                       : CCDGPU_MODEL_ELECTRON_GAS;
    rule.qn_stride = m.stride;
    rule.qn = m.qn.data();
    rule.n_sp = nsp; rule.n_particles = np; rule.n_channels = nch;
    rule.nmax = m.nmax; rule.chan_tz_max = m.chan_tz_max; rule.mod_chan_tz_max = m.mod_chan_tz_max;
    rule.device = -1;  // the calling thread's current CUDA device
    ccdgpu_pair *const dl[4] = {s->pp_all.data(), s->hh_all.data(), s->hp_all.data(), s->ph_all.data()};
    ccdgpu_pair *const dml[4] = {s->mpp_all.data(), s->mhh_all.data(), s->mhp_all.data(), s->mph_all.data()};
    const int rc = ccdgpu_build_channels(&rule, s->dims.data(), s->mdims.data(), dl, dml,
                                         chan.data(), mchan.data(), pos.data(), mpos.data());
    if (rc) return rc;
    set_offsets();
  } else {
    // Channel dimensions in unpermuted order (SPBasis.cpp:80-179).
    std::vector<ccdgpu_channel_dims> d0(nch, ccdgpu_channel_dims{0, 0, 0, 0}), md0 = d0;
    std::vector<uint32_t> c0(nsp * nsp), mc0(nsp * nsp);
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int64_t p = 0; p < (int64_t)nsp; p++)
      for (uint64_t q = 0; q < nsp; q++) {
        const uint64_t c = m.chan0(p, q), mc = m.mod0(p, q);
        if (c >= nch || mc >= nch) {
          bad = 1;
          continue;
        }
        c0[p * nsp + q] = (uint32_t)c;
        mc0[p * nsp + q] = (uint32_t)mc;
      }
    if (bad) return CCDGPU_ERR_INVALID_ARGUMENT;
    for (uint64_t p = 0; p < nsp; p++)
      for (uint64_t q = 0; q < nsp; q++) {
        const uint64_t c = c0[p * nsp + q], mc = mc0[p * nsp + q];
        bool ph = p < np, qh = q < np;
        if (ph && qh) { d0[c].hh++; md0[mc].hh++; }
        else if (ph) { d0[c].hp++; md0[mc].hp++; }
        else if (qh) { d0[c].ph++; md0[mc].ph++; }
        else { d0[c].pp++; md0[mc].pp++; }
      }

    // 1-rank first-fit-decreasing order (shared with the device construction).
    const std::vector<uint64_t> order = ffd_channel_order(d0);
    std::vector<uint32_t> inv(nch);
    for (uint64_t i = 0; i < nch; i++) {
      inv[order[i]] = (uint32_t)i;
      s->dims[i] = d0[order[i]];
      s->mdims[i] = md0[order[i]];
    }

    set_offsets();
    // Kind of a pair: 0 pp, 1 hh, 2 hp, 3 ph.  The lists are filled in parallel over contiguous
    // ranges of p: pass 1 counts each range's pairs per (channel, kind), exclusive sums over the
    // ranges give each range its start inside every list, pass 2 places the pairs.  Ranges in
    // ascending p keep every list in (p, q) order, as the sequential scan would.
    auto kind_of = [&](uint64_t p, uint64_t q) { return p < np ? (q < np ? 1 : 2) : (q < np ? 3 : 0); };
    ccdgpu_pair *lists[4] = {s->pp_all.data(), s->hh_all.data(), s->hp_all.data(), s->ph_all.data()};
    ccdgpu_pair *mlists[4] = {s->mpp_all.data(), s->mhh_all.data(), s->mhp_all.data(), s->mph_all.data()};
    const uint64_t *offs[4] = {off_pp.data(), off_hh.data(), off_hp.data(), off_ph.data()};
    const uint64_t *moffs[4] = {moff_pp.data(), moff_hh.data(), moff_hp.data(), moff_ph.data()};
    const int nrange = (int)std::max<uint64_t>(1, std::min<uint64_t>(nsp, omp_get_max_threads()));
    std::vector<uint32_t> cnt((size_t)nrange * nch * 4, 0), mcnt((size_t)nrange * nch * 4, 0);
    auto p_begin = [&](int r) { return nsp * (uint64_t)r / (uint64_t)nrange; };
#pragma omp parallel for schedule(static)
    for (int r = 0; r < nrange; r++) {
      uint32_t *ct = &cnt[(size_t)r * nch * 4], *mct = &mcnt[(size_t)r * nch * 4];
      for (uint64_t p = p_begin(r); p < p_begin(r + 1); p++)
        for (uint64_t q = 0; q < nsp; q++) {
          const int k = kind_of(p, q);
          ct[inv[c0[p * nsp + q]] * 4 + k]++;
          mct[inv[mc0[p * nsp + q]] * 4 + k]++;
        }
    }
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < (int64_t)(nch * 4); e++) {
      uint32_t a = 0, b = 0;
      for (int r = 0; r < nrange; r++) {
        const uint32_t x = cnt[(size_t)r * nch * 4 + e], y = mcnt[(size_t)r * nch * 4 + e];
        cnt[(size_t)r * nch * 4 + e] = a;
        mcnt[(size_t)r * nch * 4 + e] = b;
        a += x;
        b += y;
      }
    }
#pragma omp parallel for schedule(static)
    for (int r = 0; r < nrange; r++) {
      uint32_t *ct = &cnt[(size_t)r * nch * 4], *mct = &mcnt[(size_t)r * nch * 4];
      for (uint64_t p = p_begin(r); p < p_begin(r + 1); p++)
        for (uint64_t q = 0; q < nsp; q++) {
          const uint64_t c = inv[c0[p * nsp + q]], mc = inv[mc0[p * nsp + q]];
          const int kd = kind_of(p, q);
          const uint32_t k = ct[c * 4 + kd]++, mk = mct[mc * 4 + kd]++;
          lists[kd][offs[kd][c] + k] = ccdgpu_pair{p, q};
          mlists[kd][moffs[kd][mc] + mk] = ccdgpu_pair{p, q};
          chan[p * nsp + q] = (uint32_t)c;
          mchan[p * nsp + q] = (uint32_t)mc;
          pos[p * nsp + q] = k;
          mpos[p * nsp + q] = mk;
        }
    }
  }
  s->maps.resize(nch);
  s->mmaps.resize(nch);
  for (uint64_t c = 0; c < nch; c++) {
    s->maps[c] = {s->pp_all.data() + off_pp[c], s->hh_all.data() + off_hh[c],
                  s->hp_all.data() + off_hp[c], s->ph_all.data() + off_ph[c]};
    s->mmaps[c] = {s->mpp_all.data() + moff_pp[c], s->mhh_all.data() + moff_hh[c],
                   s->mhp_all.data() + moff_hp[c], s->mph_all.data() + moff_ph[c]};
  }

  // Three-body maps (SPBasis.cpp:181-256, 443-563): hpp(k) = {(j,a,b): (a,b) in pp(ch(k,j))},
  // phh(a) = {(b,i,j): (i,j) in hh(ch(a,b))}, both sorted lexicographically.
  s->tdims.assign(nsp, ccdgpu_three_body_dims{0, 0});
  // Block offsets inside hpp(k) / phh(a), kept for the remap tables.
  std::vector<uint64_t> hpp_blk(np * np), phh_blk(tables ? (nsp - np) * (nsp - np) : 0);
  s->hpp_off_map.assign(np + 1, 0);
  for (uint64_t k = 0; k < np; k++) {
    uint64_t n = 0;
    for (uint64_t j = 0; j < np; j++) {
      hpp_blk[k * np + j] = n;
      n += s->dims[chan[k * nsp + j]].pp;
    }
    s->tdims[k].hpp = n;
    s->hpp_off_map[k + 1] = s->hpp_off_map[k] + n;
  }
  s->phh_off_map.assign(npart + 1, 0);
  for (uint64_t a = np; a < nsp; a++) {
    uint64_t n = 0;
    for (uint64_t b = np; b < nsp; b++) {
      if (tables) phh_blk[(a - np) * npart + (b - np)] = n;
      n += s->dims[chan[a * nsp + b]].hh;
    }
    s->tdims[a].phh = n;
    s->phh_off_map[a - np + 1] = s->phh_off_map[a - np] + n;
  }
  s->hpp_all.resize(s->hpp_off_map[np]);
  s->phh_all.resize(s->phh_off_map[npart]);
#pragma omp parallel for schedule(dynamic)
  for (int64_t k = 0; k < (int64_t)np; k++) {
    uint64_t w = s->hpp_off_map[k];
    for (uint64_t j = 0; j < np; j++) {
      uint64_t c = chan[k * nsp + j];
      for (uint64_t t = 0; t < s->dims[c].pp; t++)
        s->hpp_all[w++] = ccdgpu_triple{j, s->maps[c].pp[t].p, s->maps[c].pp[t].q};
    }
  }
#pragma omp parallel for schedule(dynamic)
  for (int64_t a = (int64_t)np; a < (int64_t)nsp; a++) {
    uint64_t w = s->phh_off_map[a - np];
    for (uint64_t b = np; b < nsp; b++) {
      uint64_t c = chan[a * nsp + b];
      for (uint64_t t = 0; t < s->dims[c].hh; t++)
        s->phh_all[w++] = ccdgpu_triple{b, s->maps[c].hh[t].p, s->maps[c].hh[t].q};
    }
  }

  // V blocks for amplitude-carrying channels (load.cpp:112-318); none with CCDHOST_NO_V (the
  // solver library then generates them on the device from the model).
  auto active = [&](uint64_t c) { return vblocks && s->dims[c].pp && s->dims[c].hh; };
  auto mactive = [&](uint64_t c) { return vblocks && s->mdims[c].ph && s->mdims[c].hp; };
  std::vector<uint64_t> o_hhhh(nch + 1, 0), o_hhpp(nch + 1, 0), o_pppp(nch + 1, 0),
      o_hpph(nch + 1, 0), o_hphp(nch + 1, 0);
  for (uint64_t c = 0; c < nch; c++) {
    uint64_t pp = s->dims[c].pp, hh = s->dims[c].hh, ph = s->mdims[c].ph, hp = s->mdims[c].hp;
    bool a = active(c), ma = mactive(c);
    o_hhhh[c + 1] = o_hhhh[c] + (a ? hh * hh : 0);
    o_hhpp[c + 1] = o_hhpp[c] + (a ? hh * pp : 0);
    o_pppp[c + 1] = o_pppp[c] + ((a && load_v_pppp) ? pp * pp : 0);
    o_hpph[c + 1] = o_hpph[c] + (ma ? hp * ph : 0);
    o_hphp[c + 1] = o_hphp[c] + (ma ? hp * hp : 0);
  }
  try {
    s->v[0].resize(o_hhhh[nch]); s->v[1].resize(o_hhpp[nch]); s->v[2].resize(o_pppp[nch]);
    s->v[3].resize(o_hpph[nch]); s->v[4].resize(o_hphp[nch]);
    s->v[5].resize(vblocks ? s->hpp_off_map[np] : 0);
    s->v[6].resize(vblocks ? s->phh_off_map[npart] : 0);
  } catch (const std::bad_alloc &) {
    return CCDGPU_ERR_OUT_OF_MEMORY;
  }
  for (int k = 0; k < 5; k++) s->vptr[k].assign(nch, nullptr);
  s->vptr[5].assign(np, nullptr);
  s->vptr[6].assign(npart, nullptr);
#pragma omp parallel for schedule(dynamic)
  for (int64_t ci = 0; ci < (int64_t)nch; ci++) {
    const uint64_t c = ci;
    const uint64_t pp = s->dims[c].pp, hh = s->dims[c].hh;
    const ccdgpu_pair *P = s->maps[c].pp, *H = s->maps[c].hh;
    if (active(c)) {
      double *vh = &s->v[0][o_hhhh[c]], *vx = &s->v[1][o_hhpp[c]];
      for (uint64_t x = 0; x < hh; x++) {
        for (uint64_t y = 0; y < hh; y++) vh[x * hh + y] = s->m.tbme(H[x].p, H[x].q, H[y].p, H[y].q);
        for (uint64_t y = 0; y < pp; y++) vx[x * pp + y] = s->m.tbme(H[x].p, H[x].q, P[y].p, P[y].q);
      }
      if (load_v_pppp) {
        double *vp = &s->v[2][o_pppp[c]];
        for (uint64_t x = 0; x < pp; x++)
          for (uint64_t y = 0; y < pp; y++) vp[x * pp + y] = s->m.tbme(P[x].p, P[x].q, P[y].p, P[y].q);
      }
    }
    if (mactive(c)) {
      const uint64_t ph = s->mdims[c].ph, hp = s->mdims[c].hp;
      const ccdgpu_pair *PH = s->mmaps[c].ph, *HP = s->mmaps[c].hp;
      double *va = &s->v[3][o_hpph[c]], *vb = &s->v[4][o_hphp[c]];
      for (uint64_t x = 0; x < hp; x++) {
        // vnn_hhpp_hpph_mod[(i,a),(b,j)] = <ij|v|ab>   (load.cpp:284-293)
        for (uint64_t y = 0; y < ph; y++) va[x * ph + y] = s->m.tbme(HP[x].p, PH[y].q, HP[x].q, PH[y].p);
        // vnn_hpph_hphp_mod[(i,b),(j,a)] = <ia|v|bj>   (load.cpp:306-315)
        for (uint64_t y = 0; y < hp; y++) vb[x * hp + y] = s->m.tbme(HP[x].p, HP[y].q, HP[x].q, HP[y].p);
      }
    }
  }
  for (uint64_t c = 0; c < nch; c++) {
    if (active(c)) {
      s->vptr[0][c] = &s->v[0][o_hhhh[c]];
      s->vptr[1][c] = &s->v[1][o_hhpp[c]];
      if (load_v_pppp) s->vptr[2][c] = &s->v[2][o_pppp[c]];
    }
    if (mactive(c)) {
      s->vptr[3][c] = &s->v[3][o_hpph[c]];
      s->vptr[4][c] = &s->v[4][o_hphp[c]];
    }
  }
#pragma omp parallel for schedule(dynamic)
  for (int64_t k = 0; k < (vblocks ? (int64_t)np : 0); k++)  // vnn_h_hpp[k][(j,a,b)] = <kj|v|ab> (load.cpp:258-273)
    for (uint64_t t = s->hpp_off_map[k]; t < s->hpp_off_map[k + 1]; t++)
      s->v[5][t] = s->m.tbme(k, s->hpp_all[t].p, s->hpp_all[t].q, s->hpp_all[t].r);
#pragma omp parallel for schedule(dynamic)
  for (int64_t a = 0; a < (vblocks ? (int64_t)npart : 0); a++)  // vnn_phh_p[a][(b,i,j)] = <ij|v|ab> (load.cpp:241-256)
    for (uint64_t t = s->phh_off_map[a]; t < s->phh_off_map[a + 1]; t++)
      s->v[6][t] = s->m.tbme(s->phh_all[t].q, s->phh_all[t].r, a + np, s->phh_all[t].p);
  for (uint64_t k = 0; k < np && vblocks; k++)
    if (s->tdims[k].hpp) s->vptr[5][k] = &s->v[5][s->hpp_off_map[k]];
  for (uint64_t a = 0; a < npart && vblocks; a++)
    if (s->tdims[a + np].phh) s->vptr[6][a] = &s->v[6][s->phh_off_map[a]];

  // Remap tables (load.cpp:469-526), from block offsets instead of hash tables; skipped with
  // CCDHOST_NO_TABLES (the solver library then derives them on the device).
  std::vector<uint64_t> o_t(nch + 1, 0);
  for (uint64_t c = 0; c < nch; c++) o_t[c + 1] = o_t[c] + s->dims[c].pp * s->dims[c].hh;
  for (int k = 0; k < 8; k++) {
    s->tab[k].resize(tables ? o_t[nch] : 0);
    s->tabptr[k].assign(nch, nullptr);
  }
#pragma omp parallel for schedule(dynamic)
  for (int64_t ci = 0; ci < (tables ? (int64_t)nch : 0); ci++) {
    const uint64_t c = ci, pp = s->dims[c].pp, hh = s->dims[c].hh;
    for (uint64_t AB = 0; AB < pp; AB++)
      for (uint64_t IJ = 0; IJ < hh; IJ++) {
        const uint64_t a = s->maps[c].pp[AB].p, b = s->maps[c].pp[AB].q;
        const uint64_t i = s->maps[c].hh[IJ].p, j = s->maps[c].hh[IJ].q;
        const uint64_t e = o_t[c] + AB * hh + IJ;
        s->tab[0][e] = {j, hpp_blk[j * np + i] + AB, 0};
        s->tab[1][e] = {i, hpp_blk[i * np + j] + AB, 0};
        s->tab[2][e] = {a - np, 0, phh_blk[(a - np) * npart + (b - np)] + IJ};
        s->tab[3][e] = {b - np, 0, phh_blk[(b - np) * npart + (a - np)] + IJ};
        s->tab[4][e] = {mchan[a * nsp + i], mpos[a * nsp + i], mpos[j * nsp + b]};
        s->tab[5][e] = {mchan[a * nsp + j], mpos[a * nsp + j], mpos[i * nsp + b]};
        s->tab[6][e] = {mchan[b * nsp + i], mpos[b * nsp + i], mpos[j * nsp + a]};
        s->tab[7][e] = {mchan[b * nsp + j], mpos[b * nsp + j], mpos[i * nsp + a]};
      }
  }
  for (int k = 0; k < 8 && tables; k++)
    for (uint64_t c = 0; c < nch; c++)
      if (o_t[c + 1] > o_t[c]) s->tabptr[k][c] = &s->tab[k][o_t[c]];

  // MBPT2 (MBPT2Corr.cpp:6-38), normal-ordered energies: each channel's sum as the reference
  // forms it (in parallel over channels), then the channel sums added in channel order.
  std::vector<double> corr_c(nch, 0.0);
#pragma omp parallel for schedule(dynamic)
  for (int64_t ci = 0; ci < (int64_t)nch; ci++) {
    const uint64_t c = ci;
    if (!s->dims[c].pp || !s->dims[c].hh) continue;
    const uint64_t pp = s->dims[c].pp, hh = s->dims[c].hh;
    const double *vx = s->vptr[1][c];  // NULL with CCDHOST_NO_V: the same elements, evaluated
    double corr = 0.;
    for (uint64_t x = 0; x < hh; x++)
      for (uint64_t y = 0; y < pp; y++) {
        const ccdgpu_pair H = s->maps[c].hh[x], P = s->maps[c].pp[y];
        double den = s->eps[H.p] + s->eps[H.q] - s->eps[P.p] - s->eps[P.q];
        double v = vx ? vx[x * pp + y] : s->m.tbme(H.p, H.q, P.p, P.q);
        corr += v * v / den;
      }
    corr_c[c] = corr;
  }
  double e2 = 0.;
  for (uint64_t c = 0; c < nch; c++)
    if (s->dims[c].pp && s->dims[c].hh) e2 += 0.25 * corr_c[c];
  s->mbpt2 = e2;

  // Model description for on-the-fly V.
  s->model.kind = m.kind == kPairing ? CCDGPU_MODEL_PAIRING
                  : m.kind == kInfMatter ? CCDGPU_MODEL_INF_MATTER
                                         : CCDGPU_MODEL_ELECTRON_GAS;
  s->model.qn_stride = m.stride;
  s->model.qn = m.qn.data();
  for (double &p : s->model.params) p = 0;
  if (m.kind == kElectronGas) { s->model.params[0] = m.L; s->model.params[1] = m.e_sq; }
  if (m.kind == kInfMatter) { s->model.params[0] = pow(np / m.density, 1. / 3.); s->model.params[1] = m.density; }
  if (m.kind == kPairing) { s->model.params[0] = m.g; }

  ccdgpu_problem &P = s->prob;
  std::memset(&P, 0, sizeof(P));
  P.n_sp = nsp; P.n_particles = np; P.n_channels = nch;
  P.sp_energy = s->eps.data();
  P.chan_dims = s->dims.data(); P.chan_mod_dims = s->mdims.data();
  P.chan_maps = s->maps.data(); P.chan_mod_maps = s->mmaps.data();
  P.three_body_dims = s->tdims.data();
  P.v_hhhh = vblocks ? s->vptr[0].data() : nullptr;
  P.v_hhpp = vblocks ? s->vptr[1].data() : nullptr;
  P.v_pppp = load_v_pppp ? s->vptr[2].data() : nullptr;
  P.v_hpph_mod = vblocks ? s->vptr[3].data() : nullptr;
  P.v_hphp_mod = vblocks ? s->vptr[4].data() : nullptr;
  P.v_h_hpp = vblocks ? s->vptr[5].data() : nullptr;
  P.v_phh_p = vblocks ? s->vptr[6].data() : nullptr;
  for (int k = 0; k < 8; k++) P.maps[k] = tables ? s->tabptr[k].data() : nullptr;
  P.model = &s->model;
  return CCDGPU_OK;
}

}  // namespace

extern "C" {

int ccdhost_build_pairing(double xi, double g, uint64_t n_pair_states, uint64_t n_particles,
                          int32_t flags, ccdhost_system **out) {
  if (!out || n_pair_states == 0 || n_particles == 0 || n_particles >= 2 * n_pair_states)
    return CCDGPU_ERR_INVALID_ARGUMENT;
  ccdhost_system *s = new (std::nothrow) ccdhost_system();
  if (!s) return CCDGPU_ERR_OUT_OF_MEMORY;
  Model &m = s->m;
  m.kind = kPairing;
  m.xi = xi; m.g = g;
  m.nsp = 2 * n_pair_states; m.np = n_particles; m.nchan = 3; m.stride = 2;
  m.qn.resize(m.nsp * 2);
  for (uint64_t i = 0; i < n_pair_states; i++) {  // PairingSPBasis.cpp:27-44
    m.qn[(2 * i) * 2] = (int32_t)(i + 1); m.qn[(2 * i) * 2 + 1] = +1;
    m.qn[(2 * i + 1) * 2] = (int32_t)(i + 1); m.qn[(2 * i + 1) * 2 + 1] = -1;
  }
  m.eps.resize(m.nsp);
  for (uint64_t i = 0; i < m.nsp; i++) m.eps[i] = (m.qn[i * 2] - 1.0) * xi;
  int rc = finish(s, flags);
  if (rc) { delete s; return rc; }
  *out = s;
  return CCDGPU_OK;
}

int ccdhost_build_inf_matter(double density, int32_t tz_max, uint64_t n_shells,
                             uint64_t n_particle_shells, int32_t flags,
                             ccdhost_system **out) {
  if (!out || density <= 0 || (tz_max != 1 && tz_max != 2) || n_shells == 0 ||
      n_particle_shells == 0 || n_particle_shells >= n_shells)
    return CCDGPU_ERR_INVALID_ARGUMENT;
  ccdhost_system *s = new (std::nothrow) ccdhost_system();
  if (!s) return CCDGPU_ERR_OUT_OF_MEMORY;
  Model &m = s->m;
  m.kind = kInfMatter;
  m.density = density;
  m.tz_max = tz_max;
  plane_wave_orbitals(m, n_shells, n_particle_shells);
  // InfMatterSPBasis.cpp:165-184 (neutron mass for both species, as the reference does).
  const double hbarc = 197.3269788, massc2 = 939.565;
  double prefactor = hbarc * hbarc / (2. * massc2);
  double box = pow(m.np / density, 1. / 3.);
  m.L = box;
  m.eps.resize(m.nsp);
  for (uint64_t i = 0; i < m.nsp; i++) {
    const int32_t *r = m.q(i);
    m.eps[i] = (prefactor * 4 * M_PI * M_PI / (box * box)) * (r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
  }
  int rc = finish(s, flags);
  if (rc) { delete s; return rc; }
  *out = s;
  return CCDGPU_OK;
}

int ccdhost_build_electron_gas(double r_s, uint64_t n_shells, uint64_t n_particle_shells,
                               int32_t flags, ccdhost_system **out) {
  if (!out || r_s <= 0 || n_shells == 0 || n_particle_shells == 0 ||
      n_particle_shells >= n_shells)
    return CCDGPU_ERR_INVALID_ARGUMENT;
  ccdhost_system *s = new (std::nothrow) ccdhost_system();
  if (!s) return CCDGPU_ERR_OUT_OF_MEMORY;
  Model &m = s->m;
  m.kind = kElectronGas;
  m.tz_max = 1;  // one species (ElectronGasSPBasis.cpp:19)
  plane_wave_orbitals(m, n_shells, n_particle_shells);
  // Hartree atomic units from the same constants (ElectronGasSPBasis.cpp:173-210).
  double hbarc = 0.1973269788;
  const double ev_per_hartree = 27.21138505;
  hbarc = hbarc * 10000 / ev_per_hartree;
  double massc2 = 0.5109989461;
  massc2 = massc2 * 1000000 / ev_per_hartree;
  const double fine = 1.0 / 137.035999139;
  double r_bohr = hbarc / (massc2 * fine);
  double r_0 = r_s * r_bohr;
  double prefactor = hbarc * hbarc / (2. * massc2);
  m.L = pow((4. / 3.) * M_PI * m.np, 1. / 3.) * r_0;
  m.e_sq = fine * hbarc;
  m.eps.resize(m.nsp);
  for (uint64_t i = 0; i < m.nsp; i++) {
    const int32_t *r = m.q(i);
    m.eps[i] = (prefactor * 4 * M_PI * M_PI / (m.L * m.L)) * (r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
  }
  int rc = finish(s, flags);
  if (rc) { delete s; return rc; }
  *out = s;
  return CCDGPU_OK;
}

void ccdhost_free(ccdhost_system *s) { delete s; }

const ccdgpu_problem *ccdhost_problem(const ccdhost_system *s) { return s ? &s->prob : nullptr; }
double ccdhost_reference_energy(const ccdhost_system *s) { return s ? s->eref : 0.0; }
double ccdhost_mbpt2(const ccdhost_system *s) { return s ? s->mbpt2 : 0.0; }

int ccdhost_array(const ccdhost_system *cs, const char *name, const void **data,
                  uint64_t *count, int32_t *dtype) {
  if (!cs || !name || !data || !count || !dtype) return CCDGPU_ERR_INVALID_ARGUMENT;
  ccdhost_system *s = const_cast<ccdhost_system *>(cs);
  std::string n(name);
  static const char *vnames[7] = {"v_hhhh", "v_hhpp", "v_pppp", "v_hpph_mod", "v_hphp_mod",
                                  "v_h_hpp", "v_phh_p"};
  for (int k = 0; k < 7; k++)
    if (n == vnames[k]) {
      *data = s->v[k].data(); *count = s->v[k].size(); *dtype = 1;
      return CCDGPU_OK;
    }
  if (n == "sp_energy") {
    *data = s->eps.data(); *count = s->eps.size(); *dtype = 1;
    return CCDGPU_OK;
  }
  if (n == "sp_energy_bare") {
    *data = s->m.eps.data(); *count = s->m.eps.size(); *dtype = 1;
    return CCDGPU_OK;
  }
  static const char *tnames[8] = {"map_iab_j", "map_jab_i", "map_a_bij", "map_b_aij",
                                  "map_ai_jb", "map_aj_ib", "map_bi_ja", "map_bj_ia"};
  for (int k = 0; k < 8; k++)
    if (n == tnames[k]) {
      *data = s->tab[k].data(); *count = s->tab[k].size() * 3; *dtype = 2;
      return CCDGPU_OK;
    }
  auto pairs = [&](const std::vector<ccdgpu_pair> &v) {
    *data = v.data(); *count = v.size() * 2; *dtype = 2;
    return CCDGPU_OK;
  };
  if (n == "pp_map") return pairs(s->pp_all);
  if (n == "hh_map") return pairs(s->hh_all);
  if (n == "ph_mod_map") return pairs(s->mph_all);
  if (n == "hp_mod_map") return pairs(s->mhp_all);
  if (n == "hpp_map") { *data = s->hpp_all.data(); *count = s->hpp_all.size() * 3; *dtype = 2; return CCDGPU_OK; }
  if (n == "phh_map") { *data = s->phh_all.data(); *count = s->phh_all.size() * 3; *dtype = 2; return CCDGPU_OK; }
  if (n == "chan_dims") { *data = s->dims.data(); *count = s->dims.size() * 4; *dtype = 2; return CCDGPU_OK; }
  if (n == "chan_mod_dims") { *data = s->mdims.data(); *count = s->mdims.size() * 4; *dtype = 2; return CCDGPU_OK; }
  if (n == "three_body_dims") { *data = s->tdims.data(); *count = s->tdims.size() * 2; *dtype = 2; return CCDGPU_OK; }
  if (n == "qn") {
    *data = s->m.qn.data(); *count = s->m.qn.size(); *dtype = 4;
    return CCDGPU_OK;
  }
  return CCDGPU_ERR_INVALID_ARGUMENT;
}

}  // extern "C"
