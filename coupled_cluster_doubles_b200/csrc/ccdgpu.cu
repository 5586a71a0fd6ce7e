// ccdgpu — C ABI implementation (include/ccdgpu.h).
//
// A handle holds the whole CCD state of one system in device memory, laid out for the
// kernels in ccd_kernels.cuh:
//   * amplitudes in the reference t2_pphh layout (two buffers, ping-pong by a device-side
//     parity bit), plus the ladder operand tiles of T (T^T for V_pppp T, row tiles for T X);
//   * V_pppp pre-tiled into the swizzled shared-memory image of the pp-ladder kernel;
//   * V_hhpp transposed to pp x hh so that it streams aligned with T;
//   * the loadMaps tables as int32 flat offsets into the target slabs, validated at create;
//   * a Control block with the solve loop's state (energy history, stop rule, parity), so a
//     captured iteration graph can be replayed without host synchronisation.
#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "ccd_device.cuh"
#include "ccd_kernels.cuh"
#include "ccdgpu.h"

using namespace ccd;

namespace {

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

}  // namespace

struct ccdgpu_handle {
  ccdgpu_options opt{};
  cudaStream_t s0 = nullptr, s1 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaEvent_t ev[10] = {};
  uint64_t nch = 0, nsp = 0, np = 0, npart = 0;
  int64_t n_t = 0, n_m = 0, n_h = 0, n_p = 0;
  int n_act = 0, n_mod = 0, n_mod_small = 0, n_tiles = 0, n_tiles_narrow = 0, n_hh_tiles = 0,
      n_ranges = 0;
  size_t ladder_smem = 0, ring_smem = 0, hh_smem = 0;
  bool have_3body = false;
  std::vector<DevBuf> allocs;

  ChanInfo *chans = nullptr;
  ModInfo *mods = nullptr;        // small channels first (n_mod_small), then the others
  LadderTile *tiles = nullptr;
  HHTile *hh_tiles = nullptr;
  int32_t *rowmap = nullptr, *mirror = nullptr, *counters = nullptr;
  int2 *pk_idx = nullptr;
  double *part = nullptr;
  ElemRange *ranges = nullptr;
  int2 *pp_pairs = nullptr, *hh_pairs = nullptr;
  int32_t *pp_swap = nullptr, *hh_swap = nullptr;
  int64_t *list_off = nullptr;
  int32_t *list = nullptr;
  double *eps = nullptr, *v_pphh = nullptr, *v_hhhh = nullptr, *v_t = nullptr;
  double *v_hpph = nullptr, *v_hphp = nullptr;
  double *t[2] = {nullptr, nullptr}, *dmat = nullptr, *old_phhp = nullptr, *r_phhp = nullptr;
  double *x = nullptr, *x_t = nullptr, *t_kt = nullptr, *t_mt = nullptr;
  double *s = nullptr, *r = nullptr, *xh = nullptr, *yp = nullptr, *epart = nullptr;
  int32_t *flat = nullptr;
  int64_t *o_h = nullptr, *o_p = nullptr;
  double *v_h_hpp = nullptr, *v_phh_p = nullptr;
  double *old_h1pp_h2 = nullptr, *old_h2pp_h1 = nullptr, *diff_h2pp_h1 = nullptr;
  double *old_p1_p2hh = nullptr, *old_p2_p1hh = nullptr, *diff_p2_p1hh = nullptr;
  double *gath = nullptr;
  Control *ctl = nullptr;
  Control *h_ctl = nullptr;  // pinned mirror
  double *e_out = nullptr;
  int32_t *err = nullptr;

  cudaGraphExec_t graph = nullptr;
  int64_t kernels_per_graph = 0;
  bool profiling = false;
  ccdgpu_profile prof{};
  double flops = 0, v_bytes = 0, ladder_flops = 0;
  int64_t launches = 0;
};

namespace {

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return CCDGPU_OK;
  if (e == cudaErrorMemoryAllocation) return CCDGPU_ERR_OUT_OF_MEMORY;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return CCDGPU_ERR_NO_DEVICE;
  return CCDGPU_ERR_CUDA;
}

#define CK(call)                              \
  do {                                        \
    cudaError_t e_ = (call);                  \
    if (e_ != cudaSuccess) {                  \
      (void)cudaGetLastError();               \
      return cuda_status(e_);                 \
    }                                         \
  } while (0)

template <typename T>
int dalloc(ccdgpu_handle *h, T **p, size_t count, bool zero = true) {
  size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
  void *q = nullptr;
  CK(cudaMalloc(&q, bytes));
  h->allocs.push_back({q, bytes});
  if (zero) CK(cudaMemsetAsync(q, 0, bytes, h->s0));
  *p = static_cast<T *>(q);
  return CCDGPU_OK;
}
template <typename T>
int upload(ccdgpu_handle *h, T **p, const std::vector<T> &v) {
  int rc = dalloc(h, p, v.size(), false);
  if (rc) return rc;
  if (!v.empty()) CK(cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return CCDGPU_OK;
}

int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

int find_pair(const ccdgpu_pair *list, int64_t n, uint64_t p, uint64_t q) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = (lo + hi) / 2;
    if (list[mid].p < p || (list[mid].p == p && list[mid].q < q)) lo = mid + 1;
    else hi = mid;
  }
  if (lo < n && list[lo].p == p && list[lo].q == q) return (int)lo;
  return -1;
}

void release(ccdgpu_handle *h) {
  if (!h) return;
  if (h->graph) cudaGraphExecDestroy(h->graph);
  for (auto &b : h->allocs) cudaFree(b.p);
  h->allocs.clear();
  if (h->h_ctl) cudaFreeHost(h->h_ctl);
  for (auto &e : h->ev)
    if (e) cudaEventDestroy(e);
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_join) cudaEventDestroy(h->ev_join);
  if (h->s1) cudaStreamDestroy(h->s1);
  if (h->s0) cudaStreamDestroy(h->s0);
}

int build(ccdgpu_handle *h, const ccdgpu_problem *P) {
  const uint64_t nch = P->n_channels, nsp = P->n_sp, np = P->n_particles;
  h->nch = nch; h->nsp = nsp; h->np = np; h->npart = nsp - np;
  const ccdgpu_channel_dims *D = P->chan_dims, *MD = P->chan_mod_dims;

  // Regular channels carrying amplitudes, in channel order.
  std::vector<int64_t> o_t(nch + 1, 0), o_m(nch + 1, 0);
  for (uint64_t c = 0; c < nch; c++) {
    o_t[c + 1] = o_t[c] + (int64_t)(D[c].pp * D[c].hh);
    o_m[c + 1] = o_m[c] + (int64_t)(MD[c].ph * MD[c].hp);
  }
  h->n_t = o_t[nch];
  h->n_m = o_m[nch];
  if (h->n_t != h->n_m) return CCDGPU_ERR_BAD_TABLE;  // pphh <-> phhp must be a bijection
  if (h->n_t >= (int64_t)INT32_MAX) return CCDGPU_ERR_UNSUPPORTED;

  std::vector<ChanInfo> chans;
  std::vector<int64_t> act_of(nch, -1);
  // Packed rows (a<=b) and K pairs (c<d) per channel, from the sorted pp map.
  std::vector<int32_t> rowmap, mirror;
  std::vector<int2> pk_idx;
  std::vector<HHTile> hh_tiles;
  int64_t pp_tot = 0, hh_tot = 0, x_tot = 0, tkt = 0, tmt = 0, xt = 0, vt = 0, part_tot = 0;
  for (uint64_t c = 0; c < nch; c++) {
    const int64_t pp = D[c].pp, hh = D[c].hh;
    if (!pp || !hh) continue;
    if (hh > 8 * kMaxCG || pp > (1 << 20)) return CCDGPU_ERR_UNSUPPORTED;
    const ccdgpu_pair *pm = P->chan_maps[c].pp;
    if (!pm || !P->chan_maps[c].hh) return CCDGPU_ERR_INVALID_ARGUMENT;
    ChanInfo ci{};
    ci.pp = (int)pp; ci.hh = (int)hh;
    ci.cg = (int)ceil_div(hh, 8);
    ci.bm = ladder_bm(ci.cg);
    ci.row_off = (int64_t)rowmap.size();
    int pr = 0, pk = 0;
    for (int k = 0; k < ci.pp; k++) {
      int2 q = make_int2(-1, -1);
      if (pm[k].p < pm[k].q) q.x = pk++;
      if (pm[k].p <= pm[k].q) {
        q.y = pr++;
        rowmap.push_back(k);
        int mir = -1;
        if (pm[k].p < pm[k].q) {
          mir = find_pair(pm, ci.pp, pm[k].q, pm[k].p);
          if (mir < 0) return CCDGPU_ERR_BAD_TABLE;
        }
        mirror.push_back(mir);
      }
      pk_idx.push_back(q);
    }
    ci.pr = pr; ci.pk = pk;
    ci.nkc = (int)ceil_div(pk, kBK);
    ci.nkh = (int)ceil_div(hh, kBK);
    ci.nmt = (int)ceil_div(pr, ci.bm);
    ci.nhht = (int)ceil_div(pp, kHHRows);
    ci.t_off = o_t[c];
    ci.pp_off = pp_tot; ci.hh_off = hh_tot; ci.x_off = x_tot;
    ci.tkt_base = tkt; ci.tmt_base = tmt; ci.xt_base = xt; ci.vkt_base = vt;
    ci.part_off = part_tot;
    ci.hht0 = (int64_t)hh_tiles.size();
    const int nb = 8 * ci.cg;
    pp_tot += pp; hh_tot += hh; x_tot += hh * hh;
    tkt += (int64_t)ci.nkc * kBK * nb;
    tmt += (int64_t)ci.nmt * ci.nkh * ci.bm * kBK;
    xt += (int64_t)ci.nkh * kBK * nb;
    vt += (int64_t)ci.nmt * ci.nkc * ci.bm * kBK;
    part_tot += (int64_t)ci.nhht * hh * hh;
    act_of[c] = (int64_t)chans.size();
    for (int t = 0; t < ci.nhht; t++) hh_tiles.push_back({(int32_t)chans.size(), t * kHHRows, t, 0});
    chans.push_back(ci);
  }
  h->n_act = (int)chans.size();
  h->n_hh_tiles = (int)hh_tiles.size();

  // Pair tables, swaps and one-body segment lists.
  std::vector<int2> pp_pairs(pp_tot), hh_pairs(hh_tot);
  std::vector<int32_t> pp_swap(pp_tot), hh_swap(hh_tot);
  std::vector<std::vector<int32_t>> seg(nsp);
  for (uint64_t c = 0; c < nch; c++) {
    if (act_of[c] < 0) continue;
    const ChanInfo &ci = chans[act_of[c]];
    const ccdgpu_pair *pp = P->chan_maps[c].pp, *hh = P->chan_maps[c].hh;
    if (!pp || !hh) return CCDGPU_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < ci.pp; k++) {
      if (pp[k].p < np || pp[k].q < np || pp[k].p >= nsp || pp[k].q >= nsp) return CCDGPU_ERR_BAD_TABLE;
      pp_pairs[ci.pp_off + k] = make_int2((int)pp[k].p, (int)pp[k].q);
      int sw = find_pair(pp, ci.pp, pp[k].q, pp[k].p);
      if (sw < 0) return CCDGPU_ERR_BAD_TABLE;
      pp_swap[ci.pp_off + k] = sw;
      seg[pp[k].p].push_back((int32_t)(ci.pp_off + k));
    }
    for (int k = 0; k < ci.hh; k++) {
      if (hh[k].p >= np || hh[k].q >= np) return CCDGPU_ERR_BAD_TABLE;
      hh_pairs[ci.hh_off + k] = make_int2((int)hh[k].p, (int)hh[k].q);
      int sw = find_pair(hh, ci.hh, hh[k].q, hh[k].p);
      if (sw < 0) return CCDGPU_ERR_BAD_TABLE;
      hh_swap[ci.hh_off + k] = sw;
      seg[hh[k].p].push_back((int32_t)(ci.hh_off + k));
    }
  }
  std::vector<int64_t> list_off(nsp + 1, 0);
  for (uint64_t w = 0; w < nsp; w++) list_off[w + 1] = list_off[w] + (int64_t)seg[w].size();
  std::vector<int32_t> list(list_off[nsp]);
  for (uint64_t w = 0; w < nsp; w++) std::copy(seg[w].begin(), seg[w].end(), list.begin() + list_off[w]);

  // Modified channels.
  std::vector<ModInfo> mods, mods_big;
  std::vector<int64_t> mod_y(nch, -1);
  int64_t y_tot = 0;
  size_t ring_smem = 0;
  for (uint64_t c = 0; c < nch; c++) {
    const int64_t ph = MD[c].ph, hp = MD[c].hp;
    if (!ph || !hp) continue;
    ModInfo m{};
    m.ph = (int)ph; m.hp = (int)hp; m.m_off = o_m[c]; m.y_off = y_tot;
    mod_y[c] = y_tot;
    y_tot += hp * hp;
    if (ph <= kRingSmall && hp <= kRingSmall) {
      mods.push_back(m);
    } else {
      ring_smem = std::max(ring_smem, (size_t)(2 * ph * hp + hp * hp) * 8);
      mods_big.push_back(m);
    }
  }
  h->n_mod_small = (int)mods.size();
  mods.insert(mods.end(), mods_big.begin(), mods_big.end());
  h->n_mod = (int)mods.size();
  h->ring_smem = ring_smem;

  // Three-body chain offsets.
  std::vector<int64_t> o_h(np + 1, 0), o_p(h->npart + 1, 0);
  for (uint64_t k = 0; k < np; k++) o_h[k + 1] = o_h[k] + (int64_t)P->three_body_dims[k].hpp;
  for (uint64_t a = 0; a < h->npart; a++)
    o_p[a + 1] = o_p[a] + (int64_t)P->three_body_dims[np + a].phh;
  h->n_h = o_h[np];
  h->n_p = o_p[h->npart];

  // Remap tables -> flat int32 offsets, with range and bijection checks.
  const int64_t n_t = h->n_t;
  std::vector<int32_t> flat((size_t)8 * n_t);
  int bad = 0;
  for (int k = 0; k < 8; k++) {
    if (!P->maps[k]) return CCDGPU_ERR_INVALID_ARGUMENT;
#pragma omp parallel for schedule(dynamic) reduction(| : bad)
    for (int64_t ci = 0; ci < (int64_t)nch; ci++) {
      const uint64_t c = (uint64_t)ci;
      const int64_t n = o_t[c + 1] - o_t[c];
      if (!n) continue;
      const ccdgpu_chain_index *m = P->maps[k][c];
      if (!m) { bad |= 1; continue; }
      for (int64_t e = 0; e < n; e++) {
        const uint64_t ch = m[e].channel, row = m[e].row, col = m[e].column;
        int64_t f = -1;
        if (k <= 1) {
          if (ch < np && col == 0 && row < P->three_body_dims[ch].hpp) f = o_h[ch] + (int64_t)row;
        } else if (k <= 3) {
          if (ch < h->npart && row == 0 && col < P->three_body_dims[np + ch].phh) f = o_p[ch] + (int64_t)col;
        } else {
          if (ch < nch && row < MD[ch].ph && col < MD[ch].hp) f = o_m[ch] + (int64_t)(row * MD[ch].hp + col);
        }
        if (f < 0) { bad |= 1; continue; }
        flat[(size_t)k * n_t + o_t[c] + e] = (int32_t)f;
      }
    }
  }
  if (bad) return CCDGPU_ERR_BAD_TABLE;
  // Scatter targets must be hit exactly once (Chain::mapToDistributed writes every slot).
  {
    const int scat[5] = {CCDGPU_MAP_IAB_J, CCDGPU_MAP_JAB_I, CCDGPU_MAP_A_BIJ, CCDGPU_MAP_B_AIJ,
                         CCDGPU_MAP_AI_JB};
    const int64_t tgt[5] = {h->n_h, h->n_h, h->n_p, h->n_p, h->n_m};
    for (int q = 0; q < 5; q++) {
      if (tgt[q] != n_t) return CCDGPU_ERR_BAD_TABLE;
      std::vector<uint8_t> hit(n_t, 0);
      const int32_t *f = &flat[(size_t)scat[q] * n_t];
      for (int64_t e = 0; e < n_t; e++) {
        if (hit[f[e]]) return CCDGPU_ERR_BAD_TABLE;
        hit[f[e]] = 1;
      }
    }
  }

  // V blocks.
  std::vector<double> v_pphh(n_t), v_hhhh(x_tot), v_t(vt, 0.0), v_hpph(h->n_m), v_hphp(y_tot);
  const bool on_the_fly = h->opt.v_mode == CCDGPU_V_ON_THE_FLY;
  if (on_the_fly) return CCDGPU_ERR_UNSUPPORTED;  // generated V_pppp: not built yet
  if (!P->v_pppp || !P->v_hhpp || !P->v_hhhh || !P->v_hpph_mod || !P->v_hphp_mod)
    return CCDGPU_ERR_INVALID_ARGUMENT;
  bad = 0;
#pragma omp parallel for schedule(dynamic) reduction(| : bad)
  for (int64_t ci = 0; ci < (int64_t)nch; ci++) {
    const uint64_t c = (uint64_t)ci;
    if (act_of[c] < 0) continue;
    const ChanInfo &a = chans[act_of[c]];
    const double *vx = P->v_hhpp[c], *vh = P->v_hhhh[c], *vp = P->v_pppp[c];
    if (!vx || !vh || !vp) { bad |= 1; continue; }
    for (int ij = 0; ij < a.hh; ij++)
      for (int ab = 0; ab < a.pp; ab++) v_pphh[a.t_off + (int64_t)ab * a.hh + ij] = vx[(int64_t)ij * a.pp + ab];
    std::memcpy(&v_hhhh[a.x_off], vh, sizeof(double) * a.hh * a.hh);
    // Packed V tiles: rows a<=b (rowmap), columns c<d (pk_idx.x), zero padding elsewhere.
    std::vector<int32_t> kcol(a.pk);
    for (int k = 0; k < a.pp; k++)
      if (pk_idx[a.pp_off + k].x >= 0) kcol[pk_idx[a.pp_off + k].x] = k;
    for (int u = 0; u < a.pr; u++) {
      const int ab = rowmap[a.row_off + u];
      const int64_t tb = a.vkt_base + (int64_t)(u / a.bm) * a.nkc * a.bm * kBK;
      for (int w = 0; w < a.pk; w++)
        v_t[tb + (int64_t)(w / kBK) * a.bm * kBK + swzA(u % a.bm, w % kBK)] =
            vp[(int64_t)ab * a.pp + kcol[w]];
    }
  }
  if (bad) return CCDGPU_ERR_INVALID_ARGUMENT;
  for (uint64_t c = 0; c < nch; c++) {
    const int64_t ph = MD[c].ph, hp = MD[c].hp;
    if (!ph || !hp) continue;
    const double *va = P->v_hpph_mod[c], *vb = P->v_hphp_mod[c];
    if (!va || !vb) return CCDGPU_ERR_INVALID_ARGUMENT;
    std::memcpy(&v_hpph[o_m[c]], va, sizeof(double) * ph * hp);
    std::memcpy(&v_hphp[mod_y[c]], vb, sizeof(double) * hp * hp);
  }
  std::vector<double> v_h_hpp, v_phh_p;
  h->have_3body = P->v_h_hpp && P->v_phh_p;
  if (h->have_3body) {
    v_h_hpp.resize(h->n_h);
    v_phh_p.resize(h->n_p);
    for (uint64_t k = 0; k < np; k++) {
      const int64_t n = o_h[k + 1] - o_h[k];
      if (n && !P->v_h_hpp[k]) return CCDGPU_ERR_INVALID_ARGUMENT;
      if (n) std::memcpy(&v_h_hpp[o_h[k]], P->v_h_hpp[k], sizeof(double) * n);
    }
    for (uint64_t a = 0; a < h->npart; a++) {
      const int64_t n = o_p[a + 1] - o_p[a];
      if (n && !P->v_phh_p[a]) return CCDGPU_ERR_INVALID_ARGUMENT;
      if (n) std::memcpy(&v_phh_p[o_p[a]], P->v_phh_p[a], sizeof(double) * n);
    }
  }

  // pp-ladder work tiles, heaviest first (the on-device analogue of ffdBalance).
  std::vector<LadderTile> tiles;
  for (int ai = 0; ai < h->n_act; ai++) {
    const ChanInfo &a = chans[ai];
    for (int mt = 0; mt < a.nmt; mt++) {
      LadderTile tl{};
      tl.ch = ai; tl.mt = mt; tl.nkc = a.nkc; tl.nkh = a.nkh; tl.cg = a.cg; tl.bm = a.bm;
      tl.pr = a.pr; tl.hh = a.hh;
      tl.v_base = a.vkt_base; tl.tkt_base = a.tkt_base; tl.tmt_base = a.tmt_base;
      tl.xt_base = a.xt_base; tl.t_off = a.t_off; tl.row_off = a.row_off;
      tiles.push_back(tl);
    }
  }
  // Narrow channels (<= 32 hh columns) first, then wide ones; within each class the longest
  // K streams first so the hardware block scheduler fills in the short ones.
  std::stable_sort(tiles.begin(), tiles.end(), [](const LadderTile &x, const LadderTile &y) {
    const bool nx = x.cg <= kNarrowCG, ny = y.cg <= kNarrowCG;
    if (nx != ny) return nx;
    return (int64_t)(x.nkc + x.nkh) * (x.bm + 8 * x.cg) > (int64_t)(y.nkc + y.nkh) * (y.bm + 8 * y.cg);
  });
  h->n_tiles_narrow = 0;
  for (const LadderTile &t : tiles) h->n_tiles_narrow += t.cg <= kNarrowCG;
  h->n_tiles = (int)tiles.size();
  std::vector<ElemRange> ranges;
  const int64_t per = (int64_t)kAsmThreads * kAsmPerThread;
  for (int ai = 0; ai < h->n_act; ai++) {
    const ChanInfo &a = chans[ai];
    const int64_t n = (int64_t)a.pp * a.hh;
    for (int64_t e = 0; e < n; e += per) ranges.push_back({ai, 0, a.t_off + e, a.t_off + std::min(n, e + per)});
  }
  h->n_ranges = (int)ranges.size();

  // Work estimate (reference GEMM flops) for roofline reporting.
  double fl = 0, lf = 0, vb = 0;
  for (const ChanInfo &a : chans) {
    lf += 2.0 * a.pp * a.pp * a.hh;
    fl += 2.0 * a.pp * a.pp * a.hh + 4.0 * a.pp * a.hh * (double)a.hh;
    vb += 8.0 * a.pp * a.pp;
  }
  for (const ModInfo &m : mods) fl += 4.0 * m.ph * (double)m.hp * m.hp;
  h->flops = fl; h->ladder_flops = lf; h->v_bytes = vb;

  // Device allocations and uploads.
  int rc;
#define TRY(x) do { rc = (x); if (rc) return rc; } while (0)
  TRY(upload(h, &h->chans, chans));
  TRY(upload(h, &h->mods, mods));
  TRY(upload(h, &h->tiles, tiles));
  TRY(upload(h, &h->hh_tiles, hh_tiles));
  TRY(upload(h, &h->rowmap, rowmap));
  TRY(upload(h, &h->mirror, mirror));
  TRY(upload(h, &h->pk_idx, pk_idx));
  TRY(dalloc(h, &h->counters, h->n_act));
  TRY(dalloc(h, &h->part, part_tot));
  TRY(upload(h, &h->ranges, ranges));
  TRY(upload(h, &h->pp_pairs, pp_pairs));
  TRY(upload(h, &h->hh_pairs, hh_pairs));
  TRY(upload(h, &h->pp_swap, pp_swap));
  TRY(upload(h, &h->hh_swap, hh_swap));
  TRY(upload(h, &h->list_off, list_off));
  TRY(upload(h, &h->list, list));
  std::vector<double> eps(P->sp_energy, P->sp_energy + nsp);
  TRY(upload(h, &h->eps, eps));
  TRY(upload(h, &h->v_pphh, v_pphh));
  TRY(upload(h, &h->v_hhhh, v_hhhh));
  TRY(upload(h, &h->v_t, v_t));
  TRY(upload(h, &h->v_hpph, v_hpph));
  TRY(upload(h, &h->v_hphp, v_hphp));
  TRY(upload(h, &h->flat, flat));
  TRY(upload(h, &h->o_h, o_h));
  TRY(upload(h, &h->o_p, o_p));
  TRY(dalloc(h, &h->t[0], n_t));
  TRY(dalloc(h, &h->t[1], n_t));
  TRY(dalloc(h, &h->dmat, n_t));
  TRY(dalloc(h, &h->old_phhp, h->n_m));
  TRY(dalloc(h, &h->r_phhp, h->n_m));
  TRY(dalloc(h, &h->x, x_tot));
  TRY(dalloc(h, &h->x_t, xt));
  TRY(dalloc(h, &h->t_kt, tkt));
  TRY(dalloc(h, &h->t_mt, tmt));
  TRY(dalloc(h, &h->s, hh_tot));
  TRY(dalloc(h, &h->r, pp_tot));
  TRY(dalloc(h, &h->xh, np));
  TRY(dalloc(h, &h->yp, h->npart));
  TRY(dalloc(h, &h->epart, h->n_ranges));
  TRY(dalloc(h, &h->ctl, 1));
  TRY(dalloc(h, &h->e_out, 1));
  TRY(dalloc(h, &h->err, 1));
  if (h->have_3body) {
    TRY(upload(h, &h->v_h_hpp, v_h_hpp));
    TRY(upload(h, &h->v_phh_p, v_phh_p));
    TRY(dalloc(h, &h->old_h1pp_h2, h->n_h));
    TRY(dalloc(h, &h->old_h2pp_h1, h->n_h));
    TRY(dalloc(h, &h->diff_h2pp_h1, h->n_h));
    TRY(dalloc(h, &h->old_p1_p2hh, h->n_p));
    TRY(dalloc(h, &h->old_p2_p1hh, h->n_p));
    TRY(dalloc(h, &h->diff_p2_p1hh, h->n_p));
    TRY(dalloc(h, &h->gath, (size_t)8 * n_t));
  }
#undef TRY
  CK(cudaMallocHost(&h->h_ctl, sizeof(Control)));
  std::memset(h->h_ctl, 0, sizeof(Control));

  h->ladder_smem = (size_t)kStages * (kMaxBM * kBK + kBK * kMaxCG * 8) * 8 + 2 * kStages * 8;
  CK(cudaFuncSetAttribute(pp_ladder_kernel<1, kNarrowCG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)h->ladder_smem));
  CK(cudaFuncSetAttribute(pp_ladder_kernel<1, kNarrowCG>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  CK(cudaFuncSetAttribute(pp_ladder_kernel<kNarrowCG + 1, kMaxCG>,
                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->ladder_smem));
  CK(cudaFuncSetAttribute(pp_ladder_kernel<kNarrowCG + 1, kMaxCG>,
                          cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  int maxhh = 1;
  for (const ChanInfo &a : chans) maxhh = std::max(maxhh, a.hh);
  h->hh_smem = (size_t)2 * kHHRows * maxhh * 8;
  CK(cudaFuncSetAttribute(hh_ladder_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)h->hh_smem));
  CK(cudaFuncSetAttribute(ring_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)std::max<size_t>(h->ring_smem, 16)));
  CK(cudaStreamSynchronize(h->s0));
  return CCDGPU_OK;
}

// ---- launches -------------------------------------------------------------------------

int launch_hh_ladder(ccdgpu_handle *h, cudaStream_t st) {
  if (!h->n_hh_tiles) return CCDGPU_OK;
  hh_ladder_kernel<<<h->n_hh_tiles, kHHThreads, h->hh_smem, st>>>(
      h->hh_tiles, h->chans, h->v_pphh, h->v_hhhh, h->t[0], h->t[1], h->part, h->counters, h->x,
      h->x_t, h->s, h->r, h->ctl);
  h->launches++;
  return cuda_status(cudaGetLastError());
}
int launch_pp_ladder(ccdgpu_handle *h, cudaStream_t st) {
  if (h->n_tiles_narrow) {
    pp_ladder_kernel<1, kNarrowCG><<<h->n_tiles_narrow, kLadderThreads, h->ladder_smem, st>>>(
        h->tiles, h->v_t, h->t_kt, h->t_mt, h->x_t, h->rowmap, h->mirror, h->dmat, h->ctl, h->err);
    h->launches++;
    CK(cudaGetLastError());
  }
  const int nwide = h->n_tiles - h->n_tiles_narrow;
  if (nwide) {
    pp_ladder_kernel<kNarrowCG + 1, kMaxCG><<<nwide, kLadderThreads, h->ladder_smem, st>>>(
        h->tiles + h->n_tiles_narrow, h->v_t, h->t_kt, h->t_mt, h->x_t, h->rowmap, h->mirror,
        h->dmat, h->ctl, h->err);
    h->launches++;
    CK(cudaGetLastError());
  }
  return CCDGPU_OK;
}
int launch_ring(ccdgpu_handle *h, cudaStream_t st) {
  if (h->n_mod_small) {
    ring_small_kernel<<<(int)ceil_div(h->n_mod_small, 8), 256, 0, st>>>(
        h->mods, h->n_mod_small, h->v_hpph, h->v_hphp, h->old_phhp, h->r_phhp, h->ctl);
    h->launches++;
    CK(cudaGetLastError());
  }
  const int nbig = h->n_mod - h->n_mod_small;
  if (nbig) {
    ring_kernel<<<nbig, kRingThreads, std::max<size_t>(h->ring_smem, 16), st>>>(
        h->mods + h->n_mod_small, h->v_hpph, h->v_hphp, h->old_phhp, h->r_phhp, h->ctl);
    h->launches++;
    CK(cudaGetLastError());
  }
  return CCDGPU_OK;
}
int launch_onebody_fused(ccdgpu_handle *h, cudaStream_t st) {
  const int warps_per_block = 8;
  const int blocks = (int)ceil_div((int64_t)h->nsp, warps_per_block);
  onebody_fused_kernel<<<blocks, warps_per_block * 32, 0, st>>>((int)h->np, (int)h->nsp, h->list_off,
                                                                 h->list, h->s, h->r, h->xh, h->yp, h->ctl);
  h->launches++;
  return cuda_status(cudaGetLastError());
}
int launch_assemble_fused(ccdgpu_handle *h, cudaStream_t st) {
  if (!h->n_ranges) return CCDGPU_OK;
  const int64_t n_t = h->n_t;
  assemble_fused_kernel<<<h->n_ranges, kAsmThreads, 0, st>>>(
      h->ranges, h->chans, h->pp_pairs, h->hh_pairs, h->pp_swap, h->hh_swap, h->pk_idx, h->v_pphh,
      h->dmat,
      h->r_phhp, h->flat + 4 * n_t, h->flat + 5 * n_t, h->flat + 6 * n_t, h->flat + 7 * n_t, h->xh,
      h->yp, h->eps, (int)h->np, h->t[0], h->t[1], h->old_phhp, h->t_kt, h->t_mt, h->epart, h->ctl);
  h->launches++;
  return cuda_status(cudaGetLastError());
}
int launch_energy(ccdgpu_handle *h, cudaStream_t st, int flags) {
  energy_kernel<<<1, 1024, 0, st>>>(h->epart, h->n_ranges, h->ctl, flags, h->e_out);
  h->launches++;
  return cuda_status(cudaGetLastError());
}
int launch_map_to(ccdgpu_handle *h, cudaStream_t st, const double *src, double *dst) {
  if (!h->n_ranges) return CCDGPU_OK;
  map_to_kernel<<<h->n_ranges, 256, 0, st>>>(h->ranges, h->chans, h->pk_idx, h->flat, h->n_t, src, dst,
                                               h->old_h2pp_h1, h->old_h1pp_h2, h->old_p1_p2hh,
                                               h->old_p2_p1hh, h->old_phhp, h->t_kt, h->t_mt,
                                               h->have_3body ? 1 : 0);
  h->launches++;
  return cuda_status(cudaGetLastError());
}

// One fused iteration: hh ladder and ring concurrently, then one-body, pp ladder, assembly.
int enqueue_fused_iteration(ccdgpu_handle *h) {
  int rc;
  if (h->profiling) {
    // ev: 0 start, 1 after hh ladder, 2 after one-body, 3 after pp ladder, 4/5 ring on s1,
    // 6 after assembly, 7 after the energy reduction.
    CK(cudaEventRecord(h->ev[0], h->s0));
    CK(cudaStreamWaitEvent(h->s1, h->ev[0], 0));
    CK(cudaEventRecord(h->ev[4], h->s1));
    if ((rc = launch_ring(h, h->s1))) return rc;
    CK(cudaEventRecord(h->ev[5], h->s1));
    if ((rc = launch_hh_ladder(h, h->s0))) return rc;
    CK(cudaEventRecord(h->ev[1], h->s0));
    if ((rc = launch_onebody_fused(h, h->s0))) return rc;
    CK(cudaEventRecord(h->ev[2], h->s0));
    if ((rc = launch_pp_ladder(h, h->s0))) return rc;
    CK(cudaEventRecord(h->ev[3], h->s0));
    CK(cudaStreamWaitEvent(h->s0, h->ev[5], 0));
    CK(cudaEventRecord(h->ev[8], h->s0));
    if ((rc = launch_assemble_fused(h, h->s0))) return rc;
    CK(cudaEventRecord(h->ev[6], h->s0));
    if ((rc = launch_energy(h, h->s0, 3))) return rc;
    CK(cudaEventRecord(h->ev[7], h->s0));
    return CCDGPU_OK;
  }
  CK(cudaEventRecord(h->ev_fork, h->s0));
  CK(cudaStreamWaitEvent(h->s1, h->ev_fork, 0));
  if ((rc = launch_ring(h, h->s1))) return rc;
  CK(cudaEventRecord(h->ev_join, h->s1));
  if ((rc = launch_hh_ladder(h, h->s0))) return rc;
  if ((rc = launch_onebody_fused(h, h->s0))) return rc;
  if ((rc = launch_pp_ladder(h, h->s0))) return rc;
  CK(cudaStreamWaitEvent(h->s0, h->ev_join, 0));
  if ((rc = launch_assemble_fused(h, h->s0))) return rc;
  return launch_energy(h, h->s0, 3);
}

// Table path stages (mirrors main.cpp:591-665).
int stage_onebody_tables(ccdgpu_handle *h, int holes, int particles) {
  if (!h->have_3body) return CCDGPU_ERR_UNSUPPORTED;
  const int nb = (int)h->nsp;
  onebody_tables_kernel<<<nb, kOBThreads, 0, h->s0>>>(
      (int)h->np, h->o_h, h->o_p, h->v_h_hpp, h->old_h2pp_h1, h->old_h1pp_h2, h->diff_h2pp_h1,
      h->v_phh_p, h->old_p1_p2hh, h->old_p2_p1hh, h->diff_p2_p1hh, holes, particles);
  h->launches++;
  return cuda_status(cudaGetLastError());
}
int stage_gather(ccdgpu_handle *h) {
  if (!h->have_3body) return CCDGPU_ERR_UNSUPPORTED;
  const int blocks = (int)std::min<int64_t>(ceil_div(h->n_t, 256), 148 * 16);
  gather8_kernel<<<std::max(blocks, 1), 256, 0, h->s0>>>(h->n_t, h->flat, h->diff_h2pp_h1,
                                                         h->diff_p2_p1hh, h->r_phhp, h->gath);
  h->launches++;
  return cuda_status(cudaGetLastError());
}
int stage_assemble_tables(ccdgpu_handle *h, double mixing) {
  if (!h->have_3body) return CCDGPU_ERR_UNSUPPORTED;
  if (h->n_ranges) {
    assemble_tables_kernel<<<h->n_ranges, kAsmThreads, 0, h->s0>>>(
        h->ranges, h->chans, h->pp_pairs, h->hh_pairs, h->v_pphh, h->dmat, h->gath, h->n_t, h->eps,
        h->t[0], h->t[1], h->epart, mixing);
    h->launches++;
    CK(cudaGetLastError());
  }
  return CCDGPU_OK;
}

int sync_ctl(ccdgpu_handle *h) {
  CK(cudaMemcpyAsync(h->h_ctl, h->ctl, sizeof(Control), cudaMemcpyDeviceToHost, h->s0));
  CK(cudaStreamSynchronize(h->s0));
  return CCDGPU_OK;
}

int check_errors(ccdgpu_handle *h) {
  int32_t e = 0;
  CK(cudaMemcpy(&e, h->err, sizeof(int32_t), cudaMemcpyDeviceToHost));
  if (e & kErrTimeout) return CCDGPU_ERR_TIMEOUT;
  if (h->h_ctl->error & kErrNonFinite) return CCDGPU_ERR_NONFINITE;
  return CCDGPU_OK;
}

int set_ctl(ccdgpu_handle *h, int active, double tol, int64_t max_iters, double mixing,
            bool reset_loop, int parity = -1) {
  int rc = sync_ctl(h);
  if (rc) return rc;
  Control &c = *h->h_ctl;
  if (parity >= 0) c.parity = parity;
  if (reset_loop) {
    c.e_prev = 100.0;
    c.e_diff = 1.0;
    c.iterations = 0;
    c.done = 0;
    c.error = 0;
    std::memset(c.energies, 0, sizeof(c.energies));
  }
  c.active = active;
  c.tol = tol;
  c.max_iters = max_iters;
  c.mixing = mixing;
  CK(cudaMemcpyAsync(h->ctl, h->h_ctl, sizeof(Control), cudaMemcpyHostToDevice, h->s0));
  CK(cudaStreamSynchronize(h->s0));
  return CCDGPU_OK;
}

int fused_ready_graph(ccdgpu_handle *h) {
  if (h->graph) return CCDGPU_OK;
  cudaGraph_t g = nullptr;
  const int64_t before = h->launches;
  CK(cudaStreamBeginCapture(h->s0, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_fused_iteration(h);
  h->kernels_per_graph = h->launches - before;
  h->launches = before;
  cudaError_t e = cudaStreamEndCapture(h->s0, &g);
  if (rc) { if (g) cudaGraphDestroy(g); return rc; }
  CK(e);
  e = cudaGraphInstantiate(&h->graph, g, 0);
  cudaGraphDestroy(g);
  CK(e);
  return CCDGPU_OK;
}

// One table-path iteration: exactly the reference loop body.
int tables_iteration(ccdgpu_handle *h, double mixing, double *corr) {
  int rc;
  if ((rc = stage_onebody_tables(h, 0, 1))) return rc;     // calcT2Diff_p2_p1hh
  if ((rc = stage_onebody_tables(h, 1, 0))) return rc;     // calcT2Diff_h2pp_h1
  if ((rc = launch_ring(h, h->s0))) return rc;             // calcT2Diff_phhp
  if ((rc = launch_hh_ladder(h, h->s0))) return rc;        // calcT2Diff_pphh
  if ((rc = launch_pp_ladder(h, h->s0))) return rc;
  if ((rc = stage_gather(h))) return rc;                   // 8 x mapFromDistributed
  if ((rc = stage_assemble_tables(h, mixing))) return rc;  // calcT2_pphh
  if ((rc = launch_energy(h, h->s0, 2))) return rc;
  if ((rc = launch_map_to(h, h->s0, h->t[1], h->t[0]))) return rc;  // set + 5 x mapToDistributed
  (void)corr;
  return CCDGPU_OK;
}

}  // namespace

extern "C" {

void ccdgpu_default_options(ccdgpu_options *opt) {
  if (!opt) return;
  std::memset(opt, 0, sizeof(*opt));
  opt->device = 0;
  opt->precision = CCDGPU_PREC_FP64;
  opt->v_mode = CCDGPU_V_STORED;
  opt->path = CCDGPU_PATH_FUSED;
  opt->polish_threshold = 1e-9;
  opt->use_graph = 1;
}

const char *ccdgpu_strerror(int status) {
  switch (status) {
    case CCDGPU_OK: return "ok";
    case CCDGPU_ERR_INVALID_ARGUMENT: return "invalid argument";
    case CCDGPU_ERR_CUDA: return "CUDA error";
    case CCDGPU_ERR_OUT_OF_MEMORY: return "out of device memory";
    case CCDGPU_ERR_BAD_TABLE: return "remap table out of range or not a bijection";
    case CCDGPU_ERR_NONFINITE: return "non-finite amplitudes or energy";
    case CCDGPU_ERR_NO_DEVICE: return "no CUDA device";
    case CCDGPU_ERR_UNSUPPORTED: return "unsupported problem or option";
    case CCDGPU_ERR_NOT_CONVERGED: return "not converged within the iteration cap";
    case CCDGPU_ERR_TIMEOUT: return "device wait timed out";
    default: return "unknown status";
  }
}

int ccdgpu_create(const ccdgpu_problem *prob, const ccdgpu_options *opt, ccdgpu_handle **out) {
  if (!prob || !out) return CCDGPU_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (!prob->sp_energy || !prob->chan_dims || !prob->chan_mod_dims || !prob->chan_maps ||
      !prob->three_body_dims || prob->n_particles == 0 || prob->n_particles >= prob->n_sp)
    return CCDGPU_ERR_INVALID_ARGUMENT;
  ccdgpu_handle *h = new (std::nothrow) ccdgpu_handle();
  if (!h) return CCDGPU_ERR_OUT_OF_MEMORY;
  if (opt) h->opt = *opt;
  else ccdgpu_default_options(&h->opt);
  if (h->opt.precision != CCDGPU_PREC_FP64) { delete h; return CCDGPU_ERR_UNSUPPORTED; }
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) { (void)cudaGetLastError(); delete h; return CCDGPU_ERR_NO_DEVICE; }
  if (h->opt.device < 0 || h->opt.device >= ndev) { delete h; return CCDGPU_ERR_INVALID_ARGUMENT; }
  int rc = cuda_status(cudaSetDevice(h->opt.device));
  if (!rc) rc = cuda_status(cudaStreamCreateWithFlags(&h->s0, cudaStreamNonBlocking));
  if (!rc) rc = cuda_status(cudaStreamCreateWithFlags(&h->s1, cudaStreamNonBlocking));
  if (!rc) rc = cuda_status(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
  if (!rc) rc = cuda_status(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
  for (int i = 0; i < 10 && !rc; i++) rc = cuda_status(cudaEventCreate(&h->ev[i]));
  if (!rc) rc = build(h, prob);
  if (!rc) rc = set_ctl(h, 0, 0.0, 100, 0.5, true);
  if (rc) { release(h); delete h; return rc; }
  *out = h;
  return CCDGPU_OK;
}

void ccdgpu_destroy(ccdgpu_handle *h) {
  if (!h) return;
  cudaSetDevice(h->opt.device);
  if (h->s0) cudaStreamSynchronize(h->s0);
  release(h);
  delete h;
}

uint64_t ccdgpu_t2_size(const ccdgpu_handle *h) { return h ? (uint64_t)h->n_t : 0; }

int ccdgpu_reset(ccdgpu_handle *h) {
  if (!h) return CCDGPU_ERR_INVALID_ARGUMENT;
  CK(cudaSetDevice(h->opt.device));
  double *z[] = {h->t[0], h->t[1], h->old_phhp, h->t_kt, h->t_mt, h->old_h1pp_h2, h->old_h2pp_h1,
                 h->old_p1_p2hh, h->old_p2_p1hh};
  for (double *p : z) {
    if (!p) continue;
    for (auto &b : h->allocs)
      if (b.p == p) CK(cudaMemsetAsync(p, 0, b.bytes, h->s0));
  }
  return set_ctl(h, 0, h->h_ctl->tol, h->h_ctl->max_iters, h->h_ctl->mixing, true, 0);
}

int ccdgpu_set_t2(ccdgpu_handle *h, const double *t2, uint64_t n) {
  if (!h || !t2 || n != (uint64_t)h->n_t) return CCDGPU_ERR_INVALID_ARGUMENT;
  CK(cudaSetDevice(h->opt.device));
  int rc = sync_ctl(h);
  if (rc) return rc;
  h->h_ctl->parity = 0;
  CK(cudaMemcpyAsync(h->ctl, h->h_ctl, sizeof(Control), cudaMemcpyHostToDevice, h->s0));
  CK(cudaMemcpyAsync(h->t[1], t2, n * 8, cudaMemcpyHostToDevice, h->s0));
  if ((rc = launch_map_to(h, h->s0, h->t[1], h->t[0]))) return rc;
  CK(cudaStreamSynchronize(h->s0));
  return CCDGPU_OK;
}

int ccdgpu_get_t2(ccdgpu_handle *h, double *t2, uint64_t n) {
  if (!h || !t2 || n != (uint64_t)h->n_t) return CCDGPU_ERR_INVALID_ARGUMENT;
  CK(cudaSetDevice(h->opt.device));
  int rc = sync_ctl(h);
  if (rc) return rc;
  const double *src = h->t[h->h_ctl->parity];
  if (h->opt.path == CCDGPU_PATH_TABLES) src = h->t[1];
  CK(cudaMemcpyAsync(t2, src, n * 8, cudaMemcpyDeviceToHost, h->s0));
  CK(cudaStreamSynchronize(h->s0));
  return CCDGPU_OK;
}

int ccdgpu_step(ccdgpu_handle *h, double mixing, double *e_corr) {
  if (!h) return CCDGPU_ERR_INVALID_ARGUMENT;
  CK(cudaSetDevice(h->opt.device));
  int rc = set_ctl(h, 0, h->h_ctl->tol, INT64_MAX / 2, mixing, false);
  if (rc) return rc;
  if (h->opt.path == CCDGPU_PATH_TABLES) rc = tables_iteration(h, mixing, nullptr);
  else rc = enqueue_fused_iteration(h);
  if (rc) return rc;
  if ((rc = sync_ctl(h))) return rc;
  if ((rc = check_errors(h))) return rc;
  if (e_corr) *e_corr = h->h_ctl->e_corr;
  return std::isfinite(h->h_ctl->e_corr) ? CCDGPU_OK : CCDGPU_ERR_NONFINITE;
}

int ccdgpu_solve(ccdgpu_handle *h, double tol, int64_t max_iters, double mixing, ccdgpu_result *res) {
  if (!h || max_iters < 0 || !(tol >= 0)) return CCDGPU_ERR_INVALID_ARGUMENT;
  CK(cudaSetDevice(h->opt.device));
  int rc = set_ctl(h, 1, tol, max_iters, mixing, true);
  if (rc) return rc;
  const bool fused = h->opt.path == CCDGPU_PATH_FUSED;
  const bool graph = fused && h->opt.use_graph && !h->profiling;
  if (graph && (rc = fused_ready_graph(h))) return rc;
  auto t0 = std::chrono::steady_clock::now();
  int64_t launched = 0;
  const int64_t cap = max_iters + 1;
  while (true) {
    // Iterations are launched in batches; once the device-side stop rule fires the remaining
    // launches of the batch return immediately.
    const int64_t batch =
        (fused && !h->profiling) ? std::min<int64_t>(launched < 8 ? 4 : 8, cap - launched) : 1;
    for (int64_t b = 0; b < batch; b++) {
      if (graph) CK(cudaGraphLaunch(h->graph, h->s0));
      else if (fused) { if ((rc = enqueue_fused_iteration(h))) return rc; }
      else {
        if ((rc = tables_iteration(h, mixing, nullptr))) return rc;
      }
    }
    launched += batch;
    if (graph) h->launches += batch * h->kernels_per_graph;
    if ((rc = sync_ctl(h))) return rc;
    if (h->profiling && fused && !graph) {
      float a = 0, b = 0, c = 0, d = 0, e = 0, f = 0;
      cudaEventElapsedTime(&a, h->ev[0], h->ev[1]);
      cudaEventElapsedTime(&b, h->ev[1], h->ev[2]);
      cudaEventElapsedTime(&c, h->ev[2], h->ev[3]);
      cudaEventElapsedTime(&d, h->ev[4], h->ev[5]);
      cudaEventElapsedTime(&e, h->ev[8], h->ev[7]);
      cudaEventElapsedTime(&f, h->ev[0], h->ev[7]);
      h->prof.ms_hh_ladder += a;
      h->prof.ms_onebody += b;
      h->prof.ms_ladder += c;
      h->prof.ms_ring += d;
      h->prof.ms_assemble += e;
      h->prof.ms_total += f;
      h->prof.iterations += 1;
    }
    if (h->h_ctl->done || launched >= cap) break;
  }
  auto t1 = std::chrono::steady_clock::now();
  if ((rc = check_errors(h))) return rc;
  const Control &c = *h->h_ctl;
  if (res) {
    res->e_corr = c.e_corr;
    res->e_diff = c.e_diff;
    res->iterations = c.iterations;
    res->converged = std::fabs(c.e_diff) <= tol ? 1 : 0;
    res->polish_iterations = 0;
    res->seconds = std::chrono::duration<double>(t1 - t0).count();
  }
  return CCDGPU_OK;
}

int ccdgpu_energy_history(ccdgpu_handle *h, double *out, int64_t cap, int64_t *n_out) {
  if (!h || cap < 0) return CCDGPU_ERR_INVALID_ARGUMENT;
  CK(cudaSetDevice(h->opt.device));
  int rc = sync_ctl(h);
  if (rc) return rc;
  const int64_t n = std::min<int64_t>(h->h_ctl->iterations, 128);
  if (n_out) *n_out = n;
  if (out) std::memcpy(out, h->h_ctl->energies, sizeof(double) * std::min(n, cap));
  return CCDGPU_OK;
}

int ccdgpu_calc_t2diff_p2_p1hh(ccdgpu_handle *h) {
  if (!h) return CCDGPU_ERR_INVALID_ARGUMENT;
  int rc = set_ctl(h, 0, h->h_ctl->tol, h->h_ctl->max_iters, h->h_ctl->mixing, false);
  if (rc || (rc = stage_onebody_tables(h, 0, 1))) return rc;
  CK(cudaStreamSynchronize(h->s0));
  return CCDGPU_OK;
}
int ccdgpu_calc_t2diff_h2pp_h1(ccdgpu_handle *h) {
  if (!h) return CCDGPU_ERR_INVALID_ARGUMENT;
  int rc = set_ctl(h, 0, h->h_ctl->tol, h->h_ctl->max_iters, h->h_ctl->mixing, false);
  if (rc || (rc = stage_onebody_tables(h, 1, 0))) return rc;
  CK(cudaStreamSynchronize(h->s0));
  return CCDGPU_OK;
}
int ccdgpu_calc_t2diff_phhp(ccdgpu_handle *h) {
  if (!h) return CCDGPU_ERR_INVALID_ARGUMENT;
  int rc = set_ctl(h, 0, h->h_ctl->tol, h->h_ctl->max_iters, h->h_ctl->mixing, false);
  if (rc || (rc = launch_ring(h, h->s0))) return rc;
  CK(cudaStreamSynchronize(h->s0));
  return CCDGPU_OK;
}
int ccdgpu_calc_t2diff_pphh(ccdgpu_handle *h) {
  if (!h) return CCDGPU_ERR_INVALID_ARGUMENT;
  int rc = set_ctl(h, 0, h->h_ctl->tol, h->h_ctl->max_iters, h->h_ctl->mixing, false);
  if (rc || (rc = launch_hh_ladder(h, h->s0)) || (rc = launch_pp_ladder(h, h->s0))) return rc;
  CK(cudaStreamSynchronize(h->s0));
  return check_errors(h);
}
int ccdgpu_map_from_distributed(ccdgpu_handle *h) {
  if (!h) return CCDGPU_ERR_INVALID_ARGUMENT;
  int rc = stage_gather(h);
  if (rc) return rc;
  CK(cudaStreamSynchronize(h->s0));
  return CCDGPU_OK;
}
int ccdgpu_calc_t2_pphh(ccdgpu_handle *h, double mixing, double *corr) {
  if (!h) return CCDGPU_ERR_INVALID_ARGUMENT;
  int rc = stage_assemble_tables(h, mixing);
  if (rc || (rc = launch_energy(h, h->s0, 0))) return rc;
  double e = 0;
  CK(cudaMemcpyAsync(&e, h->e_out, 8, cudaMemcpyDeviceToHost, h->s0));
  CK(cudaStreamSynchronize(h->s0));
  if (corr) *corr = e;
  return CCDGPU_OK;
}
int ccdgpu_map_to_distributed(ccdgpu_handle *h) {
  if (!h) return CCDGPU_ERR_INVALID_ARGUMENT;
  int rc = launch_map_to(h, h->s0, h->t[1], h->t[0]);
  if (rc) return rc;
  CK(cudaStreamSynchronize(h->s0));
  return CCDGPU_OK;
}

int ccdgpu_read_chain(ccdgpu_handle *h, int32_t chain, double *out, uint64_t n, uint64_t *n_out) {
  if (!h) return CCDGPU_ERR_INVALID_ARGUMENT;
  CK(cudaSetDevice(h->opt.device));
  int rc = sync_ctl(h);
  if (rc) return rc;
  const double *src = nullptr;
  uint64_t len = 0;
  const int par = h->h_ctl->parity;
  switch (chain) {
    case CCDGPU_CHAIN_T2: src = (h->opt.path == CCDGPU_PATH_TABLES) ? h->t[1] : h->t[par]; len = h->n_t; break;
    case CCDGPU_CHAIN_T2_OLD: src = (h->opt.path == CCDGPU_PATH_TABLES) ? h->t[0] : h->t[par]; len = h->n_t; break;
    case CCDGPU_CHAIN_DIFF_PPHH: src = h->dmat; len = h->n_t; break;
    case CCDGPU_CHAIN_DIFF_PHHP: src = h->r_phhp; len = h->n_m; break;
    case CCDGPU_CHAIN_OLD_PHHP: src = h->old_phhp; len = h->n_m; break;
    case CCDGPU_CHAIN_DIFF_H2PP_H1: src = h->diff_h2pp_h1; len = h->n_h; break;
    case CCDGPU_CHAIN_DIFF_P2_P1HH: src = h->diff_p2_p1hh; len = h->n_p; break;
    default:
      if (chain >= CCDGPU_CHAIN_GATHERED0 && chain < CCDGPU_CHAIN_GATHERED0 + 8 && h->gath) {
        src = h->gath + (int64_t)(chain - CCDGPU_CHAIN_GATHERED0) * h->n_t;
        len = h->n_t;
      }
  }
  if (!src && !(chain >= 0 && chain <= 7)) return CCDGPU_ERR_INVALID_ARGUMENT;
  if (n_out) *n_out = len;
  if (!out) return CCDGPU_OK;
  if (!src) return CCDGPU_ERR_UNSUPPORTED;
  if (n < len) return CCDGPU_ERR_INVALID_ARGUMENT;
  CK(cudaMemcpy(out, src, len * 8, cudaMemcpyDeviceToHost));
  return CCDGPU_OK;
}

int ccdgpu_get_profile(ccdgpu_handle *h, ccdgpu_profile *prof) {
  if (!h || !prof) return CCDGPU_ERR_INVALID_ARGUMENT;
  *prof = h->prof;
  prof->launches = h->launches;
  return CCDGPU_OK;
}
int ccdgpu_enable_profiling(ccdgpu_handle *h, int32_t on) {
  if (!h) return CCDGPU_ERR_INVALID_ARGUMENT;
  h->profiling = on != 0;
  h->prof = ccdgpu_profile{};
  return CCDGPU_OK;
}
void *ccdgpu_stream(ccdgpu_handle *h) { return h ? (void *)h->s0 : nullptr; }
int ccdgpu_work_per_iteration(const ccdgpu_handle *h, double *flops, double *v_pppp_bytes,
                              double *ladder_flops) {
  if (!h) return CCDGPU_ERR_INVALID_ARGUMENT;
  if (flops) *flops = h->flops;
  if (v_pppp_bytes) *v_pppp_bytes = h->v_bytes;
  if (ladder_flops) *ladder_flops = h->ladder_flops;
  return CCDGPU_OK;
}

}  // extern "C"
