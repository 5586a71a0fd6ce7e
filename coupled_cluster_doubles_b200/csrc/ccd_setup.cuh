// Device-side setup kernels run once by ccdgpu_create: they turn the reference-layout inputs
// (uploaded as they are) into the solver's layouts, so that create does no O(V) host work.
#pragma once

#include <cstdint>

#include "ccd_device.cuh"
#include "ccdgpu.h"

namespace ccd {

// ChainIndex (Chain.hpp:7-11) as it arrives from the host: three size_t.
struct RawIndex {
  uint64_t channel, row, column;
};

// V_hhpp (hh x pp per channel) -> V_pphh (pp x hh), aligned with the t2 layout.
__global__ void transpose_hhpp_kernel(const ElemRange *__restrict__ ranges,
                                      const ChanInfo *__restrict__ chans,
                                      const double *__restrict__ raw, double *__restrict__ out) {
  const ElemRange rg = ranges[blockIdx.x];
  const ChanInfo ch = chans[rg.ch];
  for (int64_t e = rg.e0 + threadIdx.x; e < rg.e1; e += blockDim.x) {
    const int64_t loc = e - ch.t_off;
    const int ab = (int)(loc / ch.hh), ij = (int)(loc - (int64_t)ab * ch.hh);
    out[e] = raw[ch.t_off + (int64_t)ij * ch.pp + ab];
  }
}

// Packed, tiled V_pppp: one CTA per packed row u of one channel.  vraw holds each channel's
// packed rows (a <= b) in u order, pp values each, from vraw_off[channel].
// items[i] = (active channel, packed row); kcol[pk_off + w] = pp index of the w-th c<d pair.
__global__ void tile_v_kernel(const ChanInfo *__restrict__ chans, const int2 *__restrict__ items,
                              const int32_t *__restrict__ rowmap, const int32_t *__restrict__ kcol,
                              const int64_t *__restrict__ vraw_off, const double *__restrict__ vraw,
                              double *__restrict__ v_t) {
  const int2 it = items[blockIdx.x];
  const ChanInfo ch = chans[it.x];
  const int u = it.y;
  const double *src = vraw + vraw_off[it.x] + (int64_t)u * ch.pp;  // packed row u
  const int mt = u / ch.bm, rows = min(ch.bm, ch.pr - mt * ch.bm);
  const int ar = ladder_arows(ch.nb, rows);
  const int64_t tb = ch.vkt_base + (int64_t)mt * ladder_arows_full(ch.nb) * ch.nkc * kBK;
  for (int w = threadIdx.x; w < ch.pk; w += blockDim.x)
    v_t[tb + (int64_t)(w / kBK) * ar * kBK + ladder_aoff(ch.nb, ar, u - mt * ch.bm, w % kBK)] =
        src[kcol[ch.pk_off + w]];
}

// Packed V_pppp as nt bf16 terms in the tensor-core chunk images of the mixed-precision
// ladder (128-row tiles, 32-deep K chunks, compact last tile); one CTA per packed row.
__global__ void tile_v_tc_kernel(const ChanInfo *__restrict__ chans, const int2 *__restrict__ items,
                                 const int32_t *__restrict__ rowmap, const int32_t *__restrict__ kcol,
                                 const int64_t *__restrict__ vraw_off, const double *__restrict__ vraw,
                                 __nv_bfloat16 *__restrict__ v_tc, int64_t stride, int nt) {
  const int2 it = items[blockIdx.x];
  const ChanInfo ch = chans[it.x];
  const int u = it.y;
  const double *src = vraw + vraw_off[it.x] + (int64_t)u * ch.pp;  // packed row u
  const int mt = u >> 7, r = u & 127;
  const int rg = (min(kTcBM, ch.pr - mt * kTcBM) + 7) >> 3;
  const int64_t tb = ch.vtc_base + (int64_t)mt * kTcBM * ch.nkct * kTcKC;
  for (int w = threadIdx.x; w < ch.pk; w += blockDim.x) {
    __nv_bfloat16 hv[3];
    split_bf16(src[kcol[ch.pk_off + w]], hv, nt);
    const int64_t o = tb + (int64_t)(w >> 5) * rg * kTcGroup + tc_off(r, w & 31);
    for (int p = 0; p < nt; ++p) v_tc[p * stride + o] = hv[p];
  }
}

// ---- V_pppp generated on the device from the model (CCDGPU_V_ON_THE_FLY) ----------------
// The antisymmetrised <ab|v|cd> of SPBasis::calcTBME, evaluated for every packed element of the
// pp ladder (rows a <= b, columns c < d) and written straight into its operand images, so the
// host never builds or uploads V_pppp.
struct ModelDev {
  int32_t kind, stride;
  const int32_t *qn;   // [n_sp * stride] quantum numbers (SPBasis::indexMap)
  // Electron gas: direct Coulomb term by momentum transfer d = n_a - n_c, d_i in [-R, R],
  // stored by component magnitude: vq[(|dx| W + |dy|) W + |dz|], W = R + 1, built on the host
  // with the reference's own expression (ElectronGasSPBasis.cpp:424-448), so generated elements
  // are bit-identical.  The expression sees each component only through (2 pi d_i / L)^2, and
  // a negated d_i gives the same bits, so the folded table (17.6 KB at R = 12, instead of
  // 125 KB) stays in L1 beside the generators' random reads.
  const double *vq;
  int32_t R, W;
  double g;            // pairing strength
  double Lb;           // PNM box length, (N / rho)^(1/3)
  // Electron gas with |n_i| <= 63: per orbital its momentum components biased by 64 in bytes
  // 0-2 and its spin in byte 3, so that a matrix element reads four words instead of twelve
  // quantum numbers (null otherwise).
  const uint32_t *ocode;
};

__device__ __forceinline__ double direct_pnm_dev(const int32_t *qi, const int32_t *qj,
                                                 const int32_t *qk, const int32_t *ql,
                                                 double Lb) {
  // InfMatterSPBasis.cpp:361-437 (Minnesota), same expression order; exp from CUDA, so the
  // element may differ from the reference's by an ulp.
  const double v0r = 200, v0t = 178, v0s = 91.85;
  const double kr = 1.487, kt = 0.639, ks = 0.465;
  double q2 = 0.;
  for (int i = 0; i < 3; i++) {
    const double ki = 2 * M_PI * qi[i] / Lb, kj = 2 * M_PI * qj[i] / Lb;
    const double kk = 2 * M_PI * qk[i] / Lb, kl = 2 * M_PI * ql[i] / Lb;
    const double bra = __dmul_rn(0.5, ki - kj), ket = __dmul_rn(0.5, kk - kl);
    const double tr = bra - ket;
    q2 = __dadd_rn(q2, __dmul_rn(tr, tr));
  }
  const double L3 = Lb * Lb * Lb;
  const double vr = v0r / L3 * pow(M_PI / kr, 1.5) * exp(-q2 / (4 * kr));
  const double vt = -v0t / L3 * pow(M_PI / kt, 1.5) * exp(-q2 / (4 * kt));
  const double vs = -v0s / L3 * pow(M_PI / ks, 1.5) * exp(-q2 / (4 * ks));
  const double spin_ex = (qi[3] == ql[3] && qj[3] == qk[3]) ? 1 : 0;
  const double iso_ex = (qi[4] == ql[4] && qj[4] == qk[4]) ? 1 : 0;
  const int d_s = (qi[3] == qk[3]) * (qj[3] == ql[3]);
  const int d_t = (qi[4] == qk[4]) * (qj[4] == ql[4]);
  const double is_it = d_s * d_t, ps_it = spin_ex * d_t, ps_pt = spin_ex * iso_ex;
  const double is_pt = d_s * iso_ex;
  return 0.5 * (vr + 0.5 * vt + 0.5 * vs) * is_it + 0.25 * (vt - vs) * ps_it -
         0.5 * (vr + 0.5 * vt + 0.5 * vs) * ps_pt - 0.25 * (vt - vs) * is_pt;
}

// The electron gas's <ab|v|cd> from the orbital codes (ModelDev::ocode): the same table
// entries and the same difference as tbme_dev, so the same value.
__device__ __forceinline__ double eg_tbme_code(const ModelDev &m, uint32_t a, uint32_t b,
                                               uint32_t c, uint32_t d) {
  auto vq = [&](uint32_t x, uint32_t y) {
    const int dx = abs((int)(x & 0xff) - (int)(y & 0xff));
    const int dy = abs((int)((x >> 8) & 0xff) - (int)((y >> 8) & 0xff));
    const int dz = abs((int)((x >> 16) & 0xff) - (int)((y >> 16) & 0xff));
    return __ldg(m.vq + (dx * m.W + dy) * m.W + dz);
  };
  const uint32_t sa = a >> 24, sb = b >> 24, sc = c >> 24, sd = d >> 24;
  const double dir = (sa == sc && sb == sd) ? vq(a, c) : 0.;
  const double exc = (sa == sd && sb == sc) ? vq(a, d) : 0.;
  return dir - exc;
}

// <ab|v|cd> for orbitals a, b, c, d of one regular channel (momentum is conserved).
__device__ __forceinline__ double tbme_dev(const ModelDev &m, int a, int b, int c, int d) {
  const int32_t *qa = m.qn + (int64_t)a * m.stride, *qb = m.qn + (int64_t)b * m.stride;
  const int32_t *qc = m.qn + (int64_t)c * m.stride, *qd = m.qn + (int64_t)d * m.stride;
  if (m.kind == CCDGPU_MODEL_PAIRING) {  // PairingSPBasis.cpp:127-141
    double vout = 0.;
    if (qa[0] == qb[0] && qc[0] == qd[0] && qa[1] == -qb[1] && -qc[1] == qd[1]) {
      vout = -0.5 * m.g;
      if (qa[1] == -qc[1]) vout = -vout;
    }
    return vout;
  }
  if (m.kind == CCDGPU_MODEL_ELECTRON_GAS) {  // direct - exchange, spin diagonal
    auto vq = [&](const int32_t *x, const int32_t *y) {
      return __ldg(m.vq + (abs(x[0] - y[0]) * m.W + abs(x[1] - y[1])) * m.W + abs(x[2] - y[2]));
    };
    const double dir = (qa[3] == qc[3] && qb[3] == qd[3]) ? vq(qa, qc) : 0.;
    const double exc = (qa[3] == qd[3] && qb[3] == qc[3]) ? vq(qa, qd) : 0.;
    return dir - exc;
  }
  return direct_pnm_dev(qa, qb, qc, qd, m.Lb) - direct_pnm_dev(qa, qb, qd, qc, m.Lb);
}

// ---- The other V blocks generated on the device (problem without V blocks) ---------------
// The reference's loaders with SPBasis::calcTBME (load.cpp:112-130, 155-172, 275-318), written
// straight into the solver's layouts.  V_hhhh[ij][kl] = <ij|v|kl>, one CTA per active channel.
__global__ void gen_v_hhhh_kernel(const ChanInfo *__restrict__ chans,
                                  const int2 *__restrict__ hh_pairs, ModelDev m,
                                  double *__restrict__ v_hhhh) {
  const ChanInfo ch = chans[blockIdx.x];
  for (int e = threadIdx.x; e < ch.hh * ch.hh; e += blockDim.x) {
    const int2 ij = hh_pairs[ch.hh_off + e / ch.hh], kl = hh_pairs[ch.hh_off + e % ch.hh];
    v_hhhh[ch.x_off + e] = tbme_dev(m, ij.x, ij.y, kl.x, kl.y);
  }
}

// V_pphh[ab][ij] = V_hhpp[ij][ab] = <ij|v|ab>, over the element ranges of the amplitudes.
__global__ void gen_v_pphh_kernel(const ElemRange *__restrict__ ranges,
                                  const ChanInfo *__restrict__ chans,
                                  const int2 *__restrict__ pp_pairs,
                                  const int2 *__restrict__ hh_pairs, ModelDev m,
                                  double *__restrict__ v_pphh) {
  const ElemRange rg = ranges[blockIdx.x];
  const ChanInfo ch = chans[rg.ch];
  for (int64_t e = rg.e0 + threadIdx.x; e < rg.e1; e += blockDim.x) {
    const int64_t loc = e - ch.t_off;
    const int ab = (int)(loc / ch.hh), ij = (int)(loc - (int64_t)ab * ch.hh);
    const int2 pab = pp_pairs[ch.pp_off + ab], pij = hh_pairs[ch.hh_off + ij];
    v_pphh[e] = tbme_dev(m, pij.x, pij.y, pab.x, pab.y);
  }
}

// The three-body V of the table path (load.cpp:241-273): vnn_h_hpp[k][(j,a,b)] = <kj|v|ab>
// over (a, b) in pp(ch(k, j)), vnn_phh_p[a][(b,i,j)] = <ij|v|ab> over (i, j) in hh(ch(a, b)),
// the blocks of hpp(k) and phh(a) ordered by j and b (offsets hblk, pblk of the table
// derivation).  One CTA per active channel: its hh pairs (k, j) with its pp pairs, and its pp
// pairs (a, b) with its hh pairs.  A position outside its chain (three-body dimensions that do
// not match the channel maps) is not written and sets kErrBadIndex.
__global__ void gen_v3_kernel(const ChanInfo *__restrict__ chans, const int2 *__restrict__ pp_pairs,
                              const int2 *__restrict__ hh_pairs, ModelDev m,
                              const int64_t *__restrict__ o_h, const int64_t *__restrict__ o_p,
                              const int32_t *__restrict__ hblk, const int32_t *__restrict__ pblk,
                              int np, int npart, double *__restrict__ v_h_hpp,
                              double *__restrict__ v_phh_p, int32_t *err) {
  const ChanInfo ch = chans[blockIdx.x];
  const int n1 = ch.hh * ch.pp;
  for (int e = threadIdx.x; e < n1; e += blockDim.x) {
    const int x = e / ch.pp, ab = e - x * ch.pp;
    const int2 kj = hh_pairs[ch.hh_off + x], pab = pp_pairs[ch.pp_off + ab];
    const int64_t f = o_h[kj.x] + hblk[(int64_t)kj.x * np + kj.y] + ab;
    if (f < o_h[kj.x + 1]) v_h_hpp[f] = tbme_dev(m, kj.x, kj.y, pab.x, pab.y);
    else atomicOr(err, kErrBadIndex);
  }
  for (int e = threadIdx.x; e < n1; e += blockDim.x) {
    const int y = e / ch.hh, ij = e - y * ch.hh;
    const int2 pab = pp_pairs[ch.pp_off + y], pij = hh_pairs[ch.hh_off + ij];
    const int a = pab.x - np, b = pab.y - np;
    const int64_t f = o_p[a] + pblk[(int64_t)a * npart + b] + ij;
    if (f < o_p[a + 1]) v_phh_p[f] = tbme_dev(m, pij.x, pij.y, pab.x, pab.y);
    else atomicOr(err, kErrBadIndex);
  }
}

// Per active modified channel (channel order): its block offsets and where its ph' pairs (b, j)
// and hp' pairs (i, a) start in the pair arrays.
struct ModGen {
  int32_t ph, hp;
  int64_t m_off, y_off, ph_off, hp_off;
};

// One CTA per active modified channel:
//   V_hpph' (load.cpp:275-296): [(i,a)][(b,j)] = <ij|v|ab>, stored transposed (ph' x hp') as the
//     ring reads it;
//   V_hphp' (load.cpp:298-318): [(i,b)][(j,a)] = <ia|v|bj>.
__global__ void gen_v_mod_kernel(const ModGen *__restrict__ mods, const int2 *__restrict__ ph_pairs,
                                 const int2 *__restrict__ hp_pairs, ModelDev m,
                                 double *__restrict__ v_hpph_t, double *__restrict__ v_hphp) {
  const ModGen g = mods[blockIdx.x];
  for (int e = threadIdx.x; e < g.ph * g.hp; e += blockDim.x) {
    const int k = e / g.hp, x = e - k * g.hp;  // ph' row k, hp' column x
    const int2 bj = ph_pairs[g.ph_off + k], ia = hp_pairs[g.hp_off + x];
    v_hpph_t[g.m_off + e] = tbme_dev(m, ia.x, bj.y, ia.y, bj.x);
  }
  for (int e = threadIdx.x; e < g.hp * g.hp; e += blockDim.x) {
    const int x = e / g.hp, y = e - x * g.hp;
    const int2 ib = hp_pairs[g.hp_off + x], ja = hp_pairs[g.hp_off + y];
    v_hphp[g.y_off + e] = tbme_dev(m, ib.x, ja.y, ib.y, ja.x);
  }
}

// The (particle a, hole i) -> modified-channel lookup that derive_tables_kernel reads, from
// the ph' (a, i) and hp' (i, a) pair lists of the generated-V path (their ranges checked on the
// host): slot (a - np) * np + i holds (channel, ph' index, channel, hp' index).  One CTA per
// active modified channel; the slots start at -1 and each half is claimed once (atomicCAS), so
// a pair named twice sets kErrBadIndex.
__global__ void mod_lookup_kernel(const ModGen *__restrict__ mods, const int32_t *__restrict__ chan,
                                  const int2 *__restrict__ ph_pairs,
                                  const int2 *__restrict__ hp_pairs, int np, int4 *mlook,
                                  int32_t *err) {
  const ModGen g = mods[blockIdx.x];
  const int c = chan[blockIdx.x];
  for (int k = threadIdx.x; k < g.ph; k += blockDim.x) {
    const int2 ai = ph_pairs[g.ph_off + k];
    int *m = reinterpret_cast<int *>(mlook + (int64_t)(ai.x - np) * np + ai.y);
    if (atomicCAS(m, -1, c) != -1) atomicOr(err, kErrBadIndex);
    else m[1] = k;
  }
  for (int k = threadIdx.x; k < g.hp; k += blockDim.x) {
    const int2 ia = hp_pairs[g.hp_off + k];
    int *m = reinterpret_cast<int *>(mlook + (int64_t)(ia.y - np) * np + ia.x) + 2;
    if (atomicCAS(m, -1, c) != -1) atomicOr(err, kErrBadIndex);
    else m[1] = k;
  }
}

// E_ref and the normal-ordered single-particle energies from the bare ones (SPBasis.cpp:7-40).
// Thread p < nsp: e_p + sum_{j < nh} <pj|v|pj>, summed in the reference's order.  Thread nsp:
// E_ref = sum_{i,j < nh} 0.5 <ij|v|ij> + sum_{i < nh} e_i, one running sum in the reference's
// order, so its rounding matches.  out holds nsp energies, then E_ref.
__global__ void normal_order_kernel(ModelDev m, const double *__restrict__ bare, int nsp, int nh,
                                    double *__restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < nsp) {
    double e = bare[p];
    for (int j = 0; j < nh; ++j) e += tbme_dev(m, p, j, p, j);
    out[p] = e;
  } else if (p == nsp) {
    double eref = 0.;
    for (int i = 0; i < nh; ++i)
      for (int j = 0; j < nh; ++j) eref += 0.5 * tbme_dev(m, i, j, i, j);
    for (int i = 0; i < nh; ++i) eref += bare[i];
    out[nsp] = eref;
  }
}


// V_pppp generated straight into the ladders' operand images, one CTA per image chunk, so that
// each CTA writes one contiguous block (the chunk's elements in image order; padding rows and
// K columns past pk get zeros).  FP64 ladder: items (channel, row tile, 16-deep K chunk), block
// of ar x kBK doubles, k-major (mid and wide classes) or XOR-swizzled rows (thin class).  The
// tensor-core images of mixed handles come with the FP64 tiles from gen_v_both_chunks_kernel.
template <bool EG>  // EG: the electron gas's orbital-code path only (fewer registers)
__global__ void __launch_bounds__(256)
gen_v_chunks_kernel(const ChanInfo *__restrict__ chans, const int4 *__restrict__ items,
                    const int32_t *__restrict__ rowmap, const int32_t *__restrict__ kcol,
                    const int2 *__restrict__ pp_pairs, ModelDev m, double *__restrict__ v_t) {
  __shared__ uint2 s_ab[kMaxBM];  // electron gas: orbital codes of the chunk's rows (a, b)
  __shared__ uint2 s_cd[kBK];     // ... and of its K columns (c, d)
  const int4 it = items[blockIdx.x];
  const ChanInfo ch = chans[it.x];
  const int mt = it.y, kc = it.z;
  const int rows = min(ch.bm, ch.pr - mt * ch.bm), ar = ladder_arows(ch.nb, rows);
  const bool kmajor = ladder_kmajor(ch.nb);
  double *out = v_t + ch.vkt_base + (int64_t)mt * ladder_arows_full(ch.nb) * ch.nkc * kBK +
                (int64_t)kc * ar * kBK;
  if (EG) {  // the codes once per chunk, not once per element
    for (int r = threadIdx.x; r < rows; r += blockDim.x) {
      const int2 ab = pp_pairs[ch.pp_off + rowmap[ch.row_off + mt * ch.bm + r]];
      s_ab[r] = make_uint2(m.ocode[ab.x], m.ocode[ab.y]);
    }
    for (int k = threadIdx.x; k < kBK; k += blockDim.x) {
      const int w = kc * kBK + k;
      if (w < ch.pk) {
        const int2 cd = pp_pairs[ch.pp_off + kcol[ch.pk_off + w]];
        s_cd[k] = make_uint2(m.ocode[cd.x], m.ocode[cd.y]);
      }
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < ar * kBK; e += blockDim.x) {
    int r, k;
    if (kmajor) {
      k = e / ar;
      r = e - k * ar;
    } else {
      r = e >> 4;
      k = (e & 15) ^ (r & 15);  // swzA(r, k) = 16 r + (k ^ (r & 15))
    }
    const int u = mt * ch.bm + r, w = kc * kBK + k;
    double v = 0.0;
    if (r < rows && w < ch.pk) {
      if constexpr (EG) {
        v = eg_tbme_code(m, s_ab[r].x, s_ab[r].y, s_cd[k].x, s_cd[k].y);
      } else {
        const int2 ab = pp_pairs[ch.pp_off + rowmap[ch.row_off + u]];
        const int2 cd = pp_pairs[ch.pp_off + kcol[ch.pk_off + w]];
        v = tbme_dev(m, ab.x, ab.y, cd.x, cd.y);
      }
    }
    out[e] = v;
  }
}

// Mixed handles with generated V: both images from one evaluation of each element.  Items are
// the tensor-core chunks (channel, 128-row tile, 32-deep K chunk); the FP64 ladder's row tiles
// are also 128 rows (ladder_bm), so a chunk covers FP64 K chunks 2 kc and 2 kc + 1 of the same
// rows.  The CTA evaluates its 128 x 32 elements once into shared memory (k-major, row stride
// kGenLd; zero past the channel's rows and columns), four per thread at a time, then writes
// the NT bf16 terms of each element in the tensor core's K-major core-matrix order (8 x 8
// blocks, block of 8 rows by 32 K contiguous) and the FP64 chunks in the order of
// gen_v_chunks_kernel (padding included).
// EG: the electron gas's orbital-code path only (m.ocode set), without the other models' element
// code, so the instantiation needs fewer registers and more CTAs share an SM.
constexpr int kGenLd = kTcBM + 4;
template <int NT, bool EG>
__global__ void __launch_bounds__(256)
gen_v_both_chunks_kernel(const ChanInfo *__restrict__ chans, const int4 *__restrict__ items,
                         const int32_t *__restrict__ rowmap, const int32_t *__restrict__ kcol,
                         const int2 *__restrict__ pp_pairs, ModelDev m, double *__restrict__ v_t,
                         __nv_bfloat16 *__restrict__ v_tc, int64_t tc_stride) {
  __shared__ uint2 s_ab[kTcBM];
  __shared__ uint2 s_cd[kTcKC];
  __shared__ double tile[kTcKC * kGenLd];  // tile[k * kGenLd + r]
  const int4 it = items[blockIdx.x];
  const ChanInfo ch = chans[it.x];
  const int mt = it.y, kc = it.z;
  const int rows = min(kTcBM, ch.pr - mt * kTcBM), rg = (rows + 7) >> 3;
  if (EG) {
    for (int r = threadIdx.x; r < rows; r += blockDim.x) {
      const int2 ab = pp_pairs[ch.pp_off + rowmap[ch.row_off + mt * kTcBM + r]];
      s_ab[r] = make_uint2(m.ocode[ab.x], m.ocode[ab.y]);
    }
    for (int k = threadIdx.x; k < kTcKC; k += blockDim.x) {
      const int w = kc * kTcKC + k;
      if (w < ch.pk) {
        const int2 cd = pp_pairs[ch.pp_off + kcol[ch.pk_off + w]];
        s_cd[k] = make_uint2(m.ocode[cd.x], m.ocode[cd.y]);
      }
    }
    __syncthreads();
  }
  // Evaluate: element e -> (r = e % 128, k = e / 128), 4096 per chunk, 16 per thread.
  constexpr int kPer = kTcBM * kTcKC / 256;
  for (int j0 = 0; j0 < kPer; j0 += 4) {
    double v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = (j0 + q) * 256 + threadIdx.x;
      const int r = e & (kTcBM - 1), k = e >> 7;
      const int w = kc * kTcKC + k;
      v[q] = 0.0;
      if (r < rows && w < ch.pk) {
        if constexpr (EG) {
          v[q] = eg_tbme_code(m, s_ab[r].x, s_ab[r].y, s_cd[k].x, s_cd[k].y);
        } else {
          const int2 ab = pp_pairs[ch.pp_off + rowmap[ch.row_off + mt * kTcBM + r]];
          const int2 cd = pp_pairs[ch.pp_off + kcol[ch.pk_off + w]];
          v[q] = tbme_dev(m, ab.x, ab.y, cd.x, cd.y);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = (j0 + q) * 256 + threadIdx.x;
      tile[(e >> 7) * kGenLd + (e & (kTcBM - 1))] = v[q];
    }
  }
  __syncthreads();
  // bf16 terms: e = (r / 8) kTcGroup + (k / 8) 64 + (r % 8) 8 + k % 8 (tc_off).
  const int64_t base = ch.vtc_base + (int64_t)mt * kTcBM * ch.nkct * kTcKC + (int64_t)kc * rg * kTcGroup;
  for (int e = threadIdx.x; e < rg * kTcGroup; e += blockDim.x) {
    const int rem = e & (kTcGroup - 1);
    const int r = (e / kTcGroup) * 8 + ((rem >> 3) & 7), k = (rem >> 6) * 8 + (rem & 7);
    __nv_bfloat16 hv[NT];
    split_bf16_n<NT>(tile[k * kGenLd + r], hv);
#pragma unroll
    for (int p = 0; p < NT; ++p) v_tc[p * tc_stride + base + e] = hv[p];
  }
  // FP64 chunks 2 kc and 2 kc + 1, as gen_v_chunks_kernel (rows past `rows` are zero).
  const int ar = ladder_arows(ch.nb, rows);
  const bool kmajor = ladder_kmajor(ch.nb);
  for (int h = 0; h < 2; ++h) {
    const int kc64 = 2 * kc + h;
    if (kc64 >= ch.nkc) break;
    double *out = v_t + ch.vkt_base + (int64_t)mt * ladder_arows_full(ch.nb) * ch.nkc * kBK +
                  (int64_t)kc64 * ar * kBK;
    for (int e = threadIdx.x; e < ar * kBK; e += blockDim.x) {
      int r, k;
      if (kmajor) {
        k = e / ar;
        r = e - k * ar;
      } else {
        r = e >> 4;
        k = (e & 15) ^ (r & 15);  // swzA(r, k) = 16 r + (k ^ (r & 15))
      }
      out[e] = r < rows ? tile[(h * kBK + k) * kGenLd + r] : 0.0;
    }
  }
}

// The fused assembly's row table (one CTA per active channel): for each packed row u with
// a < b (row ab, mirror row ba), at the row's index among those rows (its K index qx), the
// offsets of rows ab and ba in the channel block, its operand-image indices, the particle
// indices and energies.
__global__ void __launch_bounds__(256)
quad_rows_kernel(const ChanInfo *__restrict__ chans, const int32_t *__restrict__ rowmap,
                 const int32_t *__restrict__ mirror, const int2 *__restrict__ pk_idx,
                 const int2 *__restrict__ pp_pairs, const double *__restrict__ eps, int np,
                 QuadRow *__restrict__ out) {
  const ChanInfo ch = chans[blockIdx.x];
  for (int u = threadIdx.x; u < ch.pr; u += blockDim.x) {
    const int ab = rowmap[ch.row_off + u], ba = mirror[ch.row_off + u];
    if (ba < 0) continue;  // a = b: zero row
    const int2 q = pk_idx[ch.pp_off + ab], pab = pp_pairs[ch.pp_off + ab];
    QuadRow r;
    r.o_ab = ab * ch.hh;
    r.o_ba = ba * ch.hh;
    r.qx = q.x;
    r.qy = q.y;
    r.pa = pab.x - np;
    r.pb = pab.y - np;
    r.ea = eps[pab.x];
    r.eb = eps[pab.y];
    out[ch.qrow_off + q.x] = r;
  }
}

// The eight loadMaps tables -> int32 flat offsets into their target chains, with range checks
// and, for the five tables that are also scatter targets (mapToDistributed), hit counts that
// check_counts_kernel then requires to be exactly one.
struct TableGeometry {
  const int64_t *o_h;      // [np+1] hpp chain offsets
  const int64_t *o_p;      // [npart+1] phh chain offsets
  const int64_t *o_m;      // [nch+1] phhp chain offsets
  const int2 *mod_dims;    // [nch] (ph', hp')
  uint64_t nch, np, npart;
};

__global__ void convert_tables_kernel(const ElemRange *__restrict__ ranges, const RawIndex *raw,
                                      int64_t n_t, TableGeometry geo, int32_t *__restrict__ flat,
                                      int32_t *__restrict__ counts, int32_t *err) {
  const ElemRange rg = ranges[blockIdx.x];
  for (int64_t e = rg.e0 + threadIdx.x; e < rg.e1; e += blockDim.x) {
#pragma unroll 1
    for (int k = 0; k < 8; ++k) {
      const RawIndex x = raw[(int64_t)k * n_t + e];
      int64_t f = -1;
      if (k <= 1) {
        if (x.channel < geo.np && x.column == 0 &&
            x.row < (uint64_t)(geo.o_h[x.channel + 1] - geo.o_h[x.channel]))
          f = geo.o_h[x.channel] + (int64_t)x.row;
      } else if (k <= 3) {
        if (x.channel < geo.npart && x.row == 0 &&
            x.column < (uint64_t)(geo.o_p[x.channel + 1] - geo.o_p[x.channel]))
          f = geo.o_p[x.channel] + (int64_t)x.column;
      } else if (x.channel < geo.nch) {
        const int2 md = geo.mod_dims[x.channel];
        if (x.row < (uint64_t)md.x && x.column < (uint64_t)md.y)
          f = geo.o_m[x.channel] + (int64_t)x.row * md.y + (int64_t)x.column;
      }
      if (f < 0 || f >= n_t) {
        atomicOr(err, kErrBadIndex);
        f = 0;
      }
      flat[(int64_t)k * n_t + e] = (int32_t)f;
      if (k <= 4) atomicAdd(&counts[(int64_t)k * n_t + f], 1);
    }
  }
}

// ---- Remap tables derived on the device (problem without loadMaps tables) ----------------
// loadMaps (load.cpp:389-532) builds the eight tables from the channel maps alone; the same
// derivation here needs only the pair lists the solver already holds.  Block sizes first:
// hsz[k * np + j] = pp of the channel of hole pair (k, j), psz[(a - np) * npart + (b - np)] =
// hh of the channel of particle pair (a, b) (zero for pairs of channels without amplitudes).
// One CTA per active channel.
__global__ void pair_sizes_kernel(const ChanInfo *__restrict__ chans, const int2 *__restrict__ pp_pairs,
                                  const int2 *__restrict__ hh_pairs, int np, int npart,
                                  int32_t *__restrict__ hsz, int32_t *__restrict__ psz) {
  const ChanInfo ch = chans[blockIdx.x];
  for (int t = threadIdx.x; t < ch.pp; t += blockDim.x) {
    const int2 ab = pp_pairs[ch.pp_off + t];
    psz[(int64_t)(ab.x - np) * npart + (ab.y - np)] = ch.hh;
  }
  for (int t = threadIdx.x; t < ch.hh; t += blockDim.x) {
    const int2 ij = hh_pairs[ch.hh_off + t];
    hsz[(int64_t)ij.x * np + ij.y] = ch.pp;
  }
}

// In-place exclusive prefix sum of each row (one CTA of 256 threads per row): block sizes ->
// offsets of the blocks inside the three-body chains hpp(k) (SPBasis.cpp:181-256) and phh(a)
// (SPBasis.cpp:443-563), whose blocks follow the partner index in ascending order.
__global__ void __launch_bounds__(256) row_scan_kernel(int32_t *__restrict__ x, int len) {
  __shared__ int32_t warp_tot[8];
  int32_t *row = x + (int64_t)blockIdx.x * len;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int32_t carry = 0;
  for (int base = 0; base < len; base += 256) {
    const int k = base + threadIdx.x;
    const int32_t v = k < len ? row[k] : 0;
    int32_t sum = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t y = __shfl_up_sync(0xffffffffu, sum, o);
      if (lane >= o) sum += y;
    }
    if (lane == 31) warp_tot[w] = sum;
    __syncthreads();
    int32_t before = 0, tile = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      before += q < w ? warp_tot[q] : 0;
      tile += warp_tot[q];
    }
    if (k < len) row[k] = carry + before + sum - v;
    carry += tile;
    __syncthreads();
  }
}

struct DeriveGeometry {
  const int64_t *o_h;      // [np+1] hpp chain offsets
  const int64_t *o_p;      // [npart+1] phh chain offsets
  const int64_t *o_m;      // [nch+1] phhp chain offsets
  const int2 *mod_dims;    // [nch] (ph', hp')
  const int32_t *hblk;     // [np * np] offset of the block of hole j inside hpp(k)
  const int32_t *pblk;     // [npart * npart] offset of the block of particle b inside phh(a)
  const int4 *mlook;       // [npart * np] of (particle a, hole i): x, y = modified channel and
                           // row of (a, i) in its ph' map; z, w = channel and column of (i, a)
                           // in its hp' map (-1 where the pair is in no active channel)
  int32_t np, npart;
};

// The eight tables as int32 flat offsets, from the pair lists (load.cpp:469-526):
//   iab_j -> hpp(j) at block i, row ab;     jab_i -> hpp(i) at block j, row ab;
//   a_bij -> phh(a) at block b, column ij;  b_aij -> phh(b) at block a, column ij;
//   ai_jb, aj_ib, bi_ja, bj_ia -> phhp block of the modified channel of the ph' pair, at
//   (row of the ph' pair, column of the hp' pair).
// Range checks and hit counts as for convert_tables_kernel.
__global__ void derive_tables_kernel(const ElemRange *__restrict__ ranges,
                                     const ChanInfo *__restrict__ chans,
                                     const int2 *__restrict__ pp_pairs,
                                     const int2 *__restrict__ hh_pairs, DeriveGeometry g,
                                     int64_t n_t, int32_t *__restrict__ flat,
                                     int32_t *__restrict__ counts, int32_t *err) {
  const ElemRange rg = ranges[blockIdx.x];
  const ChanInfo ch = chans[rg.ch];
  const int np = g.np, npart = g.npart;
  auto hole_chain = [&](int k, int j, int ab) -> int64_t {
    const int64_t f = g.o_h[k] + g.hblk[(int64_t)k * np + j] + ab;
    return f < g.o_h[k + 1] ? f : -1;
  };
  auto part_chain = [&](int a, int b, int ij) -> int64_t {
    const int64_t f = g.o_p[a] + g.pblk[(int64_t)a * npart + b] + ij;
    return f < g.o_p[a + 1] ? f : -1;
  };
  // (x, y): particle-hole pair of the ph' map; (u, v): hole-particle pair of the hp' map.
  auto ring = [&](int x, int y, int u, int v) -> int64_t {
    const int4 r = g.mlook[(int64_t)(x - np) * np + y], c = g.mlook[(int64_t)(v - np) * np + u];
    if (r.x < 0 || r.x != c.z) return -1;
    const int2 md = g.mod_dims[r.x];
    if (r.y >= md.x || c.w < 0 || c.w >= md.y) return -1;
    return g.o_m[r.x] + (int64_t)r.y * md.y + c.w;
  };
  for (int64_t e = rg.e0 + threadIdx.x; e < rg.e1; e += blockDim.x) {
    const int64_t loc = e - ch.t_off;
    const int ab = (int)(loc / ch.hh), ij = (int)(loc - (int64_t)ab * ch.hh);
    const int2 pab = pp_pairs[ch.pp_off + ab], pij = hh_pairs[ch.hh_off + ij];
    const int a = pab.x, b = pab.y, i = pij.x, j = pij.y;
    int64_t f[8];
    f[0] = hole_chain(j, i, ab);
    f[1] = hole_chain(i, j, ab);
    f[2] = part_chain(a - np, b - np, ij);
    f[3] = part_chain(b - np, a - np, ij);
    f[4] = ring(a, i, j, b);
    f[5] = ring(a, j, i, b);
    f[6] = ring(b, i, j, a);
    f[7] = ring(b, j, i, a);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      int64_t x = f[k];
      if (x < 0 || x >= n_t) {
        atomicOr(err, kErrBadIndex);
        x = 0;
      }
      flat[(int64_t)k * n_t + e] = (int32_t)x;
      if (k <= 4) atomicAdd(&counts[(int64_t)k * n_t + x], 1);
    }
  }
}

// V_hpph' blocks (hp' x ph', load.cpp:275-296) -> transposed (ph' x hp') for the ring kernels'
// outer-product loops; one CTA per modified channel.
__global__ void transpose_hpph_kernel(const ModInfo *__restrict__ mods,
                                      const double *__restrict__ raw, double *__restrict__ out) {
  const ModInfo m = mods[blockIdx.x];
  for (int e = threadIdx.x; e < m.ph * m.hp; e += blockDim.x) {
    const int i = e / m.ph, k = e - i * m.ph;
    out[m.m_off + (int64_t)k * m.hp + i] = raw[m.m_off + e];
  }
}

// Fused-path ring tables.  inv[ai_jb(e)] = e turns the phhp slab position of every amplitude
// back into its pphh element, so the ring can read T' from the amplitudes and write R in pphh
// order.  The other three ring maps of loadMaps are ai_jb composed with the swaps i<->j and
// a<->b (load.cpp:469-526 builds all four from the same (a,i),(j,b) pairing); this is checked
// here, since the fused assembly reads R_aj,ib, R_bi,ja and R_bj,ia at (ab,ji), (ba,ij) and
// (ba,ji) of the pphh-ordered R.
__global__ void ring_maps_kernel(const ElemRange *__restrict__ ranges,
                                 const ChanInfo *__restrict__ chans,
                                 const int32_t *__restrict__ pp_swap,
                                 const int32_t *__restrict__ hh_swap,
                                 const int32_t *__restrict__ flat, int64_t n_t,
                                 int32_t *__restrict__ inv, int32_t *err) {
  const ElemRange rg = ranges[blockIdx.x];
  const ChanInfo ch = chans[rg.ch];
  for (int64_t e = rg.e0 + threadIdx.x; e < rg.e1; e += blockDim.x) {
    const int64_t loc = e - ch.t_off;
    const int ab = (int)(loc / ch.hh), ij = (int)(loc - (int64_t)ab * ch.hh);
    const int ps = pp_swap[ch.pp_off + ab], hs = hh_swap[ch.hh_off + ij];
    const int64_t e_ji = ch.t_off + (int64_t)ab * ch.hh + hs;
    const int64_t e_ba = ch.t_off + (int64_t)ps * ch.hh + ij;
    const int64_t e_baji = ch.t_off + (int64_t)ps * ch.hh + hs;
    const int32_t f = flat[4 * n_t + e];
    inv[f] = (int32_t)e;
    if (flat[5 * n_t + e] != flat[4 * n_t + e_ji] || flat[6 * n_t + e] != flat[4 * n_t + e_ba] ||
        flat[7 * n_t + e] != flat[4 * n_t + e_baji])
      atomicOr(err, kErrRingMaps);
  }
}

__global__ void check_counts_kernel(const int32_t *__restrict__ counts, int64_t n, int32_t *err) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (counts[i] != 1) atomicOr(err, kErrBadIndex);
}

}  // namespace ccd
