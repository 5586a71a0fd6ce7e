// CCD iteration kernels for sm_100a (FP64 path).
//
// Reference correspondence (calc.cpp / Chain.hpp of justinlietz/coupled_cluster_doubles):
//   pp_ladder_kernel        D = 0.5 T X + 0.5 V_pppp T              calc.cpp:162-202
//                           (antisymmetry-packed, FP64 FMA pipe)
//   hh_ladder_kernel        X = V_hhhh + 0.5 V_hhpp T                calc.cpp:141-160
//   ring_*_kernel           Y = V_hphp + 0.5 V_hpph T'; R = T' Y     calc.cpp:264-313
//   onebody_tables_kernel   calcChannelT2Diff_h2pp_h1 / _p2_p1hh     calc.cpp:9-25, 73-89
//   onebody_fused_kernel    the same dot products, read from the ladder intermediates
//   gather8_kernel          Chain::mapFromDistributed x 8            Chain.hpp:710-755
//   assemble_*_kernel       calcChannelT2_pphh                       calc.cpp:368-421
//   map_to_kernel           Chain::set + mapToDistributed x 5        Chain.hpp:503-527,757-802
//   energy_kernel           reduction(+:corr) + MPI_Allreduce + stop rule, main.cpp:511-519,668-670
#pragma once

#include <cstdint>

#include "ccd_device.cuh"

namespace ccd {

constexpr uint32_t kSpinLimit = 1u << 24;  // bounded mbarrier waits (~1 s with backoff)

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait on an mbarrier phase; false once the spin budget is spent.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (uint32_t it = 0; it < kSpinLimit; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (it > 32) __nanosleep(64);
  }
  return false;
}
// 1-D bulk copy global -> shared, completion counted on an mbarrier (TMA unit, no multicast).
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes,
                                         uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
__device__ __forceinline__ bool skip_iteration(const Control *ctl) {
  return ctl->active && ctl->done;
}

// ------------------------------------------------------------------------------------------
// pp ladder + hh-ladder output on the FP64 FMA pipe:
//   D[ab,:] = sum_{c<d} V[ab,cd] T[cd,:] + T[ab,:] (X/2)     for packed rows a <= b,
//   D[ba,:] = -D[ab,:]                                        (antisymmetry of V and T).
// Warp 4 is the producer: one lane streams pre-tiled A/B stages with bulk copies (TMA, no
// multicast) into a kStages-deep shared-memory ring guarded by mbarriers.  The 128 consumer
// threads each own `cg` rows x 8 columns of the tile and run register-blocked DFMAs; V rows
// come from shared memory conflict-free (XOR swizzle), T / X columns are warp broadcasts.
// K runs over the c<d pairs (V T) and then over hh (T X) with the same pipeline.
// ------------------------------------------------------------------------------------------
template <int CG>
__device__ __forceinline__ void ladder_consume(const LadderTile &tile, const double *As,
                                               const double *Bs, uint64_t *bars, int tid,
                                               const int32_t *__restrict__ rowmap,
                                               const int32_t *__restrict__ mirror,
                                               double *__restrict__ d, int32_t *err) {
  constexpr int TM = CG, RG = kLadderConsumers / CG, NB = 8 * CG;
  const int rg = tid / CG, cg = tid - rg * CG;
  const bool worker = rg < RG;
  const int lane = tid & 31;
  double acc[TM][8];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
  const int nchunks = tile.nkc + tile.nkh;
  for (int c = 0; c < nchunks; ++c) {
    const int s = c % kStages;
    if (!mbar_wait(smem_u32(&bars[s]), (c / kStages) & 1)) {
      atomicOr(err, kErrTimeout);
      return;
    }
    const double *A = As + s * (kMaxBM * kBK);
    const double *B = Bs + s * (kBK * kMaxCG * 8);
    if (worker) {
#pragma unroll 4
      for (int k = 0; k < kBK; ++k) {
        double a[TM];
#pragma unroll
        for (int i = 0; i < TM; ++i) a[i] = A[swzA(rg + i * RG, k)];
        const double2 *bp = reinterpret_cast<const double2 *>(B + k * NB + cg * 8);
        double b[8];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const double2 v = bp[j];
          b[2 * j] = v.x;
          b[2 * j + 1] = v.y;
        }
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
          for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(smem_u32(&bars[kStages + s]));
  }
  if (!worker) return;
  double *dblk = d + tile.t_off;
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    const int u = tile.mt * tile.bm + rg + i * RG;
    if (u >= tile.pr) continue;
    const int ab = rowmap[tile.row_off + u], mir = mirror[tile.row_off + u];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int col = cg * 8 + j;
      if (col < tile.hh) {
        dblk[(int64_t)ab * tile.hh + col] = acc[i][j];
        if (mir >= 0) dblk[(int64_t)mir * tile.hh + col] = -acc[i][j];
      }
    }
  }
}

// CG_LO..CG_HI: the column-group range a launch handles (separate instantiations keep the
// register budget of narrow channels independent of the 72-column case).
template <int CG_LO, int CG_HI>
__global__ void __launch_bounds__(kLadderThreads, 2)
pp_ladder_kernel(const LadderTile *__restrict__ tiles, const double *__restrict__ v_t,
                 const double *__restrict__ t_kt, const double *__restrict__ t_mt,
                 const double *__restrict__ x_t, const int32_t *__restrict__ rowmap,
                 const int32_t *__restrict__ mirror, double *__restrict__ d, const Control *ctl,
                 int32_t *err) {
  if (skip_iteration(ctl)) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double *As = reinterpret_cast<double *>(smem_raw);
  double *Bs = As + kStages * kMaxBM * kBK;
  uint64_t *bars = reinterpret_cast<uint64_t *>(Bs + kStages * kBK * kMaxCG * 8);
  const LadderTile tile = tiles[blockIdx.x];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(smem_u32(&bars[s]), 1);
      mbar_init(smem_u32(&bars[kStages + s]), kLadderConsumers / 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  if (warp == kLadderConsumers / 32) {
    if (lane == 0) {
      const int nb = 8 * tile.cg;
      const uint32_t abytes = tile.bm * kBK * 8, bbytes = kBK * nb * 8;
      const int nchunks = tile.nkc + tile.nkh;
      for (int c = 0; c < nchunks; ++c) {
        const int s = c % kStages;
        if (c >= kStages && !mbar_wait(smem_u32(&bars[kStages + s]), ((c / kStages) - 1) & 1)) {
          atomicOr(err, kErrTimeout);
          break;
        }
        const double *asrc, *bsrc;
        if (c < tile.nkc) {
          asrc = v_t + tile.v_base + (int64_t)(tile.mt * tile.nkc + c) * tile.bm * kBK;
          bsrc = t_kt + tile.tkt_base + (int64_t)c * kBK * nb;
        } else {
          const int kh = c - tile.nkc;
          asrc = t_mt + tile.tmt_base + (int64_t)(tile.mt * tile.nkh + kh) * tile.bm * kBK;
          bsrc = x_t + tile.xt_base + (int64_t)kh * kBK * nb;
        }
        const uint32_t full = smem_u32(&bars[s]);
        mbar_expect_tx(full, abytes + bbytes);
        bulk_g2s(smem_u32(As + s * kMaxBM * kBK), asrc, abytes, full);
        bulk_g2s(smem_u32(Bs + s * kBK * kMaxCG * 8), bsrc, bbytes, full);
      }
    }
    return;
  }
  const int tid = threadIdx.x;
#define CCD_LADDER_CASE(n) \
  case n: if (n >= CG_LO && n <= CG_HI) ladder_consume<n>(tile, As, Bs, bars, tid, rowmap, mirror, d, err); break;
  switch (tile.cg) {
    CCD_LADDER_CASE(1) CCD_LADDER_CASE(2) CCD_LADDER_CASE(3) CCD_LADDER_CASE(4)
    CCD_LADDER_CASE(5) CCD_LADDER_CASE(6) CCD_LADDER_CASE(7) CCD_LADDER_CASE(8)
    CCD_LADDER_CASE(9)
    default: break;
  }
#undef CCD_LADDER_CASE
}

// ------------------------------------------------------------------------------------------
// hh ladder intermediate, split over 64-row K slices of each channel:
//   P = V_hhpp T (K = pp),  X = V_hhhh + 0.5 P  (reference layout, and X/2 as B tiles),
//   s[IJ] = P[IJ][IJ]            (x_k = sum over IJ with first hole k, calc.cpp:82-84),
//   r[AB] = sum_IJ V[IJ][AB] T[AB][IJ]  (y_a = sum over AB with first particle a, calc.cpp:18-20).
// Each CTA writes its slice's partial P; the last CTA of a channel (atomic ticket) sums the
// partials in slice order, so the result does not depend on scheduling.  V_hhpp is held
// transposed (pp x hh) so a slice is one contiguous stretch, like the T slice.
// ------------------------------------------------------------------------------------------
constexpr int kHHThreads = 256;
constexpr int kHHRows = 64;
constexpr int kHHAcc = 21;  // (72*72)/256 rounded up

__global__ void __launch_bounds__(kHHThreads)
hh_ladder_kernel(const HHTile *__restrict__ tiles, const ChanInfo *__restrict__ chans,
                 const double *__restrict__ v_pphh, const double *__restrict__ v_hhhh,
                 const double *tbuf0, const double *tbuf1, double *part, int32_t *counters,
                 double *__restrict__ x_ref, double *__restrict__ x_t, double *__restrict__ s_out,
                 double *__restrict__ r_out, const Control *ctl) {
  if (skip_iteration(ctl)) return;
  extern __shared__ __align__(16) double hsm[];
  __shared__ int last;
  const HHTile tt = tiles[blockIdx.x];
  const ChanInfo ch = chans[tt.ch];
  const double *t_old = ctl->parity ? tbuf1 : tbuf0;
  const int hh = ch.hh, tid = threadIdx.x;
  const int rows = min(kHHRows, ch.pp - tt.k0);
  double *Vs = hsm, *Ts = hsm + kHHRows * hh;
  const double *vb = v_pphh + ch.t_off + (int64_t)tt.k0 * hh;
  const double *tb = t_old + ch.t_off + (int64_t)tt.k0 * hh;
  for (int e = tid; e < rows * hh; e += kHHThreads) {
    Vs[e] = vb[e];
    Ts[e] = tb[e];
  }
  __syncthreads();
  const int nout = hh * hh;
  double *mypart = part + ch.part_off + (int64_t)tt.idx * nout;
#pragma unroll
  for (int q = 0; q < kHHAcc; ++q) {
    const int idx = tid + q * kHHThreads;
    if (idx < nout) {
      const int kl = idx / hh, ij = idx - kl * hh;
      double a = 0.0;
      for (int k = 0; k < rows; ++k) a += Vs[k * hh + kl] * Ts[k * hh + ij];
      mypart[idx] = a;
    }
  }
  if (tid < rows) {
    double rr = 0.0;
    for (int ij = 0; ij < hh; ++ij) rr += Vs[tid * hh + ij] * Ts[tid * hh + ij];
    r_out[ch.pp_off + tt.k0 + tid] = rr;
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) last = (atomicAdd(&counters[tt.ch], 1) == ch.nhht - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  const int nb = 8 * ch.cg;
  const double *pbase = part + ch.part_off;
  for (int idx = tid; idx < nout; idx += kHHThreads) {
    double p = 0.0;
    for (int t = 0; t < ch.nhht; ++t) p += __ldcg(pbase + (int64_t)t * nout + idx);
    const int kl = idx / hh, ij = idx - kl * hh;
    const double x = v_hhhh[ch.x_off + idx] + 0.5 * p;
    x_ref[ch.x_off + idx] = x;
    x_t[ch.xt_base + (int64_t)(kl / kBK) * kBK * nb + (kl % kBK) * nb + ij] = 0.5 * x;
    if (kl == ij) s_out[ch.hh_off + ij] = p;
  }
  if (tid == 0) counters[tt.ch] = 0;
}

// ------------------------------------------------------------------------------------------
// Ring term: Y = V_hphp + 0.5 V_hpph T', R = T' Y per modified channel.
// Channels with ph', hp' <= kRingSmall run one per warp; larger ones one per CTA.
// ------------------------------------------------------------------------------------------
constexpr int kRingThreads = 256;
constexpr int kRingSmall = 16;

__global__ void __launch_bounds__(256)
ring_small_kernel(const ModInfo *__restrict__ mods, int n, const double *__restrict__ v_hpph,
                  const double *__restrict__ v_hphp, const double *__restrict__ t_phhp,
                  double *__restrict__ r_phhp, const Control *ctl) {
  if (skip_iteration(ctl)) return;
  __shared__ double buf[8][3 * kRingSmall * kRingSmall];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int mi = blockIdx.x * 8 + w;
  if (mi >= n) return;
  const ModInfo m = mods[mi];
  const int ph = m.ph, hp = m.hp;
  double *Ts = buf[w], *Va = Ts + ph * hp, *Ys = Va + hp * ph;
  for (int e = lane; e < ph * hp; e += 32) {
    Ts[e] = t_phhp[m.m_off + e];
    Va[e] = v_hpph[m.m_off + e];
  }
  for (int e = lane; e < hp * hp; e += 32) Ys[e] = v_hphp[m.y_off + e];
  __syncwarp();
  for (int e = lane; e < hp * hp; e += 32) {
    const int i = e / hp, j = e - i * hp;
    double a = 0.0;
    for (int k = 0; k < ph; ++k) a += Va[i * ph + k] * Ts[k * hp + j];
    Ys[e] = 0.5 * a + Ys[e];
  }
  __syncwarp();
  for (int e = lane; e < ph * hp; e += 32) {
    const int i = e / hp, j = e - i * hp;
    double a = 0.0;
    for (int k = 0; k < hp; ++k) a += Ts[i * hp + k] * Ys[k * hp + j];
    r_phhp[m.m_off + e] = a;
  }
}

__global__ void __launch_bounds__(kRingThreads)
ring_kernel(const ModInfo *__restrict__ mods, const double *__restrict__ v_hpph,
            const double *__restrict__ v_hphp, const double *__restrict__ t_phhp,
            double *__restrict__ r_phhp, const Control *ctl) {
  if (skip_iteration(ctl)) return;
  extern __shared__ __align__(16) double rs[];
  const ModInfo m = mods[blockIdx.x];
  const int ph = m.ph, hp = m.hp, tid = threadIdx.x;
  double *Ts = rs;             // ph x hp
  double *Va = Ts + ph * hp;   // hp x ph
  double *Ys = Va + hp * ph;   // hp x hp
  for (int e = tid; e < ph * hp; e += kRingThreads) {
    Ts[e] = t_phhp[m.m_off + e];
    Va[e] = v_hpph[m.m_off + e];
  }
  for (int e = tid; e < hp * hp; e += kRingThreads) Ys[e] = v_hphp[m.y_off + e];
  __syncthreads();
  for (int e = tid; e < hp * hp; e += kRingThreads) {
    const int i = e / hp, j = e - i * hp;
    double a = 0.0;
    for (int k = 0; k < ph; ++k) a += Va[i * ph + k] * Ts[k * hp + j];
    Ys[e] = 0.5 * a + Ys[e];
  }
  __syncthreads();
  for (int e = tid; e < ph * hp; e += kRingThreads) {
    const int i = e / hp, j = e - i * hp;
    double a = 0.0;
    for (int k = 0; k < hp; ++k) a += Ts[i * hp + k] * Ys[k * hp + j];
    r_phhp[m.m_off + e] = a;
  }
}

// Deterministic block reduction (fixed tree) of one double; result valid in thread 0.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *scratch) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) {
    r = lane < NT / 32 ? scratch[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  return r;
}

// ------------------------------------------------------------------------------------------
// One-body terms through the 3-body chains (table path), one CTA per orbital:
//   hole k:     x = sum v_h_hpp * t2Old_h2pp_h1;  diff_h2pp_h1 = 0.5 x t2Old_h1pp_h2
//   particle a: y = sum t2Old_p1_p2hh * v_phh_p;  diff_p2_p1hh = -0.5 y t2Old_p2_p1hh
// (argument order of main.cpp:591-607).
// ------------------------------------------------------------------------------------------
constexpr int kOBThreads = 256;
__global__ void __launch_bounds__(kOBThreads)
onebody_tables_kernel(int np, const int64_t *__restrict__ o_h, const int64_t *__restrict__ o_p,
                      const double *__restrict__ v_h_hpp, const double *__restrict__ old_h2pp_h1,
                      const double *__restrict__ old_h1pp_h2, double *__restrict__ diff_h2pp_h1,
                      const double *__restrict__ v_phh_p, const double *__restrict__ old_p1_p2hh,
                      const double *__restrict__ old_p2_p1hh, double *__restrict__ diff_p2_p1hh,
                      int do_holes, int do_particles) {
  __shared__ double scratch[32];
  __shared__ double total;
  const int b = blockIdx.x;
  const bool hole = b < np;
  if ((hole && !do_holes) || (!hole && !do_particles)) return;
  const int64_t lo = hole ? o_h[b] : o_p[b - np], hi = hole ? o_h[b + 1] : o_p[b - np + 1];
  double part = 0.0;
  for (int64_t e = lo + threadIdx.x; e < hi; e += kOBThreads)
    part += hole ? v_h_hpp[e] * old_h2pp_h1[e] : old_p1_p2hh[e] * v_phh_p[e];
  const double sum = block_sum<kOBThreads>(part, scratch);
  if (threadIdx.x == 0) total = sum;
  __syncthreads();
  const double f = hole ? 0.5 * total : -0.5 * total;
  for (int64_t e = lo + threadIdx.x; e < hi; e += kOBThreads) {
    if (hole) diff_h2pp_h1[e] = f * old_h1pp_h2[e];
    else diff_p2_p1hh[e] = f * old_p2_p1hh[e];
  }
}

// Fused path: x_k and y_a as segmented sums of the ladder-kernel by-products s and r.
// One warp per orbital, lane-strided partial sums and a fixed shuffle tree.
__global__ void onebody_fused_kernel(int np, int nsp, const int64_t *__restrict__ list_off,
                                     const int32_t *__restrict__ list, const double *__restrict__ s,
                                     const double *__restrict__ r, double *__restrict__ xh,
                                     double *__restrict__ yp, const Control *ctl) {
  if (skip_iteration(ctl)) return;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= nsp) return;
  const bool hole = w < np;
  const double *src = hole ? s : r;
  double v = 0.0;
  for (int64_t e = list_off[w] + lane; e < list_off[w + 1]; e += 32) v += src[list[e]];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (lane == 0) {
    if (hole) xh[w] = v;
    else yp[w - np] = v;
  }
}

// Writes one amplitude into the ladder operand tiles: the B tiles of V T (rows c<d) and the A
// tiles of T X (rows a<=b).  pk_idx[AB] = (K index or -1, packed row or -1).
__device__ __forceinline__ void write_t_tiles(const ChanInfo &ch, const int2 *__restrict__ pk_idx,
                                              int ab, int ij, double t, double *t_kt,
                                              double *t_mt) {
  const int2 q = pk_idx[ch.pp_off + ab];
  const int nb = 8 * ch.cg;
  if (q.x >= 0) t_kt[ch.tkt_base + (int64_t)(q.x / kBK) * kBK * nb + (q.x % kBK) * nb + ij] = t;
  if (q.y >= 0)
    t_mt[ch.tmt_base + (int64_t)((q.y / ch.bm) * ch.nkh + ij / kBK) * ch.bm * kBK +
         swzA(q.y % ch.bm, ij % kBK)] = t;
}

// ------------------------------------------------------------------------------------------
// Fused assembly (calc.cpp:384-418 plus the remaps folded in):
//   value = V + D + R_ai,jb - R_aj,ib - R_bi,ja + R_bj,ia          (4 gathers from R in phhp layout)
//         + 0.5 x_i t_ab,ji - 0.5 x_j t_ab,ij                       (h2pp_h1 gathers, algebraically)
//         + (-0.5 y_b) t_ab,ij - (-0.5 y_a) t_ba,ij                 (p2_p1hh gathers, algebraically)
//   t_new = mixing value/(e_i+e_j-e_a-e_b) + (1-mixing) t_old;  E += V t_new
// and the next iteration's operands are written in the same pass: t_new into the phhp slab
// (mapToDistributed ai_jb) and into the ladder operand tiles.
// ------------------------------------------------------------------------------------------
constexpr int kAsmThreads = 256;
constexpr int kAsmPerThread = 1;

__global__ void __launch_bounds__(kAsmThreads)
assemble_fused_kernel(const ElemRange *__restrict__ ranges, const ChanInfo *__restrict__ chans,
                      const int2 *__restrict__ pp_pairs, const int2 *__restrict__ hh_pairs,
                      const int32_t *__restrict__ pp_swap, const int32_t *__restrict__ hh_swap,
                      const int2 *__restrict__ pk_idx,
                      const double *__restrict__ v_pphh, const double *__restrict__ dmat,
                      const double *__restrict__ r_phhp, const int32_t *__restrict__ g_ai_jb,
                      const int32_t *__restrict__ g_aj_ib, const int32_t *__restrict__ g_bi_ja,
                      const int32_t *__restrict__ g_bj_ia, const double *__restrict__ xh,
                      const double *__restrict__ yp, const double *__restrict__ eps, int np,
                      double *tbuf0, double *tbuf1, double *__restrict__ old_phhp,
                      double *__restrict__ t_kt, double *__restrict__ t_mt,
                      double *__restrict__ epart, const Control *ctl) {
  if (skip_iteration(ctl)) return;
  __shared__ double scratch[32];
  const ElemRange rg = ranges[blockIdx.x];
  const ChanInfo ch = chans[rg.ch];
  const double *t_old = ctl->parity ? tbuf1 : tbuf0;
  double *t_new = ctl->parity ? tbuf0 : tbuf1;
  const double mixing = ctl->mixing;
  const int hh = ch.hh;
  double corr = 0.0;
  for (int64_t e = rg.e0 + threadIdx.x; e < rg.e1; e += kAsmThreads) {
    const int64_t loc = e - ch.t_off;
    const int ab = (int)(loc / hh), ij = (int)(loc - (int64_t)ab * hh);
    const int2 pab = pp_pairs[ch.pp_off + ab], pij = hh_pairs[ch.hh_off + ij];
    const double v = v_pphh[e];
    const double to = t_old[e];
    const double t_ji = t_old[ch.t_off + (int64_t)ab * hh + hh_swap[ch.hh_off + ij]];
    const double t_ba = t_old[ch.t_off + (int64_t)pp_swap[ch.pp_off + ab] * hh + ij];
    double value = v;
    value += dmat[e];
    value += r_phhp[g_ai_jb[e]];
    value -= r_phhp[g_aj_ib[e]];
    value -= r_phhp[g_bi_ja[e]];
    value += r_phhp[g_bj_ia[e]];
    value += (0.5 * xh[pij.x]) * t_ji;
    value -= (0.5 * xh[pij.y]) * to;
    value += (-0.5 * yp[pab.y - np]) * to;
    value -= (-0.5 * yp[pab.x - np]) * t_ba;
    value = value / (eps[pij.x] + eps[pij.y] - eps[pab.x] - eps[pab.y]);
    value = mixing * value + (1. - mixing) * to;
    t_new[e] = value;
    old_phhp[g_ai_jb[e]] = value;
    write_t_tiles(ch, pk_idx, ab, ij, value, t_kt, t_mt);
    corr += v * value;
  }
  const double sum = block_sum<kAsmThreads>(corr, scratch);
  if (threadIdx.x == 0) epart[blockIdx.x] = sum;
}

// Table path assembly: exactly calcChannelT2_pphh over the eight gathered chains.
__global__ void __launch_bounds__(kAsmThreads)
assemble_tables_kernel(const ElemRange *__restrict__ ranges, const ChanInfo *__restrict__ chans,
                       const int2 *__restrict__ pp_pairs, const int2 *__restrict__ hh_pairs,
                       const double *__restrict__ v_pphh, const double *__restrict__ dmat,
                       const double *__restrict__ gath, int64_t n_t,
                       const double *__restrict__ eps, const double *__restrict__ t_old,
                       double *__restrict__ t_new, double *__restrict__ epart, double mixing) {
  __shared__ double scratch[32];
  const ElemRange rg = ranges[blockIdx.x];
  const ChanInfo ch = chans[rg.ch];
  const int hh = ch.hh;
  double corr = 0.0;
  for (int64_t e = rg.e0 + threadIdx.x; e < rg.e1; e += kAsmThreads) {
    const int64_t loc = e - ch.t_off;
    const int ab = (int)(loc / hh), ij = (int)(loc - (int64_t)ab * hh);
    const int2 pab = pp_pairs[ch.pp_off + ab], pij = hh_pairs[ch.hh_off + ij];
    const double v = v_pphh[e];
    double value = v;
    value += dmat[e];
    value += gath[4 * n_t + e];  // ai_jb
    value -= gath[5 * n_t + e];  // aj_ib
    value -= gath[6 * n_t + e];  // bi_ja
    value += gath[7 * n_t + e];  // bj_ia
    value += gath[1 * n_t + e];  // jab_i
    value -= gath[0 * n_t + e];  // iab_j
    value += gath[3 * n_t + e];  // b_aij
    value -= gath[2 * n_t + e];  // a_bij
    value = value / (eps[pij.x] + eps[pij.y] - eps[pab.x] - eps[pab.y]);
    value = mixing * value + (1. - mixing) * t_old[e];
    t_new[e] = value;
    corr += v * value;
  }
  const double sum = block_sum<kAsmThreads>(corr, scratch);
  if (threadIdx.x == 0) epart[blockIdx.x] = sum;
}

// The eight mapFromDistributed gathers: out_k[e] = src_k[flat_k[e]].
__global__ void gather8_kernel(int64_t n_t, const int32_t *__restrict__ flat,
                               const double *__restrict__ hpp, const double *__restrict__ phh,
                               const double *__restrict__ phhp, double *__restrict__ out) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n_t;
       e += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const double *src = k < 2 ? hpp : (k < 4 ? phh : phhp);
      out[k * n_t + e] = src[flat[k * n_t + e]];
    }
  }
}

// Chain::set + the five mapToDistributed scatters, plus the ladder operand tiles.
__global__ void map_to_kernel(const ElemRange *__restrict__ ranges, const ChanInfo *__restrict__ chans,
                              const int2 *__restrict__ pk_idx, const int32_t *__restrict__ flat,
                              int64_t n_t,
                              const double *__restrict__ t2, double *__restrict__ t2_old,
                              double *__restrict__ old_h2pp_h1, double *__restrict__ old_h1pp_h2,
                              double *__restrict__ old_p1_p2hh, double *__restrict__ old_p2_p1hh,
                              double *__restrict__ old_phhp, double *__restrict__ t_kt,
                              double *__restrict__ t_mt, int with_3body) {
  const ElemRange rg = ranges[blockIdx.x];
  const ChanInfo ch = chans[rg.ch];
  for (int64_t e = rg.e0 + threadIdx.x; e < rg.e1; e += blockDim.x) {
    const double t = t2[e];
    t2_old[e] = t;
    if (with_3body) {
      old_h2pp_h1[flat[1 * n_t + e]] = t;  // jab_i
      old_h1pp_h2[flat[0 * n_t + e]] = t;  // iab_j
      old_p1_p2hh[flat[2 * n_t + e]] = t;  // a_bij
      old_p2_p1hh[flat[3 * n_t + e]] = t;  // b_aij
    }
    old_phhp[flat[4 * n_t + e]] = t;       // ai_jb
    const int64_t loc = e - ch.t_off;
    const int ab = (int)(loc / ch.hh), ij = (int)(loc - (int64_t)ab * ch.hh);
    write_t_tiles(ch, pk_idx, ab, ij, t, t_kt, t_mt);
  }
}

// Sum of the per-CTA energy partials (Neumaier-compensated, fixed order), then the
// reference's stop rule on the device.  flags: 1 = flip the amplitude buffer parity,
// 2 = count this as an iteration of the solve loop.
__global__ void energy_kernel(const double *__restrict__ epart, int n, Control *ctl, int flags,
                              double *e_out) {
  if (skip_iteration(ctl)) return;
  __shared__ double ss[1024], cs[1024];
  double s = 0.0, c = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double x = epart[i];
    const double t = s + x;
    c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
    s = t;
  }
  ss[threadIdx.x] = s;
  cs[threadIdx.x] = c;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      const double a = ss[threadIdx.x], b = ss[threadIdx.x + w];
      const double t = a + b;
      const double e = fabs(a) >= fabs(b) ? (a - t) + b : (b - t) + a;
      ss[threadIdx.x] = t;
      cs[threadIdx.x] += cs[threadIdx.x + w] + e;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double corr = 0.25 * (ss[0] + cs[0]);
    if (e_out) *e_out = corr;
    if (flags & 2) {
      const double diff = corr - ctl->e_prev;
      ctl->e_prev = corr;
      ctl->e_corr = corr;
      ctl->e_diff = diff;
      if (ctl->iterations < 128) ctl->energies[ctl->iterations] = corr;
      ctl->iterations += 1;
      if (!isfinite(corr)) {
        ctl->error |= kErrNonFinite;
        ctl->done = 1;
      }
      if (fabs(diff) <= ctl->tol || ctl->iterations > ctl->max_iters) ctl->done = 1;
    }
    if (flags & 1) ctl->parity ^= 1;
  }
}

}  // namespace ccd
