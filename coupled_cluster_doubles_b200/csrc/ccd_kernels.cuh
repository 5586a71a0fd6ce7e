// CCD iteration kernels for sm_100a (FP64 path).
//
// Reference correspondence (calc.cpp / Chain.hpp of justinlietz/coupled_cluster_doubles):
//   pp_ladder_kernel        D = 0.5 T X + 0.5 V_pppp T              calc.cpp:162-202
//                           (antisymmetry-packed, FP64 FMA pipe)
//   hh_mma_kernel           X = V_hhhh + 0.5 V_hhpp T                calc.cpp:141-160
//   ring_*_kernel           Y = V_hphp + 0.5 V_hpph T'; R = T' Y     calc.cpp:264-313
//   onebody_tables_kernel   calcChannelT2Diff_h2pp_h1 / _p2_p1hh     calc.cpp:9-25, 73-89
//   onebody_fused_kernel    the same dot products, read from the ladder intermediates
//   gather8_kernel          Chain::mapFromDistributed x 8            Chain.hpp:710-755
//   assemble_*_kernel       calcChannelT2_pphh                       calc.cpp:368-421
//   map_to_kernel           Chain::set + mapToDistributed x 5        Chain.hpp:503-527,757-802
//   energy_kernel           reduction(+:corr) + MPI_Allreduce + stop rule, main.cpp:511-519,668-670
#pragma once

#include <cstdint>

#include <cuda_bf16.h>

#include "ccd_device.cuh"

namespace ccd {

constexpr uint64_t kWaitLimitNs = 1000000000ull;  // bounded mbarrier waits: 1 s of globaltimer

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
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait on an mbarrier phase: try_wait suspends the thread in hardware until the phase
// completes or a short internal time limit passes; give up (false) after kWaitLimitNs.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (;;) {
#pragma unroll 1
    for (int i = 0; i < 256; ++i)
      if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > kWaitLimitNs) return false;
  }
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
// sum_k a[k*sa] * b[k*sb] for k < n with four interleaved partial sums (more independent FMA
// chains in flight), combined in a fixed order.
__device__ __forceinline__ double dot4(const double *a, int sa, const double *b, int sb, int n) {
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  int k = 0;
  for (; k + 4 <= n; k += 4) {
    s0 = fma(a[k * sa], b[k * sb], s0);
    s1 = fma(a[(k + 1) * sa], b[(k + 1) * sb], s1);
    s2 = fma(a[(k + 2) * sa], b[(k + 2) * sb], s2);
    s3 = fma(a[(k + 3) * sa], b[(k + 3) * sb], s3);
  }
  for (; k < n; ++k) s0 = fma(a[k * sa], b[k * sb], s0);
  return (s0 + s1) + (s2 + s3);
}

// Programmatic dependent launch: wait until the preceding kernel of the stream has completed
// (its writes are visible), then allow the next kernel to begin launching once every CTA of
// this grid is resident.  Both are no-ops for kernels launched without the PDL attribute.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// gate 0: kernel of an FP64 iteration, gate 1: kernel of a mixed-precision iteration.  During
// a solve, an iteration whose precision does not match the phase is a no-op (a replayed batch
// can straddle the switch to the FP64 polish).
// The kernel id `tr` records its first and last CTA start in the trace of the armed iteration.
__device__ __forceinline__ void trace_start(const Control *ctl, int tr) {
  if (threadIdx.x == 0 && ctl->trace_iter == ctl->iterations) {
    Control *c = const_cast<Control *>(ctl);
    const unsigned long long t = global_ns();
    atomicMin(reinterpret_cast<unsigned long long *>(&c->trace_first[tr]), t);
    atomicMax(reinterpret_cast<unsigned long long *>(&c->trace_last[tr]), t);
  }
}
// Records, for the traced iteration, when a CTA of kernel `tr` finished (thread 0, after the
// CTA's work; the trace keeps the latest).
__device__ __forceinline__ void trace_end(const Control *ctl, int tr) {
  if (threadIdx.x == 0 && ctl->trace_iter == ctl->iterations) {
    Control *c = const_cast<Control *>(ctl);
    atomicMax(reinterpret_cast<unsigned long long *>(&c->trace_end[tr]),
              (unsigned long long)global_ns());
  }
}
__device__ __forceinline__ bool skip_iteration(const Control *ctl, int gate, int tr) {
  pdl_enter();
  trace_start(ctl, tr);
  if (!ctl->active) return false;
  return ctl->done || ((gate == 1) != (ctl->phase == 1));
}

// ------------------------------------------------------------------------------------------
// pp ladder + hh-ladder output in FP64 (FMA pipe for thin channels, FP64 MMA for the rest):
//   D[ab,:] = sum_{c<d} V[ab,cd] T[cd,:] + T[ab,:] (X/2)     for packed rows a <= b,
//   D[ba,:] = -D[ab,:]                                        (antisymmetry of V and T).
// Warp 4 is the producer: one lane streams pre-tiled A/B stages with bulk copies (TMA, no
// multicast) into a kStages-deep shared-memory ring guarded by mbarriers.  The 128 consumer
// threads run register-blocked DFMAs (thin channels: V rows from shared memory conflict-free
// by an XOR swizzle, T / X columns as warp broadcasts) or FP64 MMAs (mid and wide channels).  K runs over the c<d pairs (V T) and then over
// hh (T X) with the same pipeline.  Row blocks whose K is split over several tiles write
// partial sums that ladder_reduce_kernel adds in segment order (deterministic).
// ------------------------------------------------------------------------------------------

// FP64 tensor-core MMA (mma.sync m8n8k4, the full-rate FP64 path of sm_100a): lane
// (g = lane / 4, t = lane % 4) supplies A[g][t] and B[t][g] and accumulates C[g][2t] and
// C[g][2t + 1].  One instruction does 256 multiply-adds, so the small channel GEMMs are no longer
// bound by instruction issue and shared-memory loads.
__device__ __forceinline__ void dmma_884(double (&c)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
      : "+d"(c[0]), "+d"(c[1])
      : "d"(a), "d"(b));
}

// C (16 x 8) += A (16 x 16) B (16 x 8) in FP64, lane layout (g = lane / 4, t = lane % 4):
// a[i] = A[g + 8 (i % 2)][t + 4 (i / 2)], b[i] = B[t + 4 i][g],
// c = {C[g][2t], C[g][2t + 1], C[g + 8][2t], C[g + 8][2t + 1]}.
__device__ __forceinline__ void dmma_16816(double (&c)[4], const double (&a)[8],
                                           const double (&b)[4]) {
  asm("mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
      "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
        "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}


// Stores the finished values of packed row u_local (cols [c0, c0+n)), or its partial sum.
struct LadderOut {
  const LadderTile &tile;
  const int32_t *rowmap, *mirror;
  double *d, *part;
  // N is a compile-time count so that v stays in registers (every index is a constant).
  template <int N>
  __device__ __forceinline__ void row(int u_local, int c0, const double (&v)[N]) const {
    if (u_local >= tile.rows) return;
    if (tile.nseg > 1) {
      double *pp = part + tile.part_base + ((int64_t)tile.seg * tile.bm + u_local) * tile.nb + c0;
#pragma unroll
      for (int j = 0; j < N; ++j) pp[j] = v[j];
      return;
    }
    const int u = tile.mt * tile.bm + u_local;
    const int ab = rowmap[tile.row_off + u], mir = mirror[tile.row_off + u];
    double *dr = d + tile.t_off + (int64_t)ab * tile.hh;
    double *mr = d + tile.t_off + (int64_t)mir * tile.hh;
#pragma unroll
    for (int j = 0; j < N; ++j) {
      if (c0 + j < tile.hh) {
        dr[c0 + j] = v[j];
        if (mir >= 0) mr[c0 + j] = -v[j];
      }
    }
  }
};

// Split-K partial sums of a row block, added in segment order by ladder_reduce_kernel after the
// ladder: item = (first tile of the row block, first row of a kRedRows-row chunk).
struct RedItem {
  int32_t tile, r0;
};
constexpr int kRedRows = 16;

// D rows of split row blocks: sum of the segments' partials in segment order (deterministic),
// written to row ab and negated to its mirror ba.  Fully parallel over (row block, row chunk).
__global__ void __launch_bounds__(256)
ladder_reduce_kernel(const RedItem *__restrict__ items, const LadderTile *__restrict__ tiles,
                     const int32_t *__restrict__ rowmap, const int32_t *__restrict__ mirror,
                     double *__restrict__ d, const double *__restrict__ part, const Control *ctl,
                     int gate) {
  if (skip_iteration(ctl, gate, kTrReduce)) return;
  const RedItem it = items[blockIdx.x];
  const LadderTile tile = tiles[it.tile];
  const int nr = min(kRedRows, tile.rows - it.r0), n = nr * tile.nb;
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    const int u_local = it.r0 + e / tile.nb, col = e % tile.nb;
    if (col >= tile.hh) continue;
    // Eight segments' loads in flight together, then added in segment order.
    const double *pc = part + tile.part_base + (int64_t)u_local * tile.nb + col;
    const int64_t seg_stride = (int64_t)tile.bm * tile.nb;
    double v = 0.0;
    int sg = 0;
    for (; sg + 8 <= tile.nseg; sg += 8) {
      double x[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) x[k] = pc[(int64_t)(sg + k) * seg_stride];
#pragma unroll
      for (int k = 0; k < 8; ++k) v += x[k];
    }
    for (; sg < tile.nseg; ++sg) v += pc[(int64_t)sg * seg_stride];
    const int u = tile.mt * tile.bm + u_local;
    const int ab = rowmap[tile.row_off + u], mir = mirror[tile.row_off + u];
    d[tile.t_off + (int64_t)ab * tile.hh + col] = v;
    if (mir >= 0) d[tile.t_off + (int64_t)mir * tile.hh + col] = -v;
  }
  trace_end(ctl, kTrReduce);
}

// Thin channels (nb in {2,4,8}): consumer thread = one packed row, all nb columns.
// bstage: doubles between consecutive B stages (the producer's layout).
template <int NB>
__device__ __forceinline__ bool consume_thin(const LadderTile &tile, const double *As,
                                             const double *Bs, int bstage, uint64_t *bars,
                                             int tid, const LadderOut &out, int32_t *err,
                                             int gc0) {
  const int lane = tid & 31;
  double acc[NB];
#pragma unroll
  for (int j = 0; j < NB; ++j) acc[j] = 0.0;
  const int nchunks = tile.nks + tile.nkh;
  for (int c = 0; c < nchunks; ++c) {
    const int gch = gc0 + c, s = gch % kStages;  // chunk number gch of this CTA
    if (!mbar_wait(smem_u32(&bars[s]), (gch / kStages) & 1)) {
      atomicOr(err, kErrTimeout);
      return false;
    }
    const double *A = As + s * (kMaxAS * kBK);
    const double *B = Bs + s * bstage;
#pragma unroll
    for (int k = 0; k < kBK; ++k) {
      const double a = A[swzA(tid, k)];
      const double2 *bp = reinterpret_cast<const double2 *>(B + k * NB);
#pragma unroll
      for (int j = 0; j < NB / 2; ++j) {
        const double2 b = bp[j];
        acc[2 * j] = fma(a, b.x, acc[2 * j]);
        acc[2 * j + 1] = fma(a, b.y, acc[2 * j + 1]);
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(smem_u32(&bars[kStages + s]));
  }
  out.row<NB>(tid, 0, acc);
  return true;
}

// Mid and wide channels (nb = 8*C, C = 2..9) on the FP64 MMA: consumer warp w owns tile rows
// [16w, 16w + 16), one m16n8k16 per 8-column tile and stage (kBK = 16), 4*C accumulators per
// lane.  A (k-major, row stride ar) and B (k-major, row stride bs) fragments come from the
// stage conflict-free: both strides are 4 mod 8 doubles.  A warp whose lower 8-row half has
// no rows feeds zeros there instead of reading past the tile.
template <int C>
__device__ __forceinline__ bool consume_mma(const LadderTile &tile, const double *As,
                                            const double *Bs, int bstage, uint64_t *bars,
                                            int tid, const LadderOut &out, int32_t *err,
                                            int gc0) {
  static_assert(kBK == 16, "one m16n8k16 K step per stage");
  constexpr int NB = 8 * C, BS = NB + 4;
  const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int ar = ladder_arows(NB, tile.rows);
  const int halves = min(2, max(0, ((tile.rows + 7) >> 3) - 2 * warp));  // 8-row halves with rows
  double acc[C][4];
#pragma unroll
  for (int j = 0; j < C; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0;
  const int nchunks = tile.nks + tile.nkh;
  for (int c = 0; c < nchunks; ++c) {
    const int gch = gc0 + c, s = gch % kStages;  // chunk number gch of this CTA
    if (!mbar_wait(smem_u32(&bars[s]), (gch / kStages) & 1)) {
      atomicOr(err, kErrTimeout);
      return false;
    }
    if (halves > 0) {
      const double *A = As + s * (kMaxAS * kBK) + t * ar + 16 * warp + g;
      const double *B = Bs + s * bstage + t * BS + g;
      double a[8];
#pragma unroll
      for (int i = 0; i < 8; ++i)
        a[i] = (i % 2 == 0 || halves > 1) ? A[4 * (i / 2) * ar + 8 * (i % 2)] : 0.0;
#pragma unroll
      for (int j = 0; j < C; ++j) {
        double b[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) b[q] = B[4 * q * BS + 8 * j];
        dmma_16816(acc[j], a, b);
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(smem_u32(&bars[kStages + s]));
  }
  if (halves > 0) {
#pragma unroll
    for (int j = 0; j < C; ++j) {
      const double lo[2] = {acc[j][0], acc[j][1]}, hi[2] = {acc[j][2], acc[j][3]};
      out.row<2>(16 * warp + g, 8 * j + 2 * t, lo);
      if (halves > 1) out.row<2>(16 * warp + 8 + g, 8 * j + 2 * t, hi);
    }
  }
  return true;
}

// Column classes: CLS 0 = thin (nb <= 8), 1 = mid (nb 16..32), 2 = wide (nb 40..72).  Separate
// instantiations keep the register budget of narrow channels independent of the 72-column case.
// Persistent CTAs: CTA b runs tiles cta_off[b] .. cta_off[b+1] (a balanced assignment made on the
// host); the producer streams K chunks through the stage ring across tile boundaries and the
// consumers write each tile's rows when its last chunk is done.
template <int CLS>
__global__ void __launch_bounds__(ladder_threads(CLS), CLS == 0 ? 3 : CLS == 1 ? 2 : 1)
pp_ladder_kernel(const LadderTile *__restrict__ tiles, const int32_t *__restrict__ cta_off,
                 const double *__restrict__ v_t, const double *__restrict__ t_kt,
                 const double *__restrict__ t_mt, const double *__restrict__ x_t,
                 const int32_t *__restrict__ rowmap, const int32_t *__restrict__ mirror,
                 double *__restrict__ d, double *part, const Control *ctl, int32_t *err,
                 int gate) {
  if (skip_iteration(ctl, gate, kTrLadderThin + CLS)) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double *As = reinterpret_cast<double *>(smem_raw);
  double *Bs = As + kStages * kMaxAS * kBK;
  constexpr bool WIDE = CLS > 0;
  constexpr int kConsumerWarps = (ladder_threads(CLS) - 32) / 32;
  const int bstage = WIDE ? kBK * kMaxBS : kBK * 8;
  uint64_t *bars = reinterpret_cast<uint64_t *>(Bs + kStages * bstage);
  const int t_begin = cta_off[blockIdx.x], t_end = cta_off[blockIdx.x + 1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(smem_u32(&bars[s]), 1);
      mbar_init(smem_u32(&bars[kStages + s]), kConsumerWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  if (warp == kConsumerWarps) {
    if (lane == 0) {
      int gc = 0;  // chunks issued by this CTA
      bool stop = false;
      // Test-only fault (ccdgpu_inject_wait_timeout): CTA 0 never fills its first stage, so
      // its consumers' bounded waits run out, then this producer's wait for that stage does.
      const bool withhold = ctl->inject != 0 && blockIdx.x == 0;
      for (int ti = t_begin; ti < t_end && !stop; ++ti) {
        const LadderTile tile = tiles[ti];
        const int ar = ladder_arows(tile.nb, tile.rows);
        const int bs = ladder_bs(tile.nb), af = ladder_arows_full(tile.nb);
        const uint32_t abytes = ar * kBK * 8, bbytes = kBK * bs * 8;
        const int nchunks = tile.nks + tile.nkh;
        const int64_t vtile = tile.v_base + (int64_t)tile.mt * af * tile.nkc * kBK;
        const int64_t ttile = tile.tmt_base + (int64_t)tile.mt * af * tile.nkh * kBK;
        for (int c = 0; c < nchunks; ++c, ++gc) {
          const int s = gc % kStages;
          if (gc >= kStages &&
              !mbar_wait(smem_u32(&bars[kStages + s]), ((gc / kStages) - 1) & 1)) {
            atomicOr(err, kErrTimeout);
            stop = true;
            break;
          }
          if (withhold && gc == 0) continue;
          const double *asrc, *bsrc;
          if (c < tile.nks) {
            const int kc = tile.kc0 + c;
            asrc = v_t + vtile + (int64_t)kc * ar * kBK;
            bsrc = t_kt + tile.tkt_base + (int64_t)kc * kBK * bs;
          } else {
            const int kh = c - tile.nks;
            asrc = t_mt + ttile + (int64_t)kh * ar * kBK;
            bsrc = x_t + tile.xt_base + (int64_t)kh * kBK * bs;
          }
          const uint32_t full = smem_u32(&bars[s]);
          mbar_expect_tx(full, abytes + bbytes);
          bulk_g2s(smem_u32(As + s * kMaxAS * kBK), asrc, abytes, full);
          bulk_g2s(smem_u32(Bs + s * bstage), bsrc, bbytes, full);
        }
      }
    }
    return;
  }
  const int tid = threadIdx.x;
  int gc = 0;
  for (int ti = t_begin; ti < t_end; ++ti) {
    const LadderTile tile = tiles[ti];
    const LadderOut out{tile, rowmap, mirror, d, part};
    bool ok = true;
    if (!WIDE) {
      switch (tile.nb) {
        case 2: ok = consume_thin<2>(tile, As, Bs, bstage, bars, tid, out, err, gc); break;
        case 4: ok = consume_thin<4>(tile, As, Bs, bstage, bars, tid, out, err, gc); break;
        default: ok = consume_thin<8>(tile, As, Bs, bstage, bars, tid, out, err, gc); break;
      }
    } else {
#define CCD_WIDE8_CASE(n) \
  case n: ok = consume_mma<n>(tile, As, Bs, bstage, bars, tid, out, err, gc); break;
      if (CLS == 1) {
        switch (tile.nb / 8) { CCD_WIDE8_CASE(2) CCD_WIDE8_CASE(3) CCD_WIDE8_CASE(4) default: break; }
      } else {
        switch (tile.nb / 8) {
          CCD_WIDE8_CASE(5) CCD_WIDE8_CASE(6) CCD_WIDE8_CASE(7) CCD_WIDE8_CASE(8) CCD_WIDE8_CASE(9)
          default: break;
        }
      }
#undef CCD_WIDE8_CASE
    }
    if (!ok) break;  // a timed-out tile leaves its row block unfinished (error already set)
    gc += tile.nks + tile.nkh;
  }
  trace_end(ctl, kTrLadderThin + CLS);
}

// ------------------------------------------------------------------------------------------
// Register-tiled outer-product micro-GEMM for the small per-channel FP64 products:
//   acc[i][j] += sum_k A[k*lda + r0 + i] * B[k*ldb + c0 + j],   i, j < TM.
// Both operands are k-row major in shared memory, so a thread reads its TM-wide slices with
// 16-byte loads (TM even: lda, ldb and r0, c0 even).  Slices may run past the valid rows or
// columns (and past the last row into padding); those accumulators are never stored.
// ------------------------------------------------------------------------------------------
template <int TM>
__device__ __forceinline__ void opgemm(const double *__restrict__ A, int lda,
                                       const double *__restrict__ B, int ldb, int K, int r0,
                                       int c0, double (&acc)[TM][TM]) {
  const double *a = A + r0, *b = B + c0;
#pragma unroll 2
  for (int k = 0; k < K; ++k) {
    double av[TM], bv[TM];
    if constexpr (TM % 2 == 0) {
#pragma unroll
      for (int i = 0; i < TM / 2; ++i) {
        const double2 x = *reinterpret_cast<const double2 *>(a + 2 * i);
        const double2 y = *reinterpret_cast<const double2 *>(b + 2 * i);
        av[2 * i] = x.x;
        av[2 * i + 1] = x.y;
        bv[2 * i] = y.x;
        bv[2 * i + 1] = y.y;
      }
    } else {
#pragma unroll
      for (int i = 0; i < TM; ++i) {
        av[i] = a[i];
        bv[i] = b[i];
      }
    }
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TM; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
    a += lda;
    b += ldb;
  }
}
__host__ __device__ inline int even_up(int n) { return (n + 1) & ~1; }

// cp.async (8- and 4-byte) global -> shared copies, committed and waited for by group.
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ------------------------------------------------------------------------------------------
// hh ladder intermediate (calc.cpp:141-160 and the one-body sums of calc.cpp:18-20, 82-84):
//   P = V_hhpp T (K = pp),  X = V_hhhh + 0.5 P  (reference layout, and X/2 as B tiles),
//   s[IJ] = P[IJ][IJ],  r[AB] = sum_IJ V[IJ][AB] T[AB][IJ].
// V_hhpp is held transposed (pp x hh), so a K slice of V and of T are contiguous row ranges.
// hh_mma_kernel: one warp per (slice of kHHRows pp rows, chunk of P rows) on the FP64 MMA,
// fragments loaded straight from global memory (8 consecutive columns of 4 rows per load);
// rows past the slice and columns past hh read as zero.  The warp of chunk 0 also forms the
// row dots r from the same fragments.  Each slice writes its partial P; hh_reduce_kernel adds
// the partials in slice order (deterministic) and finishes X, its operand tiles and s.
// ------------------------------------------------------------------------------------------
constexpr int kHHWarps = 8;
constexpr int kHHRows = 32;  // pp rows of one K slice

// X, its X/2 operand tiles (FP64 and, for a mixed iteration, bf16 terms) and s from one
// finished element P[kl][ij].
__device__ __forceinline__ void hh_finish(const ChanInfo &ch, int kl, int ij, double p,
                                          const double *__restrict__ v_hhhh, double *x_ref,
                                          double *x_t, double *s_out, __nv_bfloat16 *xt_tc,
                                          int64_t xt_tc_stride, int nt) {
  const int hh = ch.hh, idx = kl * hh + ij;
  const double x = v_hhhh[ch.x_off + idx] + 0.5 * p;
  x_ref[ch.x_off + idx] = x;
  const int bs = ladder_bs(ch.nb);
  x_t[ch.xt_base + (int64_t)(kl / kBK) * kBK * bs + (kl % kBK) * bs + ij] = 0.5 * x;
  if (nt) {
    const int64_t o =
        ch.xt_tc_base + (int64_t)(kl >> 5) * (ch.nbt >> 3) * kTcGroup + tc_off_mn(ij, kl & 31);
    if (nt == 3) {
      __nv_bfloat16 hv[3];
      split_bf16_n<3>(0.5 * x, hv);
#pragma unroll
      for (int q = 0; q < 3; ++q) xt_tc[q * xt_tc_stride + o] = hv[q];
    } else {
      __nv_bfloat16 hv[2];
      split_bf16_n<2>(0.5 * x, hv);
#pragma unroll
      for (int q = 0; q < 2; ++q) xt_tc[q * xt_tc_stride + o] = hv[q];
    }
  }
  if (kl == ij) s_out[ch.hh_off + ij] = p;
}

// NMAX = column tiles of 8 held per warp: 2 for hh <= 16 (MC = 2 row tiles per warp, the whole
// P), kMaxCG for the rest (MC = 1 row tile per warp).
template <int NMAX>
__global__ void __launch_bounds__(kHHWarps * 32, NMAX <= 2 ? 4 : 2)
hh_mma_kernel(const HHTile *__restrict__ tiles, int n, const ChanInfo *__restrict__ chans,
              const double *__restrict__ v_pphh, const double *tbuf0, const double *tbuf1,
              double *__restrict__ part, double *__restrict__ r_out, const Control *ctl,
              int gate) {
  if (skip_iteration(ctl, gate, NMAX <= 2 ? kTrHHSmall : kTrHHTiled)) return;
  const int u = blockIdx.x * kHHWarps + (threadIdx.x >> 5);
  if (u >= n) return;
  const HHTile tt = tiles[u];
  const ChanInfo ch = chans[tt.ch];
  const double *t_old = ctl->parity ? tbuf1 : tbuf0;
  const int hh = ch.hh, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  constexpr int MC = NMAX <= 2 ? 2 : 1;
  const int h8 = (hh + 7) >> 3, mc0 = MC * tt.chunk, mc = min(MC, h8 - mc0);
  const bool do_dot = tt.chunk == 0;
  const double *vb = v_pphh + ch.t_off + (int64_t)tt.k0 * hh;
  const double *tb = t_old + ch.t_off + (int64_t)tt.k0 * hh;
  double acc[MC][NMAX][2];
#pragma unroll
  for (int m = 0; m < MC; ++m)
#pragma unroll
    for (int c = 0; c < NMAX; ++c) acc[m][c][0] = acc[m][c][1] = 0.0;
  // hh <= 16: all kHHRows / 4 steps unrolled, so that every fragment load of the slice is issued
  // at once (rows past the slice read as zero); wider hh: two steps at a time (registers).
  constexpr int kSteps = kHHRows / 4;
#pragma unroll(NMAX <= 2 ? kSteps : 2)
  for (int k4 = 0; k4 < kSteps; ++k4) {
    const int k = 4 * k4 + t;
    const bool kin = k < tt.rows;
    const double *vr = vb + (int64_t)k * hh, *tr = tb + (int64_t)k * hh;
    double a[MC], b[NMAX];
#pragma unroll
    for (int m = 0; m < MC; ++m) {
      const int col = (mc0 + m) * 8 + g;
      a[m] = (kin && col < hh) ? vr[col] : 0.0;
    }
#pragma unroll
    for (int c = 0; c < NMAX; ++c) {
      const int col = c * 8 + g;
      b[c] = (kin && col < hh) ? tr[col] : 0.0;
    }
#pragma unroll
    for (int m = 0; m < MC; ++m)
#pragma unroll
      for (int c = 0; c < NMAX; ++c)
        if (m < mc && c < h8) dmma_884(acc[m][c], a[m], b[c]);
    if (do_dot) {
      // Row k: lane partial over columns 8c + g, then a fixed butterfly over g.
      double d = 0.0;
#pragma unroll
      for (int c = 0; c < NMAX; ++c) {
        const int col = c * 8 + g;
        const double v = c < MC ? a[c] : ((kin && col < hh) ? vr[col] : 0.0);
        d = fma(v, b[c], d);
      }
      d += __shfl_xor_sync(0xffffffffu, d, 4);
      d += __shfl_xor_sync(0xffffffffu, d, 8);
      d += __shfl_xor_sync(0xffffffffu, d, 16);
      if (g == 0 && kin) r_out[ch.pp_off + tt.k0 + k] = d;
    }
  }
  double *pb = part + ch.part_off + (int64_t)tt.idx * hh * hh;
#pragma unroll
  for (int m = 0; m < MC; ++m)
#pragma unroll
    for (int c = 0; c < NMAX; ++c) {
      const int kl = (mc0 + m) * 8 + g, ij = c * 8 + 2 * t;
      if (m < mc && c < h8 && kl < hh) {
        if (ij < hh) pb[kl * hh + ij] = acc[m][c][0];
        if (ij + 1 < hh) pb[kl * hh + ij + 1] = acc[m][c][1];
      }
    }
  trace_end(ctl, NMAX <= 2 ? kTrHHSmall : kTrHHTiled);
}

// Channels with hh > 16: one CTA per K slice of kHHRowsL pp rows.  The slice's rows of V_pphh
// and T (two contiguous ranges of rows * hh doubles) go to shared memory with cp.async, all in
// flight at once, at a row stride of hh rounded up to 16, plus 4 (4 mod 16 doubles:
// conflict-free fragment loads); rows up to the next multiple of 16 and columns up to the
// padded width are zero.  P = V^T T runs on the FP64 m16n8k16 MMA: warp w takes items of one
// 16-row tile of P by kHHNC 8-column tiles, at most four k-steps per slice, so T is read from
// HBM once per slice and the accumulator chains are short; the warps then form the slice's
// row dots r (lanes over the columns, a fixed butterfly).  Partial P per slice as for
// hh_mma_kernel.
constexpr int kHHRowsL = 64;
constexpr int kHHSliceThreads = 256;
constexpr int kHHNC = 4;
__host__ __device__ inline int hh_slice_ld(int hh) { return ((hh + 15) & ~15) + 4; }
__host__ __device__ inline size_t hh_slice_smem(int hh) {
  return (size_t)2 * kHHRowsL * hh_slice_ld(hh) * sizeof(double);
}
__global__ void __launch_bounds__(kHHSliceThreads, 3)
hh_slice_kernel(const HHTile *__restrict__ tiles, const ChanInfo *__restrict__ chans,
                const double *__restrict__ v_pphh, const double *tbuf0, const double *tbuf1,
                double *__restrict__ part, double *__restrict__ r_out, const Control *ctl,
                int gate) {
  if (skip_iteration(ctl, gate, kTrHHTiled)) return;
  extern __shared__ __align__(16) double hs_smem[];
  const HHTile tt = tiles[blockIdx.x];
  const ChanInfo &ch = chans[tt.ch];
  const double *t_old = ctl->parity ? tbuf1 : tbuf0;
  const int hh = ch.hh, ld = hh_slice_ld(hh), hh16 = ld - 4;
  const int rows = tt.rows, rows16 = (rows + 15) & ~15;
  double *Vs = hs_smem, *Ts = hs_smem + kHHRowsL * ld;
  const int64_t base = ch.t_off + (int64_t)tt.k0 * hh;
  const double *vb = v_pphh + base, *tb = t_old + base;
  // A warp per row, lanes over the columns (no integer division); columns [hh, hh16) and rows
  // [rows, rows16) are zero.
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  for (int k = warp; k < rows16; k += kHHSliceThreads / 32) {
    for (int c = lane; c < hh16; c += 32) {
      if (k < rows && c < hh) {
        cp_async8(Vs + k * ld + c, vb + (int64_t)k * hh + c);
        cp_async8(Ts + k * ld + c, tb + (int64_t)k * hh + c);
      } else {
        Vs[k * ld + c] = 0.0;
        Ts[k * ld + c] = 0.0;
      }
    }
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  double *pb = part + ch.part_off + (int64_t)tt.idx * hh * hh;
  const int n8 = (hh + 7) >> 3, nch = (n8 + kHHNC - 1) / kHHNC, items = (hh16 >> 4) * nch;
  for (int it = warp; it < items; it += kHHSliceThreads / 32) {
    const int mt = it / nch, n0 = (it - mt * nch) * kHHNC;
    double acc[kHHNC][4];
#pragma unroll
    for (int n = 0; n < kHHNC; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.0;
    for (int k16 = 0; k16 < rows16 / 16; ++k16) {
      double a[8];
#pragma unroll
      for (int i = 0; i < 8; ++i)  // A[kl][k] = V[k][kl]
        a[i] = Vs[(16 * k16 + t + 4 * (i / 2)) * ld + 16 * mt + g + 8 * (i % 2)];
#pragma unroll
      for (int n = 0; n < kHHNC; ++n) {
        if (n0 + n >= n8) break;
        double b[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) b[q] = Ts[(16 * k16 + t + 4 * q) * ld + 8 * (n0 + n) + g];
        dmma_16816(acc[n], a, b);
      }
    }
#pragma unroll
    for (int n = 0; n < kHHNC; ++n) {
      if (n0 + n >= n8) break;
      const int ij = 8 * (n0 + n) + 2 * t;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int kl = 16 * mt + g + 8 * h;
        if (kl < hh) {
          if (ij < hh) pb[kl * hh + ij] = acc[n][2 * h];
          if (ij + 1 < hh) pb[kl * hh + ij + 1] = acc[n][2 * h + 1];
        }
      }
    }
  }
  for (int k = warp; k < rows; k += kHHSliceThreads / 32) {
    double d = 0.0;
    for (int c = lane; c < hh; c += 32) d = fma(Vs[k * ld + c], Ts[k * ld + c], d);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
    if (lane == 0) r_out[ch.pp_off + tt.k0 + k] = d;
  }
  __syncthreads();
  trace_end(ctl, kTrHHTiled);
}

// Item = 256 consecutive elements P[kl][ij] (row-major) of channel ch, from idx0.
struct HHRed {
  int32_t ch, idx0;
};
__global__ void __launch_bounds__(256)
hh_reduce_kernel(const HHRed *__restrict__ items, const ChanInfo *__restrict__ chans,
                 const double *__restrict__ v_hhhh, const double *__restrict__ part,
                 double *__restrict__ x_ref, double *__restrict__ x_t, double *__restrict__ s_out,
                 __nv_bfloat16 *__restrict__ xt_tc, int64_t xt_tc_stride, int nt,
                 const Control *ctl, int gate) {
  if (skip_iteration(ctl, gate, kTrHHReduce)) return;
  const HHRed it = items[blockIdx.x];
  const ChanInfo ch = chans[it.ch];
  const int hh = ch.hh, nout = hh * hh, idx = it.idx0 + threadIdx.x;
  if (idx >= nout) return;
  const double *pb = part + ch.part_off + idx;
  // Eight interleaved partial sums over the slices (their loads independent, so they are in
  // flight together), combined in a fixed order.
  double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  int sl = 0;
  // Sixteen slices' loads in flight together, then added to the same partial sums in the same
  // order as the eight-slice rounds below.
  for (; sl + 16 <= ch.nhht; sl += 16) {
    double x[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = __ldcg(pb + (int64_t)(sl + k) * nout);
#pragma unroll
    for (int k = 0; k < 16; ++k) acc[k & 7] += x[k];
  }
  for (; sl + 8 <= ch.nhht; sl += 8) {
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[k] += __ldcg(pb + (int64_t)(sl + k) * nout);
  }
  for (; sl < ch.nhht; ++sl) acc[0] += __ldcg(pb + (int64_t)sl * nout);
  const double p =
      ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
  hh_finish(ch, idx / hh, idx - (idx / hh) * hh, p, v_hhhh, x_ref, x_t, s_out, xt_tc,
            xt_tc_stride, nt);
  trace_end(ctl, kTrHHReduce);
}

// ------------------------------------------------------------------------------------------
// Ring term: Y = V_hphp + 0.5 V_hpph T', R = T' Y per modified channel (calc.cpp:264-313).
// T' is read from the phhp slab (t2Old_phhp; the fused assembly keeps it current); V_hpph is
// held transposed per channel (Vt[k][i] = V_hpph[i][k], k < ph', i < hp').  Result
// layout: fused path (inv != null) scatters R into pphh order, out[inv[p]] = R[p] (inv =
// inverse of the ai_jb table), so the assembly reads R_ai,jb / R_aj,ib / R_bi,ja / R_bj,ia from
// the channel's own block; table path (inv == null) writes t2Diff_phhp, out[p] = R[p].
// Channels with ph', hp' <= kRingSmall run one per warp; larger ones one per CTA, grouped by
// padded size (ring16_kernel).
// ------------------------------------------------------------------------------------------
constexpr int kRingSmall = 16;

// T' for the ring on the fused path: the phhp slab gathered from the current amplitudes,
// phhp[p] = t[inv[p]] (inv = inverse of the ai_jb table, a permutation of the n elements), at
// the head of the ring stream: coalesced index loads and slab stores, scattered reads of t
// (which the previous assembly has just written, so mostly L2 hits).  Eight elements per
// thread, all their loads in flight together.  gate < 0: run outside the iteration gating
// (a read of the slab after a solve).
constexpr int kGatherPer = 8;
__global__ void __launch_bounds__(256)
phhp_gather_kernel(const int32_t *__restrict__ inv, int64_t n, const double *tbuf0,
                   const double *tbuf1, double *__restrict__ phhp, const Control *ctl, int gate) {
  if (gate >= 0) {
    if (skip_iteration(ctl, gate, kTrGather)) return;
  } else {
    pdl_enter();
  }
  const double *__restrict__ t = ctl->parity ? tbuf1 : tbuf0;
  const int64_t p0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * kGatherPer;
  if (p0 >= n) return;
  int32_t idx[kGatherPer];
  double v[kGatherPer];
  if (p0 + kGatherPer <= n) {
    const int4 a = __ldg(reinterpret_cast<const int4 *>(inv + p0));
    const int4 b = __ldg(reinterpret_cast<const int4 *>(inv + p0) + 1);
    idx[0] = a.x; idx[1] = a.y; idx[2] = a.z; idx[3] = a.w;
    idx[4] = b.x; idx[5] = b.y; idx[6] = b.z; idx[7] = b.w;
#pragma unroll
    for (int k = 0; k < kGatherPer; ++k) v[k] = __ldcg(t + idx[k]);
    double2 *o = reinterpret_cast<double2 *>(phhp + p0);
#pragma unroll
    for (int k = 0; k < kGatherPer / 2; ++k) o[k] = make_double2(v[2 * k], v[2 * k + 1]);
  } else {
    for (int64_t p = p0; p < n; ++p) phhp[p] = __ldcg(t + inv[p]);
  }
  if (gate >= 0) trace_end(ctl, kTrGather);
}

// C (M8*8 x N8*8) = A B, K4*4 deep, on 8 x 8 tiles: warps warp, warp + nwarps, ... take items of
// one 8-row tile by NC column tiles (the A fragment is reused NC times).  A[m][k] =
// A[m * ars + k * aks], B[k][n] = B[k * ldb + n]; epi(row, col, value) stores each result.
template <int NC, class Epi>
__device__ __forceinline__ void warp_mma_gemm(const double *A, int ars, int aks, const double *B,
                                              int ldb, int M8, int N8, int K4, int warp,
                                              int nwarps, const Epi &epi) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int nch = (N8 + NC - 1) / NC;
  for (int it = warp; it < M8 * nch; it += nwarps) {
    const int mt = it / nch, n0 = (it - mt * nch) * NC, nn = min(NC, N8 - n0);
    double acc[NC][2];
#pragma unroll
    for (int n = 0; n < NC; ++n) acc[n][0] = acc[n][1] = 0.0;
    const double *ap = A + (mt * 8 + g) * ars + t * aks;
    const double *bp = B + t * ldb + n0 * 8 + g;
    const int astep = 4 * aks, bstep = 4 * ldb;
#pragma unroll 2
    for (int k4 = 0; k4 < K4; ++k4) {
      const double a = ap[k4 * astep];
#pragma unroll
      for (int n = 0; n < NC; ++n)
        if (n < nn) dmma_884(acc[n], a, bp[k4 * bstep + n * 8]);
    }
#pragma unroll
    for (int n = 0; n < NC; ++n)
      if (n < nn) {
        const int r = mt * 8 + g, c = (n0 + n) * 8 + 2 * t;
        epi(r, c, acc[n][0]);
        epi(r, c + 1, acc[n][1]);
      }
  }
}

__host__ __device__ inline int ring_pad8(int n) { return (n + 7) & ~7; }

// Channels with ph', hp' <= kRingSmall, one per warp (kRingSmallWarps per CTA), the same two
// products on the FP64 MMA: the warp's stage is padded to P, H in {8, 16} with zeros and a row
// stride of 20 doubles (4 mod 8: conflict-free fragment loads); R goes straight to global
// memory (scattered through the inverse ai_jb table on the fused path).
constexpr int kRingSmallWarps = 4;
constexpr int kRingSmallLd = kRingSmall + 4;
__global__ void __launch_bounds__(kRingSmallWarps * 32)
ring_small_kernel(const ModInfo *__restrict__ mods, int n, const double *__restrict__ v_hpph,
                  const double *__restrict__ v_hphp, const double *__restrict__ t_phhp,
                  const int32_t *__restrict__ inv, double *__restrict__ out, const Control *ctl,
                  int gate) {
  if (skip_iteration(ctl, gate, kTrRingSmall)) return;
  __shared__ __align__(16) double buf[kRingSmallWarps][3 * kRingSmall * kRingSmallLd];
  __shared__ int32_t ibuf[kRingSmallWarps][kRingSmall * kRingSmall];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int mi = blockIdx.x * kRingSmallWarps + w;
  if (mi >= n) return;  // whole warps: the MMAs below are warp-collective
  const ModInfo m = mods[mi];
  const int ph = m.ph, hp = m.hp, P = ring_pad8(ph), H = ring_pad8(hp), ld = kRingSmallLd;
  const int hs = H == 8 ? 3 : 4;  // log2 H
  double *Ts = buf[w], *Vt = Ts + kRingSmall * ld, *Ys = Vt + kRingSmall * ld;
  // Operands by cp.async (every load of the warp in flight at once), pad cells zeroed.
  for (int e = lane; e < P * H; e += 32) {
    const int r = e >> hs, c = e & (H - 1);
    if (r < ph && c < hp) {
      const int64_t src = m.m_off + r * hp + c;
      cp_async8(Ts + r * ld + c, t_phhp + src);
      cp_async8(Vt + r * ld + c, v_hpph + src);
    } else {
      Ts[r * ld + c] = 0.0;
      Vt[r * ld + c] = 0.0;
    }
  }
  for (int e = lane; e < H * H; e += 32) {
    const int r = e >> hs, c = e & (H - 1);
    if (r < hp && c < hp) cp_async8(Ys + r * ld + c, v_hphp + m.y_off + r * hp + c);
    else Ys[r * ld + c] = 0.0;
  }
  int32_t *Is = ibuf[w];  // scatter destinations (fused path), staged with the operands
  if (inv)
    for (int p = lane; p < ph * hp; p += 32) cp_async4(Is + p, inv + m.m_off + p);
  cp_async_commit();
  cp_async_wait<0>();
  __syncwarp();
  // A[i][k] = V_hpph[i][k] = Vt[k][i]; each Y element is read and written by its owner lane.
  warp_mma_gemm<2>(Vt, 1, ld, Ts, ld, H / 8, H / 8, P / 4, 0, 1,
                   [&](int r, int c, double v) { Ys[r * ld + c] = 0.5 * v + Ys[r * ld + c]; });
  __syncwarp();
  warp_mma_gemm<2>(Ts, ld, 1, Ys, ld, P / 8, H / 8, H / 4, 0, 1, [&](int r, int c, double v) {
    if (r < ph && c < hp) {
      const int p = r * hp + c;
      out[inv ? (int64_t)Is[p] : m.m_off + p] = v;
    }
  });
  trace_end(ctl, kTrRingSmall);
}

// Channels with ph', hp' > kRingSmall: one CTA per channel, the two products on the FP64
// m16n8k16 MMA (4 k-steps for a 64-wide channel instead of 14 with m8n8k4, so a warp's
// accumulator chains are short).  The channel is padded to PAD (a multiple of 16) with zeros
// in shared memory: T' [PAD][ld], Vt [PAD][ld], Y [PAD][ld] (V_hphp on arrival), ld = PAD + 4
// (4 mod 16 doubles: conflict-free fragment loads), all loaded with cp.async.  Warp w takes
// items of one 16-row tile by NC 8-column tiles.  Channels are grouped by PAD (32, 48, 64, 80),
// one launch per group, so a CTA's shared memory fits its channel and several CTAs share an SM.
constexpr int kRing16NC = 4;
__host__ __device__ constexpr int ring16_warps(int pad) {
  return (pad / 16) * ((pad / 8 + kRing16NC - 1) / kRing16NC);
}
// Operand buffers: the 32 group keeps two (T', V_hpph; Y replaces V_hpph, V_hphp is read into
// the accumulators), so that 8 CTAs share an SM; the wider groups three (T', V_hpph, V_hphp ->
// Y), which measured faster for them.
__host__ __device__ constexpr int ring16_bufs(int pad) { return pad <= 32 ? 2 : 3; }
__host__ __device__ constexpr size_t ring16_smem(int pad) {
  return (size_t)ring16_bufs(pad) * pad * (pad + 4) * sizeof(double);
}
// CTAs per SM that the shared memory allows (227 KB), kept by the register budget too.
__host__ __device__ constexpr int ring16_ctas(int pad) {
  return (int)((227 * 1024) / ring16_smem(pad)) > 8 ? 8 : (int)((227 * 1024) / ring16_smem(pad));
}
// init(slot, r, c) gives the starting accumulator of every output position of an item before
// its MMAs (it may also start loads that epi(r, c, v, slot) then uses: slot = n * 4 + the
// accumulator index).
template <int PAD, int MODE, class Init, class Epi>
__device__ __forceinline__ void ring16_gemm(const double *As, const double *Bs, int warp,
                                            const Init &init, const Epi &epi) {
  // MODE 0: A[m][k] = As[k][m] (k-major); MODE 1: A[m][k] = As[m][k].  B[k][n] = Bs[k][n].
  constexpr int ld = PAD + 4, N8 = PAD / 8, NCH = (N8 + kRing16NC - 1) / kRing16NC;
  constexpr int ITEMS = (PAD / 16) * NCH;
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  for (int it = warp; it < ITEMS; it += ring16_warps(PAD)) {
    const int mt = it / NCH, n0 = (it - mt * NCH) * kRing16NC;
    double acc[kRing16NC][4];
#pragma unroll
    for (int n = 0; n < kRing16NC; ++n) {
      const int r = 16 * mt + g, c = 8 * (n0 + n) + 2 * t;
      acc[n][0] = init(n * 4 + 0, r, c);
      acc[n][1] = init(n * 4 + 1, r, c + 1);
      acc[n][2] = init(n * 4 + 2, r + 8, c);
      acc[n][3] = init(n * 4 + 3, r + 8, c + 1);
    }
#pragma unroll
    for (int k16 = 0; k16 < PAD / 16; ++k16) {
      double a[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int m = 16 * mt + g + 8 * (i % 2), k = 16 * k16 + t + 4 * (i / 2);
        a[i] = MODE == 0 ? As[k * ld + m] : As[m * ld + k];
      }
#pragma unroll
      for (int n = 0; n < kRing16NC; ++n) {
        if (n0 + n >= N8) break;
        double b[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) b[q] = Bs[(16 * k16 + t + 4 * q) * ld + 8 * (n0 + n) + g];
        dmma_16816(acc[n], a, b);
      }
    }
#pragma unroll
    for (int n = 0; n < kRing16NC; ++n) {
      if (n0 + n >= N8) break;
      const int r = 16 * mt + g, c = 8 * (n0 + n) + 2 * t;
      epi(r, c, acc[n][0], n * 4 + 0);
      epi(r, c + 1, acc[n][1], n * 4 + 1);
      epi(r + 8, c, acc[n][2], n * 4 + 2);
      epi(r + 8, c + 1, acc[n][3], n * 4 + 3);
    }
  }
}
template <int PAD>
__global__ void __launch_bounds__(32 * ring16_warps(PAD), ring16_ctas(PAD))
ring16_kernel(const ModInfo *__restrict__ mods, const double *__restrict__ v_hpph,
              const double *__restrict__ v_hphp, const double *__restrict__ t_phhp,
              const int32_t *__restrict__ inv, double *__restrict__ out, const Control *ctl,
              int gate) {
  if (skip_iteration(ctl, gate, PAD <= 32 ? kTrRingMid : kTrRingLarge)) return;
  extern __shared__ __align__(16) double r16[];
  constexpr int ld = PAD + 4, NT = 32 * ring16_warps(PAD), N8 = PAD / 8;
  constexpr int NCH = (N8 + kRing16NC - 1) / kRing16NC;
  constexpr bool TWO = ring16_bufs(PAD) == 2;
  static_assert((PAD / 16) * NCH == ring16_warps(PAD), "one GEMM item per warp");
  double *Ts = r16, *Vs = r16 + PAD * ld, *Ys = TWO ? Vs : r16 + 2 * PAD * ld;
  const ModInfo m = mods[blockIdx.x];
  const int ph = m.ph, hp = m.hp;
  for (int e = threadIdx.x; e < PAD * PAD; e += NT) {
    const int r = e / PAD, c = e - r * PAD;
    if (r < ph && c < hp) {
      const int64_t src = m.m_off + (int64_t)r * hp + c;
      cp_async8(Ts + r * ld + c, t_phhp + src);
      cp_async8(Vs + r * ld + c, v_hpph + src);
    } else {
      Ts[r * ld + c] = 0.0;
      Vs[r * ld + c] = 0.0;
    }
    if constexpr (!TWO) {
      if (r < hp && c < hp) cp_async8(Ys + r * ld + c, v_hphp + m.y_off + (int64_t)r * hp + c);
      else Ys[r * ld + c] = 0.0;
    }
  }
  cp_async_commit();
  const int warp = threadIdx.x >> 5;
  if constexpr (TWO) {
    // 2 Y = 2 V_hphp + V_hpph T' (V_hpph[i][k] = Vt[k][i]): the accumulators start from
    // 2 V_hphp (global loads issued while the stage lands) and are halved on the way into the
    // V_hpph buffer, once every warp is done reading it.
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int mt = warp / NCH, n0 = (warp - mt * NCH) * kRing16NC;
    double y[4 * kRing16NC];
    cp_async_wait<0>();
    __syncthreads();
    ring16_gemm<PAD, 0>(
        Vs, Ts, warp,
        [&](int, int r, int c) {
          return (r < hp && c < hp) ? 2.0 * __ldg(v_hphp + m.y_off + (int64_t)r * hp + c) : 0.0;
        },
        [&](int, int, double v, int slot) { y[slot] = 0.5 * v; });
    __syncthreads();
#pragma unroll
    for (int slot = 0; slot < 4 * kRing16NC; ++slot) {
      const int n = slot >> 2, q = slot & 3;
      if (n0 + n < N8)
        Ys[(16 * mt + g + 8 * (q >> 1)) * ld + 8 * (n0 + n) + 2 * t + (q & 1)] = y[slot];
    }
  } else {
    // Y = V_hphp + 0.5 V_hpph T' in the third buffer; each Y element has one owner lane.
    cp_async_wait<0>();
    __syncthreads();
    ring16_gemm<PAD, 0>(
        Vs, Ts, warp, [](int, int, int) { return 0.0; },
        [&](int r, int c, double v, int) { Ys[r * ld + c] = 0.5 * v + Ys[r * ld + c]; });
  }
  __syncthreads();
  // R = T' Y, stored for r < ph', c < hp' (through the inverse ai_jb table on the fused path);
  // the destinations are loaded before the MMAs, so the stores do not wait on them.
  int32_t dst[4 * kRing16NC];
  ring16_gemm<PAD, 1>(
      Ts, Ys, warp,
      [&](int slot, int r, int c) {
        const int32_t p = (int32_t)(m.m_off + (int64_t)r * hp + c);
        dst[slot] = (r < ph && c < hp) ? (inv ? __ldg(inv + p) : p) : -1;
        return 0.0;
      },
      [&](int, int, double v, int slot) {
        if (dst[slot] >= 0) out[dst[slot]] = v;
      });
  trace_end(ctl, PAD <= 32 ? kTrRingMid : kTrRingLarge);
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
                                     double *__restrict__ yp, const Control *ctl, int gate) {
  if (skip_iteration(ctl, gate, kTrOneBody)) return;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= nsp) return;
  const bool hole = w < np;
  const double *src = hole ? s : r;
  // Eight lane-strided partial sums: the eight index loads of a round are issued together,
  // then the eight value loads, so a round costs two memory latencies; the last round of a
  // list is guarded (lists are mostly shorter than one round).
  double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  const int64_t hi = list_off[w + 1];
  for (int64_t e = list_off[w] + lane; e < hi; e += 256) {
    int32_t ix[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) ix[k] = e + 32 * k < hi ? __ldg(list + e + 32 * k) : -1;
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (ix[k] >= 0) acc[k] += __ldcg(src + ix[k]);
  }
  double v = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (lane == 0) {
    if (hole) xh[w] = v;
    else yp[w - np] = v;
  }
  trace_end(ctl, kTrOneBody);
}

// Writes one amplitude into the ladder operand tiles: the B tiles of V T (rows c<d) and the A
// tiles of T X (rows a<=b, compact last row tile).  pk_idx[AB] = (K index or -1, packed row
// or -1).
__device__ __forceinline__ void write_t_tiles_q(const ChanInfo &ch, int2 q, int ij, double t,
                                                double *t_kt, double *t_mt) {
  const int bs = ladder_bs(ch.nb);
  if (q.x >= 0) t_kt[ch.tkt_base + (int64_t)(q.x / kBK) * kBK * bs + (q.x % kBK) * bs + ij] = t;
  if (q.y >= 0) {
    const int mt = q.y / ch.bm, rows = min(ch.bm, ch.pr - mt * ch.bm);
    const int ar = ladder_arows(ch.nb, rows);
    t_mt[ch.tmt_base + (int64_t)mt * ladder_arows_full(ch.nb) * ch.nkh * kBK +
         (int64_t)(ij / kBK) * ar * kBK +
         ladder_aoff(ch.nb, ar, q.y - mt * ch.bm, ij % kBK)] = t;
  }
}
__device__ __forceinline__ void write_t_tiles(const ChanInfo &ch, const int2 *__restrict__ pk_idx,
                                              int ab, int ij, double t, double *t_kt,
                                              double *t_mt) {
  write_t_tiles_q(ch, pk_idx[ch.pp_off + ab], ij, t, t_kt, t_mt);
}

// The same amplitude into the mixed-precision operand images: nt bf16 terms of T in the
// tensor-core chunk layout (tc_off), V T operand B (K = c<d pair) and T X operand A (rows a<=b,
// compact last 128-row tile, K = hh).
template <int NT>
__device__ __forceinline__ void write_t_tiles_tc_n(const ChanInfo &ch, int2 q, int ij, double t,
                                                   __nv_bfloat16 *tkt_tc, int64_t tkt_stride,
                                                   __nv_bfloat16 *tmt_tc, int64_t tmt_stride) {
  __nv_bfloat16 hv[NT];
  split_bf16_n<NT>(t, hv);
  if (q.x >= 0) {
    const int64_t o =
        ch.tkt_tc_base + (int64_t)(q.x >> 5) * (ch.nbt >> 3) * kTcGroup + tc_off_mn(ij, q.x & 31);
#pragma unroll
    for (int p = 0; p < NT; ++p) tkt_tc[p * tkt_stride + o] = hv[p];
  }
  if (q.y >= 0) {
    const int mt = q.y >> 7, r = q.y & 127;
    const int rg = (min(kTcBM, ch.pr - mt * kTcBM) + 7) >> 3;
    const int64_t o = ch.tmt_tc_base + (int64_t)mt * kTcBM * ch.nkht * kTcKC +
                      (int64_t)(ij >> 5) * rg * kTcGroup + tc_off(r, ij & 31);
#pragma unroll
    for (int p = 0; p < NT; ++p) tmt_tc[p * tmt_stride + o] = hv[p];
  }
}
__device__ __forceinline__ void write_t_tiles_tc(const ChanInfo &ch, int2 q, int ij, double t,
                                                 int nt, __nv_bfloat16 *tkt_tc,
                                                 int64_t tkt_stride, __nv_bfloat16 *tmt_tc,
                                                 int64_t tmt_stride) {
  if (q.x < 0 && q.y < 0) return;  // row ba of a mirrored pair: in neither image
  if (nt == 3) write_t_tiles_tc_n<3>(ch, q, ij, t, tkt_tc, tkt_stride, tmt_tc, tmt_stride);
  else write_t_tiles_tc_n<2>(ch, q, ij, t, tkt_tc, tkt_stride, tmt_tc, tmt_stride);
}

// ------------------------------------------------------------------------------------------
// Fused assembly (calc.cpp:384-418 plus the remaps folded in):
//   value = V + D + R_ai,jb - R_aj,ib - R_bi,ja + R_bj,ia          (4 gathers from R in phhp layout)
//         + 0.5 x_i t_ab,ji - 0.5 x_j t_ab,ij                       (h2pp_h1 gathers, algebraically)
//         + (-0.5 y_b) t_ab,ij - (-0.5 y_a) t_ba,ij                 (p2_p1hh gathers, algebraically)
//   t_new = mixing value/(e_i+e_j-e_a-e_b) + (1-mixing) t_old;  E += V t_new
// and the next iteration's ladder operand tiles are written in the same pass (the ring's phhp
// slab is gathered from t_new by phhp_gather_kernel at the head of the next iteration's ring
// stream: mapToDistributed ai_jb as a coalesced write instead of a scattered one here).
// ------------------------------------------------------------------------------------------
constexpr int kAsmThreads = 256;
constexpr int kAsmPerThread = 2;  // table path: elements per thread of an ElemRange
__device__ __forceinline__ void energy_reduce(const double *epart, int n, Control *ctl, int flags,
                                              double *e_out);
// Condition of the device solve loop's WHILE node after an iteration: another iteration while
// the stop rule has not fired, below the launch's iteration limit, and (body_mixed) in the
// mixed phase or (FP64 body) past it.
__device__ __forceinline__ void loop_set_condition(const Control *ctl,
                                                   cudaGraphConditionalHandle cond,
                                                   bool body_mixed) {
  const bool more = !ctl->done && ctl->iterations < ctl->stop_at;
  const bool mixed_phase = ctl->phase == 1;
  cudaGraphSetConditional(cond, (more && (body_mixed ? mixed_phase : !mixed_phase)) ? 1u : 0u);
}

// Work is organised over quads (u, w): strict packed row u (a < b) of a channel and strict hole
// pair w (i < j).  The amplitudes are antisymmetric, t_ab,ij = -t_ab,ji = -t_ba,ij = t_ba,ji,
// and so are V, D and the combination of the four R terms; the fused path keeps them exactly
// so (the ladders write D[ba] = -D[ab]; a quad writes its four elements as +t, -t, -t, +t), and
// rows a = b or columns i = j hold zeros that no iteration changes.  One thread computes the
// quad's element (ab, ij) from V, D, t at (ab, ij) and R at the four positions, and writes all
// four elements and the operand-image entries of rows ab (row ba is in neither image).  The energy gains 4 V t_new per quad.
// Persistent CTAs stride over work items of up to kQuadPerItem quads of one channel; a thread
// takes one quad of an item and issues all its loads before the first store.
// In a mixed iteration (nt > 0) only the bf16 operand images are written; retile_kernel
// rebuilds the FP64 tiles if FP64 iterations follow.
constexpr int kQuadPerItem = kAsmThreads;  // one quad per thread and item
constexpr int kAsmCTAsPerSM = 3;

// One thread's quad of a work item: where its four elements sit in the channel block, its
// operand-image indices, one-body indices and denominator.  ok = false: no quad (past the
// item or past the last item).
struct QuadRef {
  int32_t o_ab, o_ba, c_ij, c_ji, qx, qy, pa, pb, i, j, ch;
  bool ok;
  int64_t t_off;
  double den;
};
__device__ __forceinline__ void quad_fetch(const QuadItem *__restrict__ items, int n_items,
                                           const QuadRow *__restrict__ qrows,
                                           const QuadCol *__restrict__ qcols, int it,
                                           QuadRef &r) {
  r.ok = false;
  if (it >= n_items) return;
  const QuadItem item = items[it];
  const int q = item.q0 + threadIdx.x;
  if (q >= item.q1) return;
  // q / hk as a multiply-high by ceil(2^32 / hk) (Granlund-Montgomery): exact for
  // q < 2^32 / hk (q < 2^21, hk < 2^11 here); hk = 1 has no 32-bit multiplier.
  const int hk = item.hk;
  const uint32_t magic = hk > 1 ? 0xFFFFFFFFu / (uint32_t)hk + 1u : 0u;
  const int u = hk > 1 ? (int)__umulhi((uint32_t)q, magic) : q, w = q - u * hk;
  const QuadRow rw = qrows[item.qrow_off + u];
  const QuadCol cl = qcols[item.qcol_off + w];
  r.o_ab = rw.o_ab; r.o_ba = rw.o_ba; r.qx = rw.qx; r.qy = rw.qy; r.pa = rw.pa; r.pb = rw.pb;
  r.c_ij = cl.c_ij; r.c_ji = cl.c_ji; r.i = cl.i; r.j = cl.j;
  r.den = cl.eij - rw.ea - rw.eb;
  r.ch = item.ch;
  r.t_off = item.t_off;
  r.ok = true;
}

// value of element (ab, ij) (calc.cpp:384-418) with t_ab,ji = -t and t_ba,ij = -t:
//   V + D + R_ai,jb - R_aj,ib - R_bi,ja + R_bj,ia + 0.5 x_i t_ab,ji - 0.5 x_j t_ab,ij
//     + (-0.5 y_b) t_ab,ij - (-0.5 y_a) t_ba,ij
__device__ __forceinline__ double quad_value(double v, double dm, double r1, double r2, double r3,
                                             double r4, double t, double xi, double xj,
                                             double ya, double yb, double den, double mixing) {
  double value = v;
  value += dm;
  value += r1;
  value -= r2;
  value -= r3;
  value += r4;
  value += (0.5 * xi) * (-t);
  value -= (0.5 * xj) * t;
  value += (-0.5 * yb) * t;
  value -= (-0.5 * ya) * (-t);
  value = value / den;
  return mixing * value + (1. - mixing) * t;
}

// LOOP: launched as the last kernel of a device-solve-loop body (sets the WHILE condition);
// the variant without it is the one profilers can replay.
template <bool LOOP>
__global__ void __launch_bounds__(kAsmThreads, kAsmCTAsPerSM)
assemble_fused_kernel(const QuadItem *__restrict__ items, int n_items,
                      const ChanInfo *__restrict__ chans, const QuadRow *__restrict__ qrows,
                      const QuadCol *__restrict__ qcols, const double *__restrict__ v_pphh,
                      const double *__restrict__ dmat, const double *__restrict__ d_ring,
                      const double *__restrict__ xh, const double *__restrict__ yp,
                      double *tbuf0, double *tbuf1, double *__restrict__ t_kt,
                      double *__restrict__ t_mt, double *__restrict__ epart, int32_t *ticket,
                      Control *ctl, __nv_bfloat16 *__restrict__ tkt_tc, int64_t tkt_tc_stride,
                      __nv_bfloat16 *__restrict__ tmt_tc, int64_t tmt_tc_stride, int nt,
                      cudaGraphConditionalHandle cond, int loop_body, int gate) {
  // loop_body: 0 outside the device solve loop, 1 / 2 last kernel of its FP64 / mixed body,
  // where the CTA that applies the stop rule also sets the loop condition.  A skipped body
  // (stop rule fired, or the other precision's phase) ends its loop.
  __shared__ double scratch[32];
  __shared__ int last;
  if (skip_iteration(ctl, gate, kTrAssemble)) {
    if constexpr (LOOP)
      if (blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(cond, 0u);
    return;
  }
  const double *__restrict__ t_old = ctl->parity ? tbuf1 : tbuf0;
  double *__restrict__ t_new = ctl->parity ? tbuf0 : tbuf1;
  const double mixing = ctl->mixing;
  double corr = 0.0;
  // Two-stage pipeline over the CTA's items: the next item's header and this thread's row and
  // column table entries are fetched while the current quad's operand loads are in flight.
  QuadRef nx;
  quad_fetch(items, n_items, qrows, qcols, blockIdx.x, nx);
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const QuadRef cu = nx;
    double tv = 0.0, vv = 0.0, dv = 0.0, rv[4] = {0.0, 0.0, 0.0, 0.0}, xs[2] = {0.0, 0.0},
           ys[2] = {0.0, 0.0};
    int32_t pos[4];
    pos[0] = cu.o_ab + cu.c_ij;
    pos[1] = cu.o_ab + cu.c_ji;
    pos[2] = cu.o_ba + cu.c_ij;
    pos[3] = cu.o_ba + cu.c_ji;
    if (cu.ok) {
      const int64_t p0 = cu.t_off + pos[0];
      tv = t_old[p0];
      vv = __ldg(v_pphh + p0);
      dv = __ldcg(dmat + p0);
#pragma unroll
      for (int m = 0; m < 4; ++m) rv[m] = __ldcg(d_ring + cu.t_off + pos[m]);
      // The one-body sums are small arrays every quad reads: through L1 (an L2-only load
      // would send every warp to the same few L2 slices).
      xs[0] = xh[cu.i];
      xs[1] = xh[cu.j];
      ys[0] = yp[cu.pa];
      ys[1] = yp[cu.pb];
    }
    quad_fetch(items, n_items, qrows, qcols, it + gridDim.x, nx);
    if (!cu.ok) continue;
    const double t1 = quad_value(vv, dv, rv[0], rv[1], rv[2], rv[3], tv, xs[0], xs[1], ys[0],
                                 ys[1], cu.den, mixing);
    const double sg[4] = {t1, -t1, -t1, t1};
#pragma unroll
    for (int m = 0; m < 4; ++m) t_new[cu.t_off + pos[m]] = sg[m];
    const ChanInfo &ch = chans[cu.ch];
    const int2 qa = make_int2(cu.qx, cu.qy);
    if (nt) {
      write_t_tiles_tc(ch, qa, cu.c_ij, t1, nt, tkt_tc, tkt_tc_stride, tmt_tc, tmt_tc_stride);
      write_t_tiles_tc(ch, qa, cu.c_ji, -t1, nt, tkt_tc, tkt_tc_stride, tmt_tc, tmt_tc_stride);
    } else {
      write_t_tiles_q(ch, qa, cu.c_ij, t1, t_kt, t_mt);
      write_t_tiles_q(ch, qa, cu.c_ji, -t1, t_kt, t_mt);
    }
    corr += 4.0 * (vv * t1);
  }
  const double sum = block_sum<kAsmThreads>(corr, scratch);
  trace_end(ctl, kTrAssemble);
  // The last CTA to finish sums the partials and applies the stop rule (no extra launch).
  if (threadIdx.x == 0) {
    epart[blockIdx.x] = sum;
    __threadfence();
    last = (atomicAdd(ticket, 1) == (int)gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  energy_reduce(epart, gridDim.x, ctl, 3, nullptr);
  if (threadIdx.x == 0) {
    *ticket = 0;
    if (nt) ctl->retile = 1;  // the FP64 ladder tiles were not written this iteration
    if constexpr (LOOP) loop_set_condition(ctl, cond, loop_body == 2);
  }
}

// Rebuilds the FP64 ladder operand tiles from the current amplitudes after mixed iterations
// (they write only the bf16 images); a no-op unless ctl->retile is set.  First kernel of every
// FP64 iteration of the fused path and of the FP64 ladder stage.
__global__ void __launch_bounds__(256)
retile_kernel(const ElemRange *__restrict__ ranges, const ChanInfo *__restrict__ chans,
              const int2 *__restrict__ pk_idx, const double *tbuf0, const double *tbuf1,
              double *__restrict__ t_kt, double *__restrict__ t_mt, Control *ctl, int gate) {
  if (skip_iteration(ctl, gate, kTrRetile) || !ctl->retile) return;
  const ElemRange rg = ranges[blockIdx.x];
  const ChanInfo ch = chans[rg.ch];
  const double *t = ctl->parity ? tbuf1 : tbuf0;
  for (int64_t e = rg.e0 + threadIdx.x; e < rg.e1; e += blockDim.x) {
    const int64_t loc = e - ch.t_off;
    const int ab = (int)(loc / ch.hh), ij = (int)(loc - (int64_t)ab * ch.hh);
    write_t_tiles(ch, pk_idx, ab, ij, t[e], t_kt, t_mt);
  }
}

// Clears the retile flag once every retile CTA has read it (single thread, after retile).
__global__ void retile_done_kernel(Control *ctl) {
  pdl_enter();
  if (threadIdx.x == 0) ctl->retile = 0;
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
                              double *__restrict__ t_mt, int with_3body,
                              __nv_bfloat16 *__restrict__ tkt_tc, int64_t tkt_tc_stride,
                              __nv_bfloat16 *__restrict__ tmt_tc, int64_t tmt_tc_stride, int nt) {
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
    if (nt) write_t_tiles_tc(ch, pk_idx[ch.pp_off + ab], ij, t, nt, tkt_tc, tkt_tc_stride,
                             tmt_tc, tmt_tc_stride);
  }
}

// Sum of the per-CTA energy partials (Neumaier-compensated, fixed order) by one block of
// kEnergyThreads threads, then the reference's stop rule on the device.  flags: 1 = flip the
// amplitude buffer parity, 2 = count this as an iteration of the solve loop.
constexpr int kEnergyThreads = 256;
__device__ __forceinline__ void energy_reduce(const double *epart, int n, Control *ctl, int flags,
                                              double *e_out) {
  __shared__ double ss[kEnergyThreads], cs[kEnergyThreads];
  double s = 0.0, c = 0.0;
  for (int i = threadIdx.x; i < n; i += kEnergyThreads) {
    const double x = __ldcg(epart + i);
    const double t = s + x;
    c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
    s = t;
  }
  ss[threadIdx.x] = s;
  cs[threadIdx.x] = c;
  __syncthreads();
  for (int w = kEnergyThreads / 2; w > 0; w >>= 1) {
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
      const double diff = corr - ctl->e_prev, prev_diff = ctl->e_diff;
      ctl->e_prev = corr;
      ctl->e_corr = corr;
      ctl->e_diff = diff;
      if (ctl->iterations < 128) ctl->energies[ctl->iterations] = corr;
      ctl->iterations += 1;
      if (ctl->active && ctl->phase == 2) ctl->polish_iters += 1;
      if (!isfinite(corr)) {
        ctl->error |= kErrNonFinite;
        ctl->done = 1;
      }
      if (ctl->active && ctl->phase == 1) {
        // Mixed phase: hand over to FP64 iterations once the energy change reaches the
        // rounding floor of the split-bf16 ladder, or stops shrinking.
        if (fabs(diff) <= fmax(ctl->tol, ctl->polish_rel * fabs(corr)) ||
            (ctl->iterations > 2 && fabs(diff) >= fabs(prev_diff)))
          ctl->phase = 2;
        if (ctl->iterations > ctl->max_iters) ctl->done = 1;
      } else if (fabs(diff) <= ctl->tol || ctl->iterations > ctl->max_iters) {
        ctl->done = 1;
      }
    }
    if (flags & 1) ctl->parity ^= 1;
  }
}

// Last node of an iteration body of the device solve loop (a CUDA graph with WHILE conditional
// nodes) when the system has no assembly blocks: decides from the control block whether the
// loop runs another iteration.  body_mixed: the mixed-precision loop continues in phase 1 only;
// the FP64 loop never runs in phase 1.  Otherwise the fused assembly, the last kernel of every
// body, sets the condition (also when it skipped), so no loop can spin without progress: a
// body either advances `iterations` or clears its condition.
__global__ void loop_ctl_kernel(const Control *ctl, cudaGraphConditionalHandle cond,
                                int body_mixed) {
  pdl_enter();
  trace_start(ctl, kTrLoopCtl);
  if (threadIdx.x != 0) return;
  loop_set_condition(ctl, cond, body_mixed != 0);
}

// MBPT2 (MBPT2Corr.cpp:6-38) over the elements of the active channels, one CTA per range:
// epart[range] = sum <ij|v|ab>^2 / (e_i + e_j - e_a - e_b) (energy_reduce applies the 1/4), and
// with t_out the first-order amplitudes t_ab,ij = <ab|v|ij> / (e_i + e_j - e_a - e_b).
__global__ void __launch_bounds__(256)
mbpt2_kernel(const ElemRange *__restrict__ ranges, const ChanInfo *__restrict__ chans,
             const int2 *__restrict__ pp_pairs, const int2 *__restrict__ hh_pairs,
             const double *__restrict__ v_pphh, const double *__restrict__ eps,
             double *__restrict__ t_out, double *__restrict__ epart) {
  __shared__ double scratch[32];
  const ElemRange rg = ranges[blockIdx.x];
  const ChanInfo ch = chans[rg.ch];
  double acc = 0.0;
  for (int64_t e = rg.e0 + threadIdx.x; e < rg.e1; e += blockDim.x) {
    const int64_t loc = e - ch.t_off;
    const int ab = (int)(loc / ch.hh), ij = (int)(loc - (int64_t)ab * ch.hh);
    const int2 pab = pp_pairs[ch.pp_off + ab], pij = hh_pairs[ch.hh_off + ij];
    const double den = eps[pij.x] + eps[pij.y] - eps[pab.x] - eps[pab.y];
    const double v = v_pphh[e];
    acc += v * v / den;
    if (t_out) t_out[e] = v / den;
  }
  const double sum = block_sum<256>(acc, scratch);
  if (threadIdx.x == 0) epart[blockIdx.x] = sum;
}

__global__ void __launch_bounds__(kEnergyThreads)
energy_kernel(const double *__restrict__ epart, int n, Control *ctl, int flags, double *e_out,
              int gate) {
  if (skip_iteration(ctl, gate, kTrEnergy)) return;
  energy_reduce(epart, n, ctl, flags, e_out);
}

}  // namespace ccd
