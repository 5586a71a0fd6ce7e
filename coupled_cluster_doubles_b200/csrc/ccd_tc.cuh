// Mixed-precision pp ladder on the 5th-generation tensor cores (tcgen05, sm_100a).
//
//   D[ab,:] = sum_{c<d} V[ab,cd] T[cd,:] + T[ab,:] (X/2)        packed rows a <= b
//
// is the same antisymmetry-packed product as pp_ladder_kernel (calc.cpp:162-202), with every
// operand split into NT bf16 terms, x = x_0 + x_1 (+ x_2), each term the bf16 rounding of what
// the previous ones leave.  The products x_p y_q with p + q < NT are summed by
// tcgen05.mma.kind::f16 (bf16 inputs, FP32 accumulator in tensor memory): NT = 2 carries
// about 17 significant bits per operand, NT = 3 about 25.  The ladder is the only mixed
// contraction; the CCD iteration around it stays FP64, and the solver finishes with FP64
// iterations (the fixed point does not depend on how D was rounded on the way).
//
// Operand images.  A 128-row x 32-deep K chunk of one term is stored in HBM exactly as the
// tensor core reads it from shared memory: non-swizzled canonical layouts made of 8 x 8 "core
// matrices" (128 contiguous bytes), K-major for A (V, and T rows for T X):
//   element (r, k) of a chunk -> (r / 8) * 256 + (k / 8) * 64 + (r % 8) * 8 + k % 8   (bf16)
// and MN-major for B (T for V T, X/2): element (n, k) -> (n / 8) * 256 + (k / 8) * 64 +
// (k % 8) * 8 + n % 8 (tc_off / tc_off_mn in ccd_device.cuh).  One 1-D bulk copy per term moves
// a stage, and both smem descriptors use LBO = 128 bytes (next core matrix along K) and
// SBO = 512 bytes (next 8-row / 8-column group).  The last row tile of a channel is compact (only its ceil(rows/8) row groups are
// stored); the rows beyond it in shared memory are stale and only reach accumulator rows that
// the epilogue never reads.  K padding is zero in both operands.
//
// CTA roles (192 threads): warps 0-3 read the accumulator back (warp w owns TMEM lanes
// 32w..32w+31 = tile rows), warp 4 is the bulk-copy producer, warp 5 allocates tensor memory
// and one of its lanes issues the MMAs.  Every mbarrier wait is bounded (kWaitLimitNs); on a
// timeout the kernel sets kErrTimeout, lets the copies it issued land, waits for its MMAs and
// frees its tensor memory before returning.
#pragma once

#include <cuda_bf16.h>

#include <cstdint>
#include <type_traits>

#include "ccd_device.cuh"
#include "ccd_kernels.cuh"

namespace ccd {

__host__ __device__ constexpr int tc_stages(int nt) { return nt == 2 ? 4 : 3; }
__host__ __device__ constexpr size_t tc_stage_bytes(int nt) {
  return (size_t)nt * (kTcAPlane + kTcBPlane) * 2;
}
// V_pppp generated inside the ladder (electron gas): generator warps.
constexpr int kTcGenWarps = 4;
__host__ __device__ constexpr int tc_threads(bool gen) {
  return kTcThreads + (gen ? 32 * kTcGenWarps : 0);
}
// Dynamic shared memory: 1024 bytes of alignment slack, the stages, then the barriers
// (2 S + 5 + 2 kTcTQ of them).  (The generator's q^2 table is a static shared array.)
__host__ __device__ constexpr size_t tc_smem_bytes(int nt) {
  return 1024 + tc_stages(nt) * tc_stage_bytes(nt) + 256;
}

// ---- V_pppp of the electron gas generated in the ladder ----------------------------------
// <ab|v|cd> = [s_a = s_c] w(|n_a - n_c|^2) - [s_b = s_c] w(|n_c - n_b|^2)
// (ElectronGasSPBasis.cpp:418-471: direct minus exchange, spin-diagonal Coulomb term that
// depends only on the momentum transfer, zero at q = 0).  Inside a channel n_a + n_b = n_c + n_d
// and s_a + s_b = s_c + s_d, so n_a - n_d = n_c - n_b, and s_a = s_c implies s_b = s_d (the
// direct term's other spin condition) as s_b = s_c implies s_a = s_d.  An orbital's code holds
// n_x, n_y, n_z biased by 64 in bytes 0-2 and kVGenSpin * [s > 0] in byte 3.  For two codes,
// (x - y + 0x80808080) ^ 0x80808080 holds the signed byte differences (every biased byte
// difference lies in [107, 149], so nothing borrows across bytes), and one dp4a of it with
// itself gives q^2 plus kVGenSpin^2 = 441 > 432 when the spins differ.  w is a table by that
// index, zero at 0 and beyond 432: spin mismatches and q = 0 read zeros.  FP32 for the 2-term
// split (which keeps about 16 bits), FP64 for the 3-term split, so the element is exact to the
// precision its split carries.
struct VGenRow {
  uint32_t na, nb;
};
constexpr uint32_t kVGenZero = 0x404040u;  // momentum (0, 0, 0), spin down, biased
constexpr int kVGenSpin = 21;
constexpr int kTcGenTab = 3 * 12 * 12 + kVGenSpin * kVGenSpin + 1;  // |n_i| <= 6: 874 entries
template <int NT>
using VGenT = typename std::conditional<NT == 3, double, float>::type;
__device__ __forceinline__ int vgen_q2(uint32_t x, uint32_t y) {
  const int d = (int)((x - y + 0x80808080u) ^ 0x80808080u);
  return __dp4a(d, d, 0);
}
template <typename T>
__device__ __forceinline__ T vgen_elem(const VGenRow &r, uint32_t nc, const T *tab) {
  return tab[vgen_q2(r.na, nc)] - tab[vgen_q2(r.nb, nc)];
}
// Two K-adjacent elements -> one 32-bit word (element k in the low half) of the current bf16
// term, and the remainders for the next term.
__device__ __forceinline__ uint32_t vgen_split(float &x0, float &x1) {
  const __nv_bfloat162 t = __floats2bfloat162_rn(x0, x1);
  x0 -= __low2float(t);
  x1 -= __high2float(t);
  return *reinterpret_cast<const uint32_t *>(&t);
}
__device__ __forceinline__ uint32_t vgen_split(double &x0, double &x1) {
  const __nv_bfloat16 a = __double2bfloat16(x0), b = __double2bfloat16(x1);
  x0 -= (double)__bfloat162float(a);
  x1 -= (double)__bfloat162float(b);
  const __nv_bfloat162 t = __halves2bfloat162(a, b);
  return *reinterpret_cast<const uint32_t *>(&t);
}

// --- tcgen05 / descriptor helpers --------------------------------------------------------

// Shared-memory matrix descriptor, K-major, no swizzle (sm_100 version 1 descriptor).
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) |
         ((uint64_t)(512 >> 4) << 32) | (1ull << 46);
}
// Instruction descriptor: bf16 x bf16 -> f32, A K-major, B MN-major (bit 16), M = 128, N = n.
__host__ __device__ constexpr uint32_t tc_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (1u << 16) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(kTcBM >> 4) << 24);
}
__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// Arrive (once) on an mbarrier when every tcgen05 operation this thread issued so far is done.
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// 32 lanes x 16 consecutive 32-bit columns: thread t of the warp gets lane (base + t).
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Tensor-memory columns for an N-column FP32 accumulator (a power of two, at least 32).
__host__ __device__ inline uint32_t tc_tmem_cols(int nb) {
  return nb <= 32 ? 32u : nb <= 64 ? 64u : 128u;
}

// AND of a predicate over the 128 epilogue threads (named barrier 1): a uniform decision.
__device__ __forceinline__ bool consumers_all(bool v) {
  uint32_t r;
  asm volatile(
      "{ .reg .pred p, q; setp.ne.u32 p, %1, 0; bar.red.and.pred q, 1, %2, p; "
      "selp.u32 %0, 1, 0, q; }"
      : "=r"(r)
      : "r"((uint32_t)v), "n"(kLadderConsumers)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ int read_flag(const int *f) { return *(const volatile int *)f; }

// Bulk copies of the stages that were issued but may not have landed (error path only).
__device__ __forceinline__ void tc_drain(const uint64_t *full, int issued, int stages) {
  for (int c = issued - stages < 0 ? 0 : issued - stages; c < issued; ++c)
    (void)mbar_wait(smem_u32(&full[c % stages]), (c / stages) & 1);
}

// Persistent CTAs claim tiles from a launch-wide counter (tiles sorted by decreasing work, so
// the claims are longest-first list scheduling, and a CTA that starts late because another
// stream's kernel still holds its SM takes fewer tiles); the producer publishes each claimed
// tile in a small shared-memory queue that the MMA thread, the epilogue warps and (GEN) the
// generator warps follow.  The producer streams K chunks through the S-stage ring without a
// break at tile boundaries; the MMA thread accumulates tile number lt of the CTA into
// tensor-memory buffer lt & 1 (two 128-column accumulators), so that the epilogue warps read
// tile lt back while tile lt + 1 is loaded and multiplied.  Barriers: full / empty per stage,
// acc_full / acc_empty per accumulator (tcgen05.commit, and one arrival per epilogue warp),
// tq_full / tq_empty per queue slot.  Every wait is bounded and checks the CTA's abort flag.
// Tiles are bm = 128 rows, nb = UMMA N columns, K chunks of kTcKC; image arrays hold NT planes
// each, plane p at base + p * stride.  A mixed-phase kernel (gate 1 of skip_iteration).
constexpr uint32_t kTcAccCols = 128;  // columns of one accumulator buffer (nb <= kTcMaxNB)
constexpr int kTcTQ = 4;              // slots of a CTA's queue of claimed tiles
constexpr int kTcGrid = 2 * 148;      // persistent grid: two CTAs on each of the 148 SMs
// GEN (electron gas, V generated in the ladder): warps 6 .. 6 + kTcGenWarps - 1 write the V
// operand planes of every V T chunk into the stage (fence.proxy.async, then one arrival per
// warp on the stage's full barrier, for every chunk); the producer copies only the B planes of
// those chunks.  No V image is read from HBM.
template <int NT, bool GEN>
__global__ void __launch_bounds__(tc_threads(GEN), GEN ? 2 : 1)
pp_ladder_tc_kernel(const LadderTile *__restrict__ tiles, int n_tiles, int32_t *sched,
                    const __nv_bfloat16 *__restrict__ v_tc, int64_t v_stride,
                    const __nv_bfloat16 *__restrict__ tkt_tc, int64_t tkt_stride,
                    const __nv_bfloat16 *__restrict__ tmt_tc, int64_t tmt_stride,
                    const __nv_bfloat16 *__restrict__ xt_tc, int64_t xt_stride,
                    const int32_t *__restrict__ rowmap, const int32_t *__restrict__ mirror,
                    double *__restrict__ d, double *part, const Control *ctl, int32_t *err,
                    const ChanInfo *__restrict__ chans, const VGenRow *__restrict__ vg_rows,
                    const uint32_t *__restrict__ vg_cols, const double *__restrict__ vg_tab) {
  if (skip_iteration(ctl, 1, kTrLadderTC)) return;
  constexpr int S = tc_stages(NT);
  constexpr uint32_t kStageBytes = (uint32_t)tc_stage_bytes(NT);
  extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
  __shared__ uint32_t tmem_holder;
  __shared__ int abort_flag, issued_chunks;
  const uint32_t raw = smem_u32(tc_smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;  // stage s at base + s * kStageBytes
  uint64_t *bars = reinterpret_cast<uint64_t *>(tc_smem_raw + (base - raw) + S * kStageBytes);
  uint64_t *full = bars, *empty = bars + S, *acc_full = bars + 2 * S,
           *acc_empty = bars + 2 * S + 2, *done = bars + 2 * S + 4;
  uint64_t *tq_full = bars + 2 * S + 5, *tq_empty = tq_full + kTcTQ;
  __shared__ int tile_q[kTcTQ];
  // The generator's table: a separate shared array, so that its loads are independent of the
  // generators' stores into the stages.
  __shared__ VGenT<NT> gtab[GEN ? kTcGenTab : 1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if constexpr (GEN) {
    if (warp >= 6)
      for (int i = threadIdx.x - 192; i < kTcGenTab; i += 32 * kTcGenWarps)
        gtab[i] = (VGenT<NT>)vg_tab[i];
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(smem_u32(&full[s]), GEN ? 1 + kTcGenWarps : 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&acc_full[b]), 1);
      mbar_init(smem_u32(&acc_empty[b]), kLadderConsumers / 32);
    }
    mbar_init(smem_u32(done), 1);
    for (int q = 0; q < kTcTQ; ++q) {
      mbar_init(smem_u32(&tq_full[q]), 1);
      mbar_init(smem_u32(&tq_empty[q]), 1 + kLadderConsumers / 32 + (GEN ? kTcGenWarps : 0));
    }
    abort_flag = 0;
    issued_chunks = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(&tmem_holder)), "r"(2 * kTcAccCols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_holder;
  auto fail = [&]() {
    atomicOr(err, kErrTimeout);
    atomicExch(&abort_flag, 1);
  };
  // The k-th tile of this CTA as the producer published it (waiting for it), -1 at the end;
  // after the lanes in `mask` read it, one arrival per warp frees the slot.  `ok` = false: the
  // wait ran out.
  auto queued = [&](int k, bool &ok, unsigned mask) {
    const int slot = k % kTcTQ;
    ok = mbar_wait(smem_u32(&tq_full[slot]), (k / kTcTQ) & 1);
    const int ti = ok ? *(volatile int *)&tile_q[slot] : -1;
    __syncwarp(mask);
    if (lane == 0 && ok) mbar_arrive(smem_u32(&tq_empty[slot]));
    return ti;
  };

  if (warp == 4) {
    // ---- producer ----
    if (lane == 0) {
      int gc = 0;  // chunks issued by this CTA (all its tiles)
      bool stop = false;
      for (int k = 0; !stop; ++k) {
        // Claim the next tile of the launch (tiles are sorted by decreasing work, so this is
        // longest-first list scheduling: a CTA that starts late simply takes fewer tiles) and
        // publish it to the other roles.
        const int slot = k % kTcTQ;
        if (k >= kTcTQ && !mbar_wait(smem_u32(&tq_empty[slot]), ((k / kTcTQ) - 1) & 1)) {
          fail();
          break;
        }
        int ti = read_flag(&abort_flag) ? n_tiles : atomicAdd(&sched[0], 1);
        if (ti >= n_tiles) ti = -1;
        tile_q[slot] = ti;
        mbar_arrive(smem_u32(&tq_full[slot]));
        if (ti < 0) break;
        const LadderTile tile = tiles[ti];
        const int nchunks = tile.nks + tile.nkh;
        const int rg = (tile.rows + 7) >> 3;  // stored row groups of the A chunks
        const int ng = tile.nb >> 3;          // row groups of a B chunk
        const uint32_t abytes = (uint32_t)rg * kTcGroup * 2, bbytes = (uint32_t)ng * kTcGroup * 2;
        const int64_t vtile = tile.v_base + (int64_t)tile.mt * kTcBM * tile.nkc * kTcKC;
        const int64_t ttile = tile.tmt_base + (int64_t)tile.mt * kTcBM * tile.nkh * kTcKC;
        for (int c = 0; c < nchunks; ++c, ++gc) {
          const int s = gc % S;
          if (read_flag(&abort_flag) ||
              (gc >= S && !mbar_wait(smem_u32(&empty[s]), ((gc / S) - 1) & 1))) {
            fail();
            stop = true;
            break;
          }
          const __nv_bfloat16 *asrc, *bsrc;
          int64_t as, bs;
          if (c < tile.nks) {
            const int kc = tile.kc0 + c;
            asrc = v_tc + vtile + (int64_t)kc * rg * kTcGroup;
            bsrc = tkt_tc + tile.tkt_base + (int64_t)kc * ng * kTcGroup;
            as = v_stride;
            bs = tkt_stride;
          } else {
            const int kh = c - tile.nks;
            asrc = tmt_tc + ttile + (int64_t)kh * rg * kTcGroup;
            bsrc = xt_tc + tile.xt_base + (int64_t)kh * ng * kTcGroup;
            as = tmt_stride;
            bs = xt_stride;
          }
          const uint32_t fb = smem_u32(&full[s]);
          const uint32_t sa = base + s * kStageBytes, sb = sa + NT * kTcAPlane * 2;
          const bool copy_a = !GEN || c >= tile.nks;  // GEN: the generator warps write V
          mbar_expect_tx(fb, NT * ((copy_a ? abytes : 0u) + bbytes));
#pragma unroll
          for (int p = 0; p < NT; ++p) {
            if (copy_a) bulk_g2s(sa + p * kTcAPlane * 2, asrc + p * as, abytes, fb);
            bulk_g2s(sb + p * kTcBPlane * 2, bsrc + p * bs, bbytes, fb);
          }
        }
      }
      issued_chunks = gc;
    }
  } else if (warp == 5) {
    // ---- MMA issuer ----
    if (lane == 0) {
      int gc = 0;
      for (int lt = 0;; ++lt) {
        bool got;
        const int ti = queued(lt, got, 1u);
        if (!got) {
          fail();
          break;
        }
        if (ti < 0) break;
        const LadderTile tile = tiles[ti];
        const int buf = lt & 1, use = lt >> 1;
        if (read_flag(&abort_flag) ||
            (use > 0 && !mbar_wait(smem_u32(&acc_empty[buf]), (use - 1) & 1))) {
          fail();
          break;
        }
        tc_fence_after();
        const uint32_t acc = tmem + buf * kTcAccCols;
        const uint32_t idesc = tc_idesc(tile.nb);
        const int nchunks = tile.nks + tile.nkh;
        bool ok = true;
        for (int c = 0; c < nchunks; ++c, ++gc) {
          const int s = gc % S;
          if (read_flag(&abort_flag) || !mbar_wait(smem_u32(&full[s]), (gc / S) & 1)) {
            fail();
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = base + s * kStageBytes, sb = sa + NT * kTcAPlane * 2;
#pragma unroll
          for (int j = 0; j < kTcKC / 16; ++j) {
#pragma unroll
            for (int pa = 0; pa < NT; ++pa)
#pragma unroll
              for (int pb = 0; pb < NT - pa; ++pb)
                tc_mma(acc, tc_desc(sa + pa * kTcAPlane * 2 + j * 256),
                       tc_desc(sb + pb * kTcBPlane * 2 + j * 256), idesc,
                       (c | j | pa | pb) != 0 ? 1u : 0u);
          }
          tc_commit(smem_u32(&empty[s]));
        }
        tc_commit(smem_u32(&acc_full[buf]));  // also after an abort: the epilogue's wait ends
        if (!ok) break;
      }
      tc_commit(smem_u32(done));
    }
  } else if (GEN && warp >= 6) {
    // ---- V generators: warp gw owns row groups gw, gw + G, ... of each tile; a lane writes
    // row 8 rg + lane / 4, K columns 8 kg + 2 (lane % 4) + {0, 1} of every core matrix (one
    // 32-bit word per plane: conflict-free).  The K columns' codes of the next chunk are
    // loaded while the current one is generated. ----
    using GT = VGenT<NT>;
    const int gw = warp - 6;
    constexpr int RG = (kTcBM / 8) / kTcGenWarps;  // row groups per generator warp
    unsigned char *stage0 = tc_smem_raw + (base - raw);
    int gc = 0;
    bool stop = false;
    for (int k = 0; !stop; ++k) {
      bool got;
      const int ti = queued(k, got, 0xffffffffu);
      if (!got) {
        fail();
        break;
      }
      if (ti < 0) break;
      const LadderTile tile = tiles[ti];
      const int nchunks = tile.nks + tile.nkh;
      const int64_t pk_off = chans[tile.ch].pk_off;
      const int pk = chans[tile.ch].pk;
      VGenRow rw[RG];
#pragma unroll
      for (int i = 0; i < RG; ++i) {
        const int r = 8 * (gw + i * kTcGenWarps) + (lane >> 2);
        // Rows past the tile: zero momenta, so the index stays inside the table (their
        // accumulator rows are never read).
        rw[i] = r < tile.rows ? vg_rows[tile.row_off + (int64_t)tile.mt * kTcBM + r]
                              : VGenRow{kVGenZero, kVGenZero};
      }
      // Column codes of a chunk; K padding (w >= pk) gets weight 0.
      uint32_t cn[8], ck[8];
      auto load_cols = [&](int c, uint32_t *n, uint32_t *k) {
        const int kc = tile.kc0 + c;
#pragma unroll
        for (int j = 0; j < 8; ++j) {  // columns 8 (j / 2) + 2 (lane % 4) + j % 2
          const int w = kc * kTcKC + 8 * (j >> 1) + 2 * (lane & 3) + (j & 1);
          n[j] = w < pk ? vg_cols[pk_off + w] : kVGenZero;
          k[j] = w < pk;
        }
      };
      if (tile.nks > 0) load_cols(0, cn, ck);
      for (int c = 0; c < nchunks; ++c, ++gc) {
        const int s = gc % S;
        uint32_t nn[8], nk[8];
        const bool pre = c + 1 < tile.nks;
        if (pre) load_cols(c + 1, nn, nk);
        if (read_flag(&abort_flag) ||
            (gc >= S && !mbar_wait(smem_u32(&empty[s]), ((gc / S) - 1) & 1))) {
          fail();
          stop = true;
          break;
        }
        if (c < tile.nks) {
          unsigned char *sa = stage0 + s * kStageBytes;
#pragma unroll
          for (int i = 0; i < RG; ++i) {
            const int rg = gw + i * kTcGenWarps;
            if (8 * rg >= tile.rows) continue;
            GT v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = vgen_elem<GT>(rw[i], cn[j], gtab) * (GT)ck[j];
            const uint32_t off =
                (uint32_t)(rg * kTcGroup + (lane >> 2) * 8 + 2 * (lane & 3)) * 2;
#pragma unroll
            for (int p = 0; p < NT; ++p)
#pragma unroll
              for (int kg = 0; kg < 4; ++kg)
                *reinterpret_cast<uint32_t *>(sa + p * kTcAPlane * 2 + off + kg * 128) =
                    vgen_split(v[2 * kg], v[2 * kg + 1]);
          }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&full[s]));
        if (pre) {
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            cn[j] = nn[j];
            ck[j] = nk[j];
          }
        }
      }
    }
  } else {
    // ---- epilogue: accumulator rows -> D (or split-K partials) ----
    const int tid = threadIdx.x;
    for (int lt = 0;; ++lt) {
      bool got;
      const int ti = queued(lt, got, 0xffffffffu);
      if (!consumers_all(got)) {  // one decision for all four warps
        fail();
        break;
      }
      if (ti < 0) break;  // every epilogue thread read the same slot
      const LadderTile tile = tiles[ti];
      const int buf = lt & 1, use = lt >> 1;
      const bool ok = mbar_wait(smem_u32(&acc_full[buf]), use & 1);
      tc_fence_after();
      if (!ok) fail();
      // One decision for all four warps (tcgen05.ld is warp-collective).
      if (!consumers_all(ok && !read_flag(&abort_flag))) break;
      if (tile.nks + tile.nkh > 0) {
        const LadderOut out{tile, rowmap, mirror, d, part};
        const uint32_t lane_addr = tmem + buf * kTcAccCols + ((uint32_t)(warp * 32) << 16);
        for (int c0 = 0; c0 < tile.nb; c0 += 16) {
          float v[16];
          tc_ld16(lane_addr + c0, v);
          double dv[16];
#pragma unroll
          for (int i = 0; i < 16; ++i) dv[i] = (double)v[i];
          out.row<16>(tid, c0, dv);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&acc_empty[buf]));
    }
  }
  tc_fence_before();
  __syncthreads();
  // After an abort, copies the MMA warp never waited for may still be in flight: let them land
  // before the CTA's shared memory is released.
  if (warp == 4 && lane == 0 && read_flag(&abort_flag)) tc_drain(full, issued_chunks, S);
  if (warp == 5) {
    // The MMAs this CTA issued are complete once `done` has fired (it was committed on every
    // path); only then is the accumulator released.
    (void)mbar_wait(smem_u32(done), 0);
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 ::"r"(tmem), "r"(2 * kTcAccCols) : "memory");
  }
  trace_end(ctl, kTrLadderTC);
  // The last CTA to finish resets the tile counter for the next launch (every producer has
  // claimed its last tile by then).
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&sched[1], 1) == (int)gridDim.x - 1) {
      sched[0] = 0;
      sched[1] = 0;
      __threadfence();
    }
  }
}

}  // namespace ccd
