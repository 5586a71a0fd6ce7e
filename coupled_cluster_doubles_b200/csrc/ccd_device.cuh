// Device-side data structures and small helpers shared by the CCD kernels.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace ccd {

// pp-ladder tiling.  V_pppp is antisymmetric in both pair indices (calcTBME is
// f(p,q,r,s) - f(p,q,s,r)), so D[ab,ij] = 1/2 sum_cd V[ab,cd] T[cd,ij] is evaluated as
// sum_{c<d} V[ab,cd] T[cd,ij] over rows a<=b and mirrored to the b>a rows with a sign flip:
// one quarter of the V bytes and flops of the full product.
//
// Operand tiles are stored in HBM already in their shared-memory image so that one bulk copy
// (TMA) moves a whole stage:
//   thin channels (hh <= 8, nb in {2, 4, 8}, one row per consumer thread):
//     A tiles [rows][kBK] row-major, column XOR-swizzled by (row & 15): a warp reading 16
//             consecutive rows at one k hits 16 distinct bank pairs;
//     B tiles [kBK][nb] k-major, read as warp broadcasts;
//   mid and wide channels (nb = 8*C, FP64 MMA fragments):
//     A tiles [kBK][as] k-major, as = rows rounded up to 8, plus 4;
//     B tiles [kBK][bs] k-major, bs = nb + 4;
//     strides of 4 mod 8 doubles put the 4 k-rows of an FP64 MMA fragment load (m16n8k16 in
//     the ladder) on distinct banks.
// The last row tile of a channel is stored compact (only its real rows, rounded up to 8).
constexpr int kBK = 16;        // K depth of one pipeline stage
constexpr int kStages = 4;     // bulk-copy pipeline depth
constexpr int kMaxCG = 9;      // column groups of 8 -> up to 72 hh columns
constexpr int kLadderConsumers = 128;
constexpr int kLadderThreads = kLadderConsumers + 32;  // + 1 producer warp
// Mid and wide classes: 8 consumer warps of 16 rows each (two CTAs per SM).
constexpr int kLadderConsumersMMA = 256;
__host__ __device__ constexpr int ladder_threads(int cls) {
  return (cls == 0 ? kLadderConsumers : kLadderConsumersMMA) + 32;
}
constexpr int kMaxBM = 128;
constexpr int kMaxNB = 8 * kMaxCG;
constexpr int kMaxAS = kMaxBM + 4;  // A stage row stride bound (doubles)
constexpr int kMaxBS = kMaxNB + 4;  // B stage row stride bound (doubles)

__host__ __device__ inline int swzA(int row, int k) { return row * kBK + (k ^ (row & 15)); }
// Padded column count of a channel with hh hole pairs.
__host__ __device__ inline int ladder_nb(int hh) {
  return hh <= 2 ? 2 : hh <= 4 ? 4 : 8 * ((hh + 7) / 8);
}
// Rows per tile: thin channels one row per consumer thread; mid and wide ones (nb >= 16)
// 16 rows x nb columns per consumer warp.
__host__ __device__ inline int ladder_bm(int nb) { return kLadderConsumers; }
// A chunks of mid and wide channels are k-major (row stride `arows`, see above); thin ones are
// row-major and XOR-swizzled (one row per thread).
__host__ __device__ inline bool ladder_kmajor(int nb) { return nb >= 16; }
// A row stride (doubles per k row of an A chunk) of a row tile with `rows` real rows.
__host__ __device__ inline int ladder_arows(int nb, int rows) {
  return ladder_kmajor(nb) ? ((rows + 7) & ~7) + 4 : rows;
}
// A image of row tile mt starts at mt * ladder_arows(nb, kMaxBM) * nk * kBK (full tiles).
__host__ __device__ inline int ladder_arows_full(int nb) { return ladder_arows(nb, kMaxBM); }
// B row stride (doubles per k row of a B chunk).
__host__ __device__ inline int ladder_bs(int nb) { return ladder_kmajor(nb) ? nb + 4 : nb; }
__host__ __device__ inline int ladder_aoff(int nb, int arows, int r, int k) {
  return ladder_kmajor(nb) ? k * arows + r : swzA(r, k);
}

// Mixed-precision pp-ladder images (tensor-core operands, ccd_tc.cuh).  A K chunk of a
// 128-row tile holds kTcKC bf16 per row in 8 x 8 core matrices, K-major, no swizzle:
//   element (r, k) -> (r / 8) * kTcGroup + (k / 8) * 64 + (r % 8) * 8 + k % 8.
constexpr int kTcKC = 32;                    // K depth of one chunk (bf16 elements)
constexpr int kTcBM = 128;                   // rows per tile = UMMA M
constexpr int kTcMaxNB = 80;                 // padded columns = UMMA N (multiple of 16)
constexpr int kTcThreads = 192;
constexpr int kTcAPlane = kTcBM * kTcKC;     // bf16 elements of one A term per stage (8 KB)
constexpr int kTcBPlane = kTcMaxNB * kTcKC;  // one B term per stage (5 KB)
constexpr int kTcGroup = 8 * kTcKC;          // bf16 elements of one 8-row group of a chunk

// Padded UMMA N for hh columns.
__host__ __device__ inline int tc_nb(int hh) { return 16 * ((hh + 15) / 16); }
// Offset of element (r, k) inside a chunk image (bf16 units), 0 <= k < kTcKC: K-major core
// matrices (8 rows of 8 consecutive k), used for the A operands.
__host__ __device__ inline int tc_off(int r, int k) {
  return (r >> 3) * kTcGroup + (k >> 3) * 64 + (r & 7) * 8 + (k & 7);
}
// The B operands (N = hh columns) in MN-major core matrices (8 k-rows of 8 consecutive n):
// neighbouring columns are neighbouring bytes, as the assembly and hh ladder write them.  Same
// 8 x 8 block positions as tc_off, so the shared-memory descriptors are the same.
__host__ __device__ inline int tc_off_mn(int n, int k) {
  return (n >> 3) * kTcGroup + (k >> 3) * 64 + (k & 7) * 8 + (n & 7);
}
// x -> nt bf16 terms, each the round-to-nearest of what the previous ones leave (the
// remainders are exact in double).
// bf16 bits of a double h that has at most 8 significant bits: sign, exponent rebased from
// 1023 to 127, top 7 mantissa bits.  Zero and magnitudes below bf16's normal range (2^-126)
// give a signed zero; NaN stays NaN.
__device__ __forceinline__ __nv_bfloat16 bf16_of_short(double h) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(h);
  const unsigned short sign = (unsigned short)((b >> 48) & 0x8000u);
  const int e = (int)((b >> 52) & 0x7FF) - 1023 + 127;
  unsigned short bits;
  if (e <= 0) bits = sign;
  else if (e >= 255) bits = (unsigned short)(sign | 0x7F80u | ((b << 12) ? 0x40u : 0u));
  else bits = (unsigned short)(sign | (e << 7) | (unsigned)((b >> 45) & 0x7F));
  return __ushort_as_bfloat16(bits);
}

// x = t_0 + t_1 (+ t_2) + remainder, each t_p a bf16 (nt terms): t_p is the remainder rounded
// to 8 significant bits by Dekker's splitting (Dekker 1971: c = r (2^45 + 1), t = c - (c - r)),
// which is exact in bf16, and the next remainder r - t_p is exact in FP64.  Only FP64 and
// integer arithmetic, no conversion instructions.
__device__ __forceinline__ double split_bf16_step(double &x) {
  // Explicitly rounded operations: an FMA contraction of c - x would skip the rounding of c
  // that the splitting relies on.
  const double c = __dmul_rn(x, 35184372088833.0);  // 2^45 + 1
  double hi = __dsub_rn(c, __dsub_rn(c, x));
  if (fabs(hi) < 1.1754943508222875e-38) hi = 0.0;  // below bf16's normal range
  x = __dsub_rn(x, hi);
  return hi;
}
__device__ __forceinline__ void split_bf16(double x, __nv_bfloat16 *out, int nt) {
  for (int p = 0; p < nt; ++p) out[p] = bf16_of_short(split_bf16_step(x));
}
// The same with the term count known at compile time (the terms stay in registers).
template <int NT>
__device__ __forceinline__ void split_bf16_n(double x, __nv_bfloat16 (&out)[NT]) {
#pragma unroll
  for (int p = 0; p < NT; ++p) out[p] = bf16_of_short(split_bf16_step(x));
}

// One pp-ladder work tile: packed rows [mt*bm, mt*bm+rows) of channel `ch`, V-part K chunks
// [kc0, kc0+nks).  Tiles of one row block that split K write partial sums; the last one to
// finish (ticket on counter `group`) adds them in segment order.  The segment with seg ==
// nseg-1 also runs the T X chunks.
struct LadderTile {
  int32_t ch, mt, kc0, nks, nkc, nkh, nb, bm, rows, pr, hh, seg, nseg, group;
  int64_t v_base;    // A tiles of V:  + mt*arows_full*nkc*kBK + kc * arows*kBK
  int64_t tkt_base;  // B tiles of T:  + kc * kBK*bs
  int64_t tmt_base;  // A tiles of T (rows a<=b, K = hh): + mt*bm*nkh*kBK + kh * rows*kBK
  int64_t xt_base;   // B tiles of X/2: + kh * kBK*bs
  int64_t t_off;     // offset of the channel's pp x hh block in the t2 layout
  int64_t row_off;   // offset into rowmap / mirror
  int64_t part_base; // partial sums of this row block: nseg * bm * nb doubles
};

// Per active regular channel.
struct ChanInfo {
  int32_t pp, hh, nb, nkc, nkh, nmt, bm, pr, pk, nhht;
  int64_t t_off;     // pphh block offset (reference t2 layout)
  int64_t pp_off;    // offset into pp_pairs / pp_swap / pk_idx / r
  int64_t hh_off;    // offset into hh_pairs / hh_swap / s
  int64_t x_off;     // hh x hh block offset (V_hhhh and X)
  int64_t tkt_base, tmt_base, xt_base, vkt_base;
  int64_t row_off;   // offset into rowmap / mirror (pr entries)
  int64_t pk_off;    // offset into kcol (pk entries)
  int64_t part_off;  // hh-ladder partial products: nhht * hh*hh doubles
  int64_t hht0;      // first hh-ladder tile of the channel
  // Mixed-precision operand images (bf16 terms, tensor-core layout; see ccd_tc.cuh):
  // nbt = UMMA N, nkct / nkht = 32-deep K chunks of V T / T X.
  int32_t nbt, nkct, nkht, pad_tc;
  int64_t vtc_base, tkt_tc_base, tmt_tc_base, xt_tc_base;
  // Fused assembly: hk = strict hole pairs (i < j); quad tables from qrow_off (pk strict
  // packed rows a < b) and qcol_off (hk entries).
  int32_t hk, pad_q;
  int64_t qrow_off, qcol_off;
};

// hh-ladder unit: rows [k0, k0+rows) of channel ch (slice idx), a chunk of P rows.
struct HHTile {
  int32_t ch, k0, idx, rows, chunk, pad;
};

// Fused assembly, static data of strict packed row u (a < b) of a channel (index
// qrow_off + u): offsets of rows ab and ba inside the channel block (ab * hh, ba * hh), the
// operand-image indices of row ab (pk_idx: K index, packed row), particle indices a - np,
// b - np, and e_a, e_b ...
struct QuadRow {
  int32_t o_ab, o_ba;
  int32_t qx, qy;
  int32_t pa, pb;
  double ea, eb;
};
// ... and of strict hole pair w (i < j, index qcol_off + w): the columns ij and ji, the hole
// indices i, j and e_i + e_j.
struct QuadCol {
  int32_t c_ij, c_ji, i, j;
  double eij;
};
// Work item of the fused assembly: quads [q0, q1) (q = u * hk + w) of active channel ch, with
// the channel's hk, block offset and table offsets (so a thread's table reads depend on the
// item alone).
struct QuadItem {
  int32_t ch, q0, q1, hk;
  int64_t t_off, qrow_off, qcol_off;
};

// Per active modified channel.
struct ModInfo {
  int32_t ph, hp;
  int64_t m_off;     // ph' x hp' block offset in the phhp slab (V_hpph uses the same size)
  int64_t y_off;     // hp' x hp' block offset (V_hphp)
};

// Contiguous element range [e0, e1) of one channel for the element-wise kernels.
struct ElemRange {
  int32_t ch;
  int32_t pad;
  int64_t e0, e1;
};

// Kernel ids of the start-time trace (Control::trace_*).
enum TraceKernel {
  kTrRingSmall = 0, kTrRingMid, kTrRingLarge, kTrHHSmall, kTrHHTiled, kTrOneBody, kTrLadderThin,
  kTrLadderMid, kTrLadderWide, kTrLadderTC, kTrAssemble, kTrLoopCtl, kTrEnergy, kTrRetile,
  kTrReduce, kTrHHReduce, kTrGather, kTraceKernels
};

// Device control block: iteration state of the solve loop lives on the device so that a
// captured iteration can be replayed without host round trips.
struct Control {
  double e_prev;         // corrEnergyPrev (starts at 100, main.cpp:494)
  double e_corr;         // corrCCD of the last iteration
  double e_diff;         // energyDiff
  double tol;
  double mixing;
  int64_t iterations;    // iterations performed
  int64_t max_iters;
  int32_t done;          // set when |dE| <= tol or the cap is reached; kernels then no-op
  int32_t parity;        // which t2 buffer holds the current amplitudes
  int32_t error;         // bit flags, see kErr*
  int32_t active;        // 1 while a solve is running (0: kernels run unconditionally)
  int32_t phase;         // mixed-precision solve: 1 = split-bf16 ladder, 2 = FP64 polish
  int32_t retile;        // the FP64 ladder operand tiles are stale (a mixed iteration ran)
  int32_t inject;        // test-only fault: 1 = the first FP64 pp-ladder CTA of each class
                         // withholds its first stage (its bounded waits run out)
  int32_t pad0;
  double polish_rel;     // phase 1 -> 2 once |dE| <= max(tol, polish_rel * |E|)
  int64_t polish_iters;  // iterations run in phase 2
  int64_t stop_at;       // device solve loop: one graph launch runs while iterations < stop_at
  int64_t trace_iter;    // kernel trace: the iteration whose kernels record start times
  uint64_t trace_first[kTraceKernels];  // %globaltimer of the first / last CTA start
  uint64_t trace_last[kTraceKernels];
  uint64_t trace_end[kTraceKernels];    // %globaltimer when the last CTA finished
  double energies[128];  // corrCCD per iteration (first 128)
};

constexpr int32_t kErrNonFinite = 1;
constexpr int32_t kErrTimeout = 2;
constexpr int32_t kErrBadIndex = 4;
constexpr int32_t kErrRingMaps = 8;  // aj_ib / bi_ja / bj_ia are not ai_jb under the swaps

}  // namespace ccd
