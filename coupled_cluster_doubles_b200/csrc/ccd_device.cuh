// Device-side data structures and small helpers shared by the CCD kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ccd {

// pp-ladder / hh-ladder tiling.  Operand tiles are stored in HBM already in their shared-memory
// image: [rows][kBK] doubles, column index XOR-swizzled by (row & 3) << 2 so that the FP64
// mma.m16n8k4 fragment loads (4 rows x 4 k per half-warp) hit 16 distinct 8-byte bank pairs.
constexpr int kBM = 64;        // rows of D per work tile (4 consumer warps x 16 rows)
constexpr int kBK = 16;        // K depth of one pipeline stage
constexpr int kStages = 6;     // bulk-copy pipeline depth
constexpr int kMaxFrag = 9;    // up to 72 hh columns (8 per n-fragment)
constexpr int kLadderThreads = 160;  // 4 consumer warps + 1 producer warp

__host__ __device__ inline int swz(int row, int k) { return row * kBK + (k ^ ((row & 3) << 2)); }

// One pp-ladder work tile: rows [mt*kBM, mt*kBM+kBM) of channel `ch`'s D block.
struct LadderTile {
  int32_t ch;        // active-channel index
  int32_t mt;        // row tile
  int32_t nkc;       // K chunks over pp (V_pppp x T part)
  int32_t nkh;       // K chunks over hh (T x X part)
  int32_t nfrag;     // n-fragments of 8 columns (ceil(hh/8))
  int32_t pp, hh;
  int32_t pad;
  int64_t v_base;    // V_pppp tiles: + (mt*nkc + kc) * kBM*kBK
  int64_t tkt_base;  // T^T tiles (B operand of V T): + kc * (8*nfrag)*kBK
  int64_t tmt_base;  // T row tiles (A operand of T X): + (mt*nkh + kh) * kBM*kBK
  int64_t xt_base;   // X^T tiles (B operand of T X): + kh * (8*nfrag)*kBK
  int64_t t_off;     // offset of the channel's pp x hh block in the t2 layout
};

// Per active regular channel.
struct ChanInfo {
  int32_t pp, hh, nfrag, nkc, nkh, nmt;
  int64_t t_off;     // pphh block offset (reference t2 layout)
  int64_t pp_off;    // offset into pp_pairs / pp_swap / r
  int64_t hh_off;    // offset into hh_pairs / hh_swap / s
  int64_t x_off;     // hh x hh block offset (V_hhhh and X)
  int64_t tkt_base, tmt_base, xt_base, vkt_base;
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
  double energies[128];  // corrCCD per iteration (first 128)
};

constexpr int32_t kErrNonFinite = 1;
constexpr int32_t kErrTimeout = 2;
constexpr int32_t kErrBadIndex = 4;

}  // namespace ccd
