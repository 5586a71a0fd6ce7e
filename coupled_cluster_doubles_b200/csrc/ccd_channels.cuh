// Channel construction on the device: the channel of every ordered orbital pair and the sorted
// channel maps (SPBasis.cpp:80-441, setUpChannelDims / setUpChannelMaps), for
// ccdgpu_build_channels.  The channel order (first-fit-decreasing, one rank) is applied on the
// host between the counting and the placement pass.
//
// A pair (p, q) is of kind 0 pp, 1 hh, 2 hp, 3 ph (p, q particle or hole).  Its code is
// p * n_sp + q, so that sorting codes sorts pairs by (p, q).
#pragma once

#include <cstdint>

#include "ccdgpu.h"

namespace ccd {

struct ChannelRuleDev {
  const int32_t *qn;
  int32_t kind, stride, nmax, chan_tz_max, mod_chan_tz_max;
  uint64_t nsp, np, nch;
};

// Unpermuted regular and modified channel of (p, r) (ElectronGasSPBasis.cpp:572-624,
// InfMatterSPBasis.cpp:458-510, PairingSPBasis.cpp:168-181), with the host builder's
// integer arithmetic.
__device__ __forceinline__ uint64_t chan0_dev(const ChannelRuleDev &r, const int32_t *a,
                                              const int32_t *b) {
  if (r.kind == CCDGPU_MODEL_PAIRING) return (uint64_t)((a[1] + b[1] + 2) / 2);
  const uint64_t n = 4 * (uint64_t)r.nmax + 1, s = 3, t = 2 + r.chan_tz_max / 2;
  uint64_t nx = a[0] + b[0] + n / 2, ny = a[1] + b[1] + n / 2, nz = a[2] + b[2] + n / 2;
  uint64_t sz = (a[3] + b[3] + 2) / 2, tz = (a[4] + b[4] + 2) / 2;
  return nx * n * n * s * t + ny * n * s * t + nz * s * t + sz * t + tz;
}
__device__ __forceinline__ uint64_t mod0_dev(const ChannelRuleDev &r, const int32_t *a,
                                             const int32_t *b) {
  if (r.kind == CCDGPU_MODEL_PAIRING) return (uint64_t)((a[1] - b[1] + 2) / 2);
  const uint64_t n = 4 * (uint64_t)r.nmax + 1, s = 3, t = 1 + r.mod_chan_tz_max;
  uint64_t nx = a[0] - b[0] + n / 2, ny = a[1] - b[1] + n / 2, nz = a[2] - b[2] + n / 2;
  uint64_t sz = (a[3] - b[3] + 2) / 2, tz = (a[4] - b[4] + r.mod_chan_tz_max) / 2;
  return nx * n * n * s * t + ny * n * s * t + nz * s * t + sz * t + tz;
}

__device__ __forceinline__ int pair_kind(uint64_t p, uint64_t q, uint64_t np) {
  return p < np ? (q < np ? 1 : 2) : (q < np ? 3 : 0);
}

// Pass 1: channel of every pair and the count of every (unpermuted channel, kind).
__global__ void pair_channel_kernel(ChannelRuleDev r, uint32_t *__restrict__ c0,
                                    uint32_t *__restrict__ mc0, uint32_t *__restrict__ cnt,
                                    uint32_t *__restrict__ mcnt, int32_t *err) {
  const uint64_t n = r.nsp * r.nsp;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t p = i / r.nsp, q = i - p * r.nsp;
    const int32_t *a = r.qn + p * r.stride, *b = r.qn + q * r.stride;
    const uint64_t c = chan0_dev(r, a, b), mc = mod0_dev(r, a, b);
    if (c >= r.nch || mc >= r.nch) {
      atomicOr(err, 1);
      c0[i] = mc0[i] = 0;
      continue;
    }
    const int k = pair_kind(p, q, r.np);
    c0[i] = (uint32_t)c;
    mc0[i] = (uint32_t)mc;
    atomicAdd(&cnt[c * 4 + k], 1u);
    atomicAdd(&mcnt[mc * 4 + k], 1u);
  }
}

// Pass 2: every pair into its (permuted channel, kind) segment, in arrival order; seg_off[c *
// 4 + k] is the segment's start in `codes` (kinds one after another, channels in permuted
// order inside a kind).  Also the permuted channel of every pair.
__global__ void place_pairs_kernel(uint64_t nsp, uint64_t np, const uint32_t *__restrict__ c0,
                                   const uint32_t *__restrict__ mc0,
                                   const uint32_t *__restrict__ inv,
                                   const uint32_t *__restrict__ seg_off,
                                   const uint32_t *__restrict__ mseg_off,
                                   uint32_t *__restrict__ fill, uint32_t *__restrict__ mfill,
                                   uint32_t *__restrict__ codes, uint32_t *__restrict__ mcodes,
                                   uint32_t *__restrict__ chan, uint32_t *__restrict__ mchan) {
  const uint64_t n = nsp * nsp;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t p = i / nsp, q = i - p * nsp;
    const int k = pair_kind(p, q, np);
    const uint32_t c = inv[c0[i]], mc = inv[mc0[i]];
    codes[seg_off[c * 4 + k] + atomicAdd(&fill[c * 4 + k], 1u)] = (uint32_t)i;
    mcodes[mseg_off[mc * 4 + k] + atomicAdd(&mfill[mc * 4 + k], 1u)] = (uint32_t)i;
    chan[i] = c;
    mchan[i] = mc;
  }
}

// One non-empty segment of `codes`: its start, length and the position array it fills.
struct PairSegment {
  uint32_t off, len, mod, pad;
};
constexpr int kMaxSegment = 8192;  // pairs of one (channel, kind); larger is unsupported

// Pass 3, one CTA per segment: bitonic sort of the codes in shared memory (ascending codes are
// ascending (p, q)), then pos[code] = index inside the segment.
__global__ void __launch_bounds__(512)
sort_segments_kernel(const PairSegment *__restrict__ segs, uint32_t *__restrict__ codes,
                     uint32_t *__restrict__ mcodes, uint32_t *__restrict__ pos,
                     uint32_t *__restrict__ mpos) {
  __shared__ uint32_t key[kMaxSegment];
  const PairSegment sg = segs[blockIdx.x];
  uint32_t *src = (sg.mod ? mcodes : codes) + sg.off;
  uint32_t *out = sg.mod ? mpos : pos;
  const int len = (int)sg.len;
  int n2 = 1;
  while (n2 < len) n2 <<= 1;
  for (int i = threadIdx.x; i < n2; i += blockDim.x) key[i] = i < len ? src[i] : 0xFFFFFFFFu;
  __syncthreads();
  for (int k = 2; k <= n2; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < n2; i += blockDim.x) {
        const int x = i ^ j;
        if (x > i) {
          const uint32_t a = key[i], b = key[x];
          if ((a > b) == ((i & k) == 0)) {
            key[i] = b;
            key[x] = a;
          }
        }
      }
      __syncthreads();
    }
  for (int i = threadIdx.x; i < len; i += blockDim.x) {
    src[i] = key[i];
    out[key[i]] = (uint32_t)i;
  }
}

}  // namespace ccd
