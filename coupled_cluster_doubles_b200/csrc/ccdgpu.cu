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
#include <atomic>
#include <queue>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "ccd_channels.cuh"
#include "ccd_device.cuh"
#include "ccd_kernels.cuh"
#include "ccd_setup.cuh"
#include "ccd_tc.cuh"
#include "ccdgpu.h"
#include "host/channel_order.h"

using namespace ccd;

namespace {

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

}  // namespace

// A handle's streams and events (see the pool below).
struct StreamSet {
  int dev = -1;
  cudaStream_t s[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t ev[16] = {};
};

struct ccdgpu_handle {
  ccdgpu_options opt{};
  StreamSet sset;  // the streams and events below, from the process-wide pool
  cudaStream_t s0 = nullptr, s1 = nullptr, s2 = nullptr, s3 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_fork2 = nullptr, ev_join2 = nullptr;
  cudaEvent_t ev_fork3 = nullptr, ev_join3 = nullptr;  // one-body sums beside the pp ladder
  cudaEvent_t ev[10] = {};
  uint64_t nch = 0, nsp = 0, np = 0, npart = 0;
  int64_t n_t = 0, n_m = 0, n_h = 0, n_p = 0;
  int n_hh_small = 0;  // hh-ladder units of channels with hh <= 16 (first in hh_tiles)
  size_t hh_slice_smem = 0;  // dynamic shared memory of hh_slice_kernel (largest hh > 16)
  int n_hh_red = 0;    // hh-ladder reduction items
  int n_act = 0, n_mod = 0, n_mod_small = 0, n_mod_mid = 0, n_tiles = 0, n_hh_tiles = 0;
  int n_ranges = 0;
  int n_asm_blocks = 0;  // fused assembly CTAs (persistent, striding over quad_items)
  int n_cls[3] = {0, 0, 0};  // pp-ladder tiles per column class (thin, mid, wide), in that order
  size_t ladder_smem_thin = 0;
  size_t ladder_smem = 0, hh_smem = 0;
  int n_mod_pad[4] = {0, 0, 0, 0};  // ring channels by padded size 32, 48, 64, 80 (after small)
  bool have_3body = false;
  std::vector<DevBuf> allocs;

  ChanInfo *chans = nullptr;
  ModInfo *mods = nullptr;        // small (n_mod_small), then by padded size 32 .. 80
  LadderTile *tiles = nullptr;
  HHTile *hh_tiles = nullptr;
  HHRed *hh_red = nullptr;
  int32_t *rowmap = nullptr, *mirror = nullptr;
  int2 *pk_idx = nullptr;
  double *part = nullptr, *lpart = nullptr;
  ElemRange *ranges = nullptr;
  QuadItem *quad_items = nullptr;  // fused assembly: work items of quads (u, w)
  QuadRow *quad_rows = nullptr;    // fused assembly: per strict packed row / hole pair tables
  int64_t n_quad_rows = 0;
  QuadCol *quad_cols = nullptr;
  int n_quad_items = 0;
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
  int32_t *inv4 = nullptr;   // phhp position -> pphh element (inverse of the ai_jb table)
  double create_ms[5] = {};   // ccdgpu_profile::ms_create
  double loop_graph_ms = 0;   // ccdgpu_profile::ms_loop_graph
  double *d_ring = nullptr;  // fused path: ring result R in pphh order
  int64_t *o_h = nullptr, *o_p = nullptr;
  double *v_h_hpp = nullptr, *v_phh_p = nullptr;
  double *old_h1pp_h2 = nullptr, *old_h2pp_h1 = nullptr, *diff_h2pp_h1 = nullptr;
  double *old_p1_p2hh = nullptr, *old_p2_p1hh = nullptr, *diff_p2_p1hh = nullptr;
  double *gath = nullptr;
  Control *ctl = nullptr;
  Control *h_ctl = nullptr;  // pinned mirror
  int32_t *ticket = nullptr;  // assembly's last-CTA ticket
  double *e_out = nullptr;
  int32_t *err = nullptr;
  // The interaction model on the device (present when the problem carries one), and the
  // buffer of ccdgpu_reference_energy: n_sp bare energies in, n_sp normal-ordered + E_ref out.
  ModelDev md{};
  bool has_model = false;
  double *eps_io = nullptr;

  cudaGraphExec_t graph = nullptr;
  int64_t kernels_per_graph = 0;
  bool profiling = false;
  bool inject_next_step = false;  // ccdgpu_inject_wait_timeout armed for the next step
  ccdgpu_profile prof{};
  double flops = 0, v_bytes = 0, v_packed_bytes = 0, ladder_flops = 0, ladder_bytes = 0;
  int64_t n_tkt = 0, n_tmt = 0;
  int64_t launches = 0;

  // pp-ladder work lists (make_ladder_tiles), in their own allocation so the autotuner can
  // rebuild them.
  std::vector<ChanInfo> host_chans;
  std::vector<ModInfo> host_mods;
  int64_t n_list = 0;  // entries of the one-body segment lists
  ccdgpu_schedule schedule{};
  void *tile_mem = nullptr;
  size_t tile_bytes = 0;
  RedItem *red_fp = nullptr, *red_tc = nullptr;  // split-K reduction items
  int32_t *tc_sched = nullptr;  // tensor-core ladder: tile counter, exit ticket (zero between launches)
  int tc_grid = 0;
  int32_t *fp_cta_off = nullptr;  // FP64 ladder classes: tile ranges of their persistent CTAs
  int fp_grid[3] = {0, 0, 0}, fp_off_base[3] = {0, 0, 0};
  int n_red_fp = 0, n_red_tc = 0, n_red_cls[3] = {0, 0, 0};

  // Mixed precision (nt bf16 terms per operand; 0 for an FP64 handle).
  int nt = 0;
  int n_tc_tiles = 0;
  LadderTile *tc_tiles = nullptr;
  int32_t *kcol = nullptr;  // pp index of the w-th c<d pair of each channel (pk_off + w)
  double *tc_part = nullptr;
  __nv_bfloat16 *v_tc = nullptr, *tkt_tc = nullptr, *tmt_tc = nullptr, *xt_tc = nullptr;
  // Electron gas with V generated on the device: the tensor-core ladder generates its V
  // planes itself (no v_tc images) from these per-row / per-K-column codes and the q^2 table.
  bool tc_gen = false;
  VGenRow *vg_rows = nullptr;
  uint32_t *vg_cols = nullptr;
  double *vg_tab = nullptr;
  int64_t n_vtc = 0, n_tkttc = 0, n_tmttc = 0, n_xttc = 0;  // plane strides (elements)
  size_t tc_smem = 0;
  double ladder_bytes_tc = 0;
  cudaGraphExec_t graph_tc = nullptr;
  int64_t kernels_per_graph_tc = 0;

  // Device solve loop: graphs of WHILE conditional nodes whose bodies are one iteration each
  // (loop64: FP64 iterations; loop_tc: mixed iterations, then FP64 ones).  loop_state: 0 not
  // built yet, 1 built, -1 unavailable (the batched graph replay is used instead).  A mixed
  // handle builds loop_tc first and loop64 only when a launch needs it (a solve still in FP64
  // iterations after a whole loop chunk); loop_pdl: the capture that worked used PDL launches.
  cudaGraphExec_t loop64 = nullptr, loop_tc = nullptr;
  int loop_state = 0;
  bool loop_pdl = true;
  int loop_capture = 0;  // while capturing a loop body: 1 FP64 body, 2 mixed body
  cudaGraphConditionalHandle loop_cond = 0;
  int64_t kernels_per_body64 = 0, kernels_per_body_tc = 0;
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

// Swap partner of every pair of a channel map sorted by (p, q): sw[k] = index of (q_k, p_k),
// -1 if absent.  One pass records where each first index's run starts (row[p], stamped with
// the channel so that the array is never cleared), then each partner is found by a scan of
// its run (a channel holds few pairs per first index), O(n) instead of n binary searches
// whose unpredictable branches dominated create on the largest bases.
struct SwapIndex {
  std::vector<int32_t> row;
  std::vector<uint32_t> stamp;
  uint32_t cur = 0;
  explicit SwapIndex(size_t nsp) : row(nsp, 0), stamp(nsp, 0) {}
  bool build(const ccdgpu_pair *m, int64_t n, int32_t *sw) {
    ++cur;
    for (int64_t k = 0; k < n; k++)
      if (k == 0 || m[k].p != m[k - 1].p) {
        if (m[k].p >= row.size()) return false;
        row[m[k].p] = (int32_t)k;
        stamp[m[k].p] = cur;
      }
    for (int64_t k = 0; k < n; k++) {
      const uint64_t a = m[k].p, b = m[k].q;
      sw[k] = -1;
      if (b >= row.size() || stamp[b] != cur) continue;
      for (int64_t j = row[b]; j < n && m[j].p == b && m[j].q <= a; j++)
        if (m[j].q == a) { sw[k] = (int32_t)j; break; }
    }
    return true;
  }
};

// Process-wide cache of device blocks given back by destroyed handles, by create's scratch
// and by schedule changes, reused by later allocations on the same device instead of
// cudaMalloc / cudaFree (hundreds of microseconds each; cudaFree also waits for the whole
// device).  Holds at most kCacheMax bytes; ccdgpu_release_cached_memory returns them.
constexpr size_t kCacheMax = size_t(16) << 30;

struct CachedBlock {
  int dev;
  void *p;
  size_t bytes;
};

struct BlockCache {
  std::mutex mu;
  std::vector<CachedBlock> blocks;
  size_t total = 0;
};

BlockCache &block_cache() {
  static BlockCache c;
  return c;
}

// Frees the cached blocks of device `dev` (all devices for dev < 0).
void release_cache(int dev) {
  BlockCache &C = block_cache();
  std::vector<CachedBlock> drop;
  {
    std::lock_guard<std::mutex> lock(C.mu);
    std::vector<CachedBlock> keep;
    for (const CachedBlock &b : C.blocks) (dev < 0 || b.dev == dev ? drop : keep).push_back(b);
    C.blocks.swap(keep);
    for (const CachedBlock &b : drop) C.total -= b.bytes;
  }
  int cur = 0;
  if (cudaGetDevice(&cur) != cudaSuccess) cur = -1;
  for (const CachedBlock &b : drop) {
    cudaSetDevice(b.dev);
    cudaFree(b.p);
  }
  if (cur >= 0) cudaSetDevice(cur);
  (void)cudaGetLastError();
}

// A block of at least `bytes` on the current device: the smallest cached one that is at most
// twice as large (plus 64 MiB), else a new allocation, retried once after this device's cache
// has been freed.  *got receives the block's size.
cudaError_t dev_alloc(size_t bytes, void **p, size_t *got) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  BlockCache &C = block_cache();
  {
    std::lock_guard<std::mutex> lock(C.mu);
    int best = -1;
    for (int i = 0; i < (int)C.blocks.size(); i++) {
      const CachedBlock &b = C.blocks[i];
      if (b.dev == dev && b.bytes >= bytes && b.bytes <= 2 * bytes + (size_t(64) << 20) &&
          (best < 0 || b.bytes < C.blocks[best].bytes))
        best = i;
    }
    if (best >= 0) {
      *p = C.blocks[best].p;
      *got = C.blocks[best].bytes;
      C.total -= *got;
      C.blocks.erase(C.blocks.begin() + best);
      return cudaSuccess;
    }
  }
  e = cudaMalloc(p, bytes);
  if (e == cudaErrorMemoryAllocation) {
    (void)cudaGetLastError();
    release_cache(dev);
    e = cudaMalloc(p, bytes);
  }
  *got = bytes;
  return e;
}

// Gives a block back (to the cache while it has room).  The caller has waited for every use.
void dev_free(void *p, size_t bytes) {
  if (!p) return;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) {
    BlockCache &C = block_cache();
    std::lock_guard<std::mutex> lock(C.mu);
    if (C.total + bytes <= kCacheMax) {
      C.blocks.push_back({dev, p, bytes});
      C.total += bytes;
      return;
    }
  }
  cudaFree(p);
}

// Page-locked Control mirrors, handed out from slabs of 64 that live for the process:
// cudaMallocHost / cudaFreeHost per handle cost more than a small create's own work.
struct CtlPool {
  std::mutex mu;
  std::vector<Control *> free;
};

CtlPool &ctl_pool() {
  static CtlPool p;
  return p;
}

Control *ctl_acquire() {
  CtlPool &pool = ctl_pool();
  std::lock_guard<std::mutex> lock(pool.mu);
  if (pool.free.empty()) {
    Control *slab = nullptr;
    if (cudaMallocHost(reinterpret_cast<void **>(&slab), 64 * sizeof(Control)) != cudaSuccess) {
      (void)cudaGetLastError();
      return nullptr;
    }
    for (int i = 63; i >= 0; i--) pool.free.push_back(slab + i);
  }
  Control *c = pool.free.back();
  pool.free.pop_back();
  std::memset(c, 0, sizeof(Control));
  return c;
}

void ctl_release(Control *c) {
  CtlPool &pool = ctl_pool();
  std::lock_guard<std::mutex> lock(pool.mu);
  pool.free.push_back(c);
}

// Process-wide pool of the streams and events a handle uses (four streams, sixteen events per
// set), by device: a create takes a set that a destroyed handle gave back instead of creating
// twenty objects, and a destroy returns its set (after its streams are idle) instead of
// destroying them.  Emptied by ccdgpu_release_cached_memory.
struct StreamPool {
  std::mutex mu;
  std::vector<StreamSet> sets;
};
StreamPool &stream_pool() {
  static StreamPool p;
  return p;
}
void destroy_set(StreamSet &ss) {
  for (cudaEvent_t &e : ss.ev)
    if (e) cudaEventDestroy(e);
  for (cudaStream_t &st : ss.s)
    if (st) cudaStreamDestroy(st);
}
// A set for the current device: from the pool, else new (events 0-9 time, the rest only order).
cudaError_t acquire_set(StreamSet &ss) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  {
    StreamPool &P = stream_pool();
    std::lock_guard<std::mutex> lock(P.mu);
    for (size_t i = 0; i < P.sets.size(); i++)
      if (P.sets[i].dev == dev) {
        ss = P.sets[i];
        P.sets.erase(P.sets.begin() + i);
        return cudaSuccess;
      }
  }
  ss.dev = dev;
  for (int k = 0; k < 4 && e == cudaSuccess; k++)
    e = cudaStreamCreateWithFlags(&ss.s[k], cudaStreamNonBlocking);
  for (int k = 0; k < 16 && e == cudaSuccess; k++)
    e = k < 10 ? cudaEventCreate(&ss.ev[k]) : cudaEventCreateWithFlags(&ss.ev[k], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    destroy_set(ss);
    ss = StreamSet{};
  }
  return e;
}
void release_set(StreamSet &ss) {
  if (ss.dev < 0) return;
  StreamPool &P = stream_pool();
  std::lock_guard<std::mutex> lock(P.mu);
  P.sets.push_back(ss);
  ss = StreamSet{};
}
void release_stream_pool() {
  std::vector<StreamSet> drop;
  {
    StreamPool &P = stream_pool();
    std::lock_guard<std::mutex> lock(P.mu);
    drop.swap(P.sets);
  }
  int cur = 0;
  if (cudaGetDevice(&cur) != cudaSuccess) cur = -1;
  for (StreamSet &ss : drop) {
    cudaSetDevice(ss.dev);
    destroy_set(ss);
  }
  if (cur >= 0) cudaSetDevice(cur);
  (void)cudaGetLastError();
}

void release(ccdgpu_handle *h) {
  if (!h) return;
  // Cached blocks are handed to other handles: nothing of this one may still run on them.
  for (cudaStream_t st : {h->s0, h->s1, h->s2, h->s3})
    if (st) cudaStreamSynchronize(st);
  for (cudaGraphExec_t g : {h->graph, h->graph_tc, h->loop64, h->loop_tc})
    if (g) cudaGraphExecDestroy(g);
  h->graph = h->graph_tc = h->loop64 = h->loop_tc = nullptr;
  for (auto &b : h->allocs) dev_free(b.p, b.bytes);
  h->allocs.clear();
  dev_free(h->tile_mem, h->tile_bytes);
  h->tile_mem = nullptr;
  if (h->h_ctl) ctl_release(h->h_ctl);
  h->h_ctl = nullptr;
  // The streams are idle (synchronised above): their set goes back to the pool.
  if (cudaGetLastError() == cudaSuccess) release_set(h->sset);
  else destroy_set(h->sset);
}

// Bump allocator over one device allocation (256-byte aligned pieces), zero-filled on s0 at
// commit, except the pieces added with add_unset, which follow the others and which the
// caller writes in full before anything reads them.
struct Arena {
  size_t used = 0, unset = 0;
  std::vector<std::pair<void **, size_t>> reqs, unset_reqs;
  static size_t piece(size_t bytes) { return (std::max<size_t>(bytes, 1) + 255) & ~size_t(255); }
  template <typename T>
  void add(T **p, size_t count) {
    reqs.push_back({reinterpret_cast<void **>(p), used});
    used += piece(count * sizeof(T));
  }
  template <typename T>
  void add_unset(T **p, size_t count) {
    unset_reqs.push_back({reinterpret_cast<void **>(p), unset});
    unset += piece(count * sizeof(T));
  }
  int commit(ccdgpu_handle *h) {
    void *base = nullptr;
    size_t got = 0;
    CK(dev_alloc(used + unset, &base, &got));
    h->allocs.push_back({base, got});
    CK(cudaMemsetAsync(base, 0, used, h->s0));
    for (auto &r : reqs) *r.first = static_cast<char *>(base) + r.second;
    for (auto &r : unset_reqs) *r.first = static_cast<char *>(base) + used + r.second;
    return CCDGPU_OK;
  }
};

// Process-wide pinned staging for large host -> device uploads: two page-locked buffers of
// kStageChunk bytes, allocated on first use and kept until the process exits.  A copy from
// pageable memory is bounced by the driver through small internal buffers at a fraction of
// the link bandwidth; here host threads fill one pinned buffer while the copy engine drains
// the other.  Creates on other threads that find the buffers busy copy directly.
constexpr size_t kStageChunk = size_t(16) << 20;
constexpr size_t kStageMin = size_t(1) << 20;  // smaller copies go direct

struct Staging {
  std::mutex mu;
  char *buf = nullptr;  // 2 * kStageChunk, cudaHostAllocPortable
  bool failed = false;
};

Staging &staging() {
  static Staging s;
  return s;
}

// Host runs (src[i], bytes[i]) to consecutive device bytes from dst.  Large totals go through
// the staging buffers: each chunk is filled by host threads from pieces of the runs (a run may
// span chunks, a chunk may hold many runs) and moved by one device copy.
int copy_runs_to_device(ccdgpu_handle *h, char *dst, const std::vector<const char *> &src,
                        const std::vector<size_t> &bytes) {
  size_t total = 0;
  std::vector<size_t> at(src.size());
  for (size_t i = 0; i < src.size(); i++) {
    at[i] = total;
    total += bytes[i];
  }
  if (!total) return CCDGPU_OK;
  Staging &S = staging();
  std::unique_lock<std::mutex> lock(S.mu, std::defer_lock);
  if (total >= kStageMin && lock.try_lock()) {
    if (!S.buf && !S.failed &&
        cudaHostAlloc(reinterpret_cast<void **>(&S.buf), 2 * kStageChunk,
                      cudaHostAllocPortable) != cudaSuccess) {
      (void)cudaGetLastError();
      S.buf = nullptr;
      S.failed = true;
    }
    if (S.buf) {
      cudaEvent_t ev[2] = {nullptr, nullptr};
      bool pending[2] = {false, false};
      cudaError_t e = cudaSuccess;
      for (int k = 0; k < 2 && e == cudaSuccess; k++)
        e = cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming);
      const int threads = std::max(1, std::min(omp_get_max_threads(), 16));
      size_t r0 = 0;  // first run that reaches into the current chunk
      struct Piece {
        size_t to;
        const char *from;
        size_t n;
      };
      std::vector<Piece> pieces;
      for (size_t off = 0, k = 0; off < total && e == cudaSuccess; off += kStageChunk, k ^= 1) {
        const size_t n = std::min(kStageChunk, total - off), end = off + n;
        char *stage = S.buf + k * kStageChunk;
        if (pending[k] && (e = cudaEventSynchronize(ev[k])) != cudaSuccess) break;
        // Pieces of at most n / threads bytes, so that one large run is copied in parallel too.
        const size_t piece = std::max<size_t>(size_t(64) << 10, (n + threads - 1) / threads);
        pieces.clear();
        while (at[r0] + bytes[r0] <= off) r0++;
        for (size_t i = r0; i < src.size() && at[i] < end; i++) {
          const size_t lo = std::max(at[i], off), hi = std::min(at[i] + bytes[i], end);
          for (size_t x = lo; x < hi; x += piece)
            pieces.push_back(Piece{x - off, src[i] + (x - at[i]), std::min(piece, hi - x)});
        }
#pragma omp parallel for num_threads(threads) schedule(dynamic, 8)
        for (int64_t j = 0; j < (int64_t)pieces.size(); j++)
          std::memcpy(stage + pieces[j].to, pieces[j].from, pieces[j].n);
        e = cudaMemcpyAsync(dst + off, stage, n, cudaMemcpyHostToDevice, h->s0);
        if (e == cudaSuccess) e = cudaEventRecord(ev[k], h->s0);
        pending[k] = e == cudaSuccess;
      }
      // The buffers are free for the next upload only once their copies have completed.
      for (int k = 0; k < 2; k++) {
        if (pending[k]) {
          const cudaError_t w = cudaEventSynchronize(ev[k]);
          if (e == cudaSuccess) e = w;
        }
        if (ev[k]) cudaEventDestroy(ev[k]);
      }
      if (e != cudaSuccess) {
        (void)cudaStreamSynchronize(h->s0);
        (void)cudaGetLastError();
        return e == cudaErrorMemoryAllocation ? CCDGPU_ERR_OUT_OF_MEMORY : CCDGPU_ERR_CUDA;
      }
      return CCDGPU_OK;
    }
  }
  for (size_t i = 0; i < src.size(); i++)
    if (bytes[i]) CK(cudaMemcpyAsync(dst + at[i], src[i], bytes[i], cudaMemcpyHostToDevice, h->s0));
  return CCDGPU_OK;
}

// Device bytes [src, src + total) to host memory dst, through the staging buffers for large
// totals, in slots of kD2HSlot bytes: the copy engine fills up to kD2HSlots slots ahead while
// host threads move each landed slot into dst, so only the last slot's host copy trails the
// transfer (a pageable device-to-host copy runs at about half of that).  Returns after every
// byte has arrived.
constexpr size_t kD2HSlot = size_t(4) << 20;
constexpr int kD2HSlots = (int)(2 * kStageChunk / kD2HSlot);

int copy_from_device(ccdgpu_handle *h, char *dst, const char *src, size_t total) {
  if (!total) return CCDGPU_OK;
  Staging &S = staging();
  std::unique_lock<std::mutex> lock(S.mu, std::defer_lock);
  if (total >= kStageMin && lock.try_lock()) {
    if (!S.buf && !S.failed &&
        cudaHostAlloc(reinterpret_cast<void **>(&S.buf), 2 * kStageChunk,
                      cudaHostAllocPortable) != cudaSuccess) {
      (void)cudaGetLastError();
      S.buf = nullptr;
      S.failed = true;
    }
    if (S.buf) {
      cudaEvent_t ev[kD2HSlots] = {};
      cudaError_t e = cudaSuccess;
      for (int k = 0; k < kD2HSlots && e == cudaSuccess; k++)
        e = cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming);
      const int threads = std::max(1, std::min(omp_get_max_threads(), 16));
      const size_t nchunks = (total + kD2HSlot - 1) / kD2HSlot;
      auto issue = [&](size_t c) {
        const size_t off = c * kD2HSlot, n = std::min(kD2HSlot, total - off);
        const int k = (int)(c % kD2HSlots);
        cudaError_t r = cudaMemcpyAsync(S.buf + k * kD2HSlot, src + off, n,
                                        cudaMemcpyDeviceToHost, h->s0);
        if (r == cudaSuccess) r = cudaEventRecord(ev[k], h->s0);
        return r;
      };
      size_t issued = 0;
      for (; e == cudaSuccess && issued < std::min<size_t>(nchunks, kD2HSlots); issued++)
        e = issue(issued);
      for (size_t c = 0; c < nchunks && e == cudaSuccess; c++) {
        const int k = (int)(c % kD2HSlots);
        if ((e = cudaEventSynchronize(ev[k])) != cudaSuccess) break;
        const size_t off = c * kD2HSlot, n = std::min(kD2HSlot, total - off);
        const char *stage = S.buf + k * kD2HSlot;
        const size_t piece = std::max<size_t>(size_t(64) << 10, (n + threads - 1) / threads);
#pragma omp parallel for num_threads(threads) schedule(static)
        for (int64_t x = 0; x < (int64_t)((n + piece - 1) / piece); x++) {
          const size_t lo = (size_t)x * piece;
          std::memcpy(dst + off + lo, stage + lo, std::min(piece, n - lo));
        }
        if (issued < nchunks) e = issue(issued++);  // into the slot just emptied
      }
      (void)cudaStreamSynchronize(h->s0);
      for (int k = 0; k < kD2HSlots; k++)
        if (ev[k]) cudaEventDestroy(ev[k]);
      if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return CCDGPU_ERR_CUDA;
      }
      return CCDGPU_OK;
    }
  }
  CK(cudaMemcpyAsync(dst, src, total, cudaMemcpyDeviceToHost, h->s0));
  CK(cudaStreamSynchronize(h->s0));
  return CCDGPU_OK;
}

// One host array bound for its own device destination.
struct UploadPiece {
  char *dst;
  const char *src;
  size_t n;
};

// Many host arrays to their device destinations in one pass.  Large batches go through the
// staging buffers: host threads pack the next pieces into one buffer (16-byte aligned), then
// every piece is one asynchronous copy out of page-locked memory, so the copy engine runs
// them back to back while the host packs the other buffer.  Small batches are pageable copies.
// Returns after every byte has arrived, except with `hold` when the batch fit one buffer: the
// copies are then left in flight on s0 and the staging lock moves to *hold, which the caller
// keeps until s0 has passed them (no staging use by this thread meanwhile).
int copy_pieces_to_device(ccdgpu_handle *h, const std::vector<UploadPiece> &pcs,
                          std::unique_lock<std::mutex> *hold = nullptr) {
  size_t total = 0;
  for (const UploadPiece &p : pcs) total += p.n;
  if (!total) return CCDGPU_OK;
  Staging &S = staging();
  std::unique_lock<std::mutex> lock(S.mu, std::defer_lock);
  if (total >= kStageMin && lock.try_lock()) {
    if (!S.buf && !S.failed &&
        cudaHostAlloc(reinterpret_cast<void **>(&S.buf), 2 * kStageChunk,
                      cudaHostAllocPortable) != cudaSuccess) {
      (void)cudaGetLastError();
      S.buf = nullptr;
      S.failed = true;
    }
    if (S.buf) {
      cudaEvent_t ev[2] = {nullptr, nullptr};
      bool pending[2] = {false, false};
      cudaError_t e = cudaSuccess;
      for (int k = 0; k < 2 && e == cudaSuccess; k++)
        e = cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming);
      const int threads = std::max(1, std::min(omp_get_max_threads(), 16));
      struct Part {
        size_t off;  // in the staging buffer
        const char *src;
        char *dst;
        size_t n;
      };
      std::vector<Part> parts, work;
      size_t i = 0, done = 0;  // current piece, and its bytes already placed
      for (int k = 0; i < pcs.size() && e == cudaSuccess; k ^= 1) {
        char *stage = S.buf + k * kStageChunk;
        if (pending[k] && (e = cudaEventSynchronize(ev[k])) != cudaSuccess) break;
        parts.clear();
        size_t used = 0;
        while (i < pcs.size() && used < kStageChunk) {
          const size_t n = std::min(pcs[i].n - done, kStageChunk - used);
          if (n) parts.push_back(Part{used, pcs[i].src + done, pcs[i].dst + done, n});
          used = std::min(kStageChunk, used + ((n + 15) & ~size_t(15)));
          done += n;
          if (done == pcs[i].n) {
            i++;
            done = 0;
          }
        }
        // Host threads fill the buffer in slices of at most used / threads bytes.
        const size_t slice = std::max<size_t>(size_t(64) << 10, (used + threads - 1) / threads);
        work.clear();
        for (const Part &p : parts)
          for (size_t x = 0; x < p.n; x += slice)
            work.push_back(Part{p.off + x, p.src + x, nullptr, std::min(slice, p.n - x)});
#pragma omp parallel for num_threads(threads) schedule(dynamic, 4)
        for (int64_t j = 0; j < (int64_t)work.size(); j++)
          std::memcpy(stage + work[j].off, work[j].src, work[j].n);
        for (size_t j = 0; j < parts.size() && e == cudaSuccess; j++)
          e = cudaMemcpyAsync(parts[j].dst, stage + parts[j].off, parts[j].n,
                              cudaMemcpyHostToDevice, h->s0);
        if (e == cudaSuccess) e = cudaEventRecord(ev[k], h->s0);
        pending[k] = e == cudaSuccess;
      }
      if (hold && e == cudaSuccess && total <= kStageChunk) {
        for (int k = 0; k < 2; k++)
          if (ev[k]) cudaEventDestroy(ev[k]);
        *hold = std::move(lock);
        return CCDGPU_OK;
      }
      for (int k = 0; k < 2; k++) {
        if (pending[k]) {
          const cudaError_t w = cudaEventSynchronize(ev[k]);
          if (e == cudaSuccess) e = w;
        }
        if (ev[k]) cudaEventDestroy(ev[k]);
      }
      if (e != cudaSuccess) {
        (void)cudaStreamSynchronize(h->s0);
        (void)cudaGetLastError();
        return CCDGPU_ERR_CUDA;
      }
      return CCDGPU_OK;
    }
  }
  for (const UploadPiece &p : pcs)
    if (p.n) CK(cudaMemcpyAsync(p.dst, p.src, p.n, cudaMemcpyHostToDevice, h->s0));
  return CCDGPU_OK;
}

// Copies per-channel host blocks (block k of `count[k]` elements at src[k]) to consecutive
// device positions; blocks adjacent in host memory form one run.
template <typename T>
int upload_runs(ccdgpu_handle *h, T *dst, const std::vector<const T *> &src,
                const std::vector<int64_t> &count) {
  std::vector<const char *> rs;
  std::vector<size_t> rl;
  for (size_t k = 0; k < src.size(); k++) {
    if (!count[k]) continue;
    const char *p = reinterpret_cast<const char *>(src[k]);
    const size_t n = (size_t)count[k] * sizeof(T);
    if (!rs.empty() && rs.back() + rl.back() == p) {
      rl.back() += n;
    } else {
      rs.push_back(p);
      rl.push_back(n);
    }
  }
  return copy_runs_to_device(h, reinterpret_cast<char *>(dst), rs, rl);
}

// pp-ladder work tiles for a schedule (split factors of K per column class), in their own
// device allocation; drops captured graphs, which hold the old lists.
//   FP64 ladder: thin row blocks stream at full bandwidth on their own, so K is split only when
//   there are fewer of them than SMs (up to thin_split_mul tiles per SM); mid/wide tiles are
//   compute-latency bound per CTA, so K is split into segments of at least four chunks until
//   the class has about wide_split_mul tiles per SM.
//   Tensor-core ladder: each CTA is bandwidth bound, so K is split until there are about
//   tc_split_mul tiles per SM.
// Split row blocks are reduced after the ladder by ladder_reduce_kernel (segment order, so
// deterministic), one item per (row block, 16-row chunk), FP64 items grouped by class.
// Longest-processing-time assignment of tiles[lo, hi) to G persistent CTAs: sorted by cost,
// largest first, each tile goes to the CTA with the least work so far; the range is rewritten
// grouped by CTA and the CTAs' ranges are appended to `off` (absolute indices, G + 1 entries).
template <class Cost>
void lpt_group(std::vector<LadderTile> &tiles, size_t lo, size_t hi, int G, Cost cost,
               std::vector<int32_t> &off) {
  // Costs once; (-cost, position) pairs sorted ascending give the order of a stable sort by
  // decreasing cost.
  const size_t n = hi - lo;
  std::vector<std::pair<int64_t, int32_t>> order(n);
  for (size_t i = 0; i < n; i++) order[i] = {-cost(tiles[lo + i]), (int32_t)i};
  std::sort(order.begin(), order.end());
  std::priority_queue<std::pair<int64_t, int>, std::vector<std::pair<int64_t, int>>,
                      std::greater<std::pair<int64_t, int>>> load;
  for (int b = 0; b < G; b++) load.push({0, b});
  std::vector<int32_t> owner(n), count(G + 1, 0);
  for (size_t i = 0; i < n; i++) {
    auto [w, b] = load.top();
    load.pop();
    owner[i] = b;
    count[b + 1]++;
    load.push({w - order[i].first, b});
  }
  // Each CTA's tiles in the order they were assigned, CTA after CTA.
  for (int b = 0; b < G; b++) count[b + 1] += count[b];
  std::vector<LadderTile> placed(n);
  std::vector<int32_t> next(count.begin(), count.end() - 1);
  for (size_t i = 0; i < n; i++) placed[next[owner[i]]++] = tiles[lo + order[i].second];
  std::copy(placed.begin(), placed.end(), tiles.begin() + lo);
  for (int b = 0; b <= G; b++) off.push_back((int32_t)(lo + count[b]));
}

int make_ladder_tiles(ccdgpu_handle *h, const ccdgpu_schedule &sch) {
  const std::vector<ChanInfo> &chans = h->host_chans;
  auto cls_of = [](int nb) { return nb <= 8 ? 0 : nb <= 32 ? 1 : 2; };
  int64_t blocks[3] = {0, 0, 0};
  for (const ChanInfo &a : chans) blocks[cls_of(a.nb)] += a.nmt;
  const int64_t kSMs = 148;
  const int mid_mul = sch.mid_split_mul > 0 ? sch.mid_split_mul : sch.wide_split_mul;
  auto want_of = [&](int64_t mul, int64_t b) {
    return (int)std::min<int64_t>(64, std::max<int64_t>(1, ceil_div(mul * kSMs, std::max<int64_t>(b, 1))));
  };
  const int want_cls[3] = {
      blocks[0] >= kSMs ? 1 : (int)std::min<int64_t>(8, ceil_div(sch.thin_split_mul * kSMs, std::max<int64_t>(blocks[0], 1))),
      want_of(mid_mul, blocks[1]), want_of(sch.wide_split_mul, blocks[2])};
  std::vector<LadderTile> tiles;
  int64_t lpart_tot = 0;
  int32_t groups = 0;
  for (int ai = 0; ai < h->n_act; ai++) {
    const ChanInfo &a = chans[ai];
    const int want = want_cls[cls_of(a.nb)];
    const int min_chunks = 4;
    const int nseg = std::max(1, std::min(want, a.nkc / min_chunks));
    for (int mt = 0; mt < a.nmt; mt++) {
      const int rows = std::min(a.bm, a.pr - mt * a.bm);
      const int64_t pbase = lpart_tot;
      if (nseg > 1) lpart_tot += (int64_t)nseg * a.bm * a.nb;
      for (int sg = 0; sg < nseg; sg++) {
        LadderTile tl{};
        tl.ch = ai; tl.mt = mt;
        tl.kc0 = (int)((int64_t)a.nkc * sg / nseg);
        tl.nks = (int)((int64_t)a.nkc * (sg + 1) / nseg) - tl.kc0;
        tl.nkc = a.nkc;
        tl.nkh = (sg == nseg - 1) ? a.nkh : 0;
        tl.nb = a.nb; tl.bm = a.bm; tl.rows = rows; tl.pr = a.pr; tl.hh = a.hh;
        tl.seg = sg; tl.nseg = nseg; tl.group = groups;
        tl.v_base = a.vkt_base; tl.tkt_base = a.tkt_base; tl.tmt_base = a.tmt_base;
        tl.xt_base = a.xt_base; tl.t_off = a.t_off; tl.row_off = a.row_off;
        tl.part_base = pbase;
        tiles.push_back(tl);
      }
      groups++;
    }
  }
  // Thin channels first, then mid and wide ones; each class runs on persistent CTAs (3, 2 and
  // 1 per SM) with a balanced (LPT) assignment.  Cost = bytes per 16-deep chunk x chunks, plus
  // two chunks' worth for the pipeline fill and the epilogue.
  {  // stable by class: three passes
    std::vector<LadderTile> by_cls;
    by_cls.reserve(tiles.size());
    for (int k = 0; k < 3; k++)
      for (const LadderTile &t : tiles)
        if (cls_of(t.nb) == k) by_cls.push_back(t);
    tiles.swap(by_cls);
  }
  std::vector<int32_t> fp_cta_off;
  {
    auto fp_cost = [](const LadderTile &x) {
      return (int64_t)(x.nks + x.nkh + 2) * (ladder_arows(x.nb, x.rows) + ladder_bs(x.nb));
    };
    size_t lo = 0;
    const int slots[3] = {3 * 148, 2 * 148, 148};
    for (int k = 0; k < 3; k++) {
      size_t hi = lo;
      while (hi < tiles.size() && cls_of(tiles[hi].nb) == k) hi++;
      h->fp_off_base[k] = (int)fp_cta_off.size();
      h->fp_grid[k] = (int)std::min<size_t>(hi - lo, slots[k]);
      if (hi > lo) lpt_group(tiles, lo, hi, h->fp_grid[k], fp_cost, fp_cta_off);
      lo = hi;
    }
  }
  std::vector<LadderTile> tc_tiles;
  int64_t tcpart_tot = 0;
  int32_t tc_groups = 0;
  if (h->nt) {
    int64_t blocks = 0;
    for (const ChanInfo &a : chans) blocks += ceil_div(a.pr, kTcBM);
    const int want = (int)std::min<int64_t>(32, std::max<int64_t>(1, ceil_div(sch.tc_split_mul * kSMs, blocks)));
    for (int ai = 0; ai < h->n_act; ai++) {
      const ChanInfo &a = chans[ai];
      const int nmt = (int)ceil_div(a.pr, kTcBM);
      const int nseg = std::max(1, std::min(want, a.nkct / 4));
      for (int mt = 0; mt < nmt; mt++) {
        const int rows = std::min(kTcBM, a.pr - mt * kTcBM);
        const int64_t pbase = tcpart_tot;
        if (nseg > 1) tcpart_tot += (int64_t)nseg * kTcBM * a.nbt;
        for (int sg = 0; sg < nseg; sg++) {
          LadderTile tl{};
          tl.ch = ai; tl.mt = mt;
          tl.kc0 = (int)((int64_t)a.nkct * sg / nseg);
          tl.nks = (int)((int64_t)a.nkct * (sg + 1) / nseg) - tl.kc0;
          tl.nkc = a.nkct;
          tl.nkh = (sg == nseg - 1) ? a.nkht : 0;
          tl.nb = a.nbt; tl.bm = kTcBM; tl.rows = rows; tl.pr = a.pr; tl.hh = a.hh;
          tl.seg = sg; tl.nseg = nseg; tl.group = tc_groups;
          tl.v_base = a.vtc_base; tl.tkt_base = a.tkt_tc_base; tl.tmt_base = a.tmt_tc_base;
          tl.xt_base = a.xt_tc_base; tl.t_off = a.t_off; tl.row_off = a.row_off;
          tl.part_base = pbase;
          tc_tiles.push_back(tl);
        }
        tc_groups++;
      }
    }
    // The persistent CTAs claim tiles in list order from a launch-wide counter: sorted by
    // decreasing cost, that is longest-first list scheduling.  Cost = bytes streamed per
    // 32-deep chunk x chunks, plus two chunks' worth for the pipeline fill and the epilogue.
    auto tc_cost = [](const LadderTile &x) {
      return (int64_t)(x.nks + x.nkh + 2) * (((x.rows + 7) & ~7) + x.nb);
    };
    // (-cost, position) pairs sorted ascending: the order of a stable sort by decreasing cost.
    std::vector<std::pair<int64_t, int32_t>> ord(tc_tiles.size());
    for (size_t i = 0; i < tc_tiles.size(); i++) ord[i] = {-tc_cost(tc_tiles[i]), (int32_t)i};
    std::sort(ord.begin(), ord.end());
    std::vector<LadderTile> sorted(tc_tiles.size());
    for (size_t i = 0; i < ord.size(); i++) sorted[i] = tc_tiles[ord[i].second];
    tc_tiles.swap(sorted);
  }
  // Reduction items of split row blocks.
  auto red_items = [](const std::vector<LadderTile> &tl, std::vector<RedItem> &out, int *per_cls,
                      bool by_class, int (*cls)(int)) {
    std::vector<std::vector<RedItem>> parts(by_class ? 3 : 1);
    std::vector<char> seen;
    for (size_t i = 0; i < tl.size(); i++) {
      const LadderTile &t = tl[i];
      if (t.nseg <= 1) continue;
      if ((size_t)t.group >= seen.size()) seen.resize(t.group + 1, 0);
      if (seen[t.group]) continue;
      seen[t.group] = 1;
      for (int r0 = 0; r0 < t.rows; r0 += kRedRows)
        parts[by_class ? cls(t.nb) : 0].push_back({(int32_t)i, r0});
    }
    for (size_t k = 0; k < parts.size(); k++) {
      if (per_cls) per_cls[k] = (int)parts[k].size();
      out.insert(out.end(), parts[k].begin(), parts[k].end());
    }
  };
  std::vector<RedItem> red_fp, red_tc;
  red_items(tiles, red_fp, h->n_red_cls, true, [](int nb) { return nb <= 8 ? 0 : nb <= 32 ? 1 : 2; });
  red_items(tc_tiles, red_tc, nullptr, false, nullptr);
  // Device copies: one allocation, counters zeroed, written on s3, which s0 then waits for.
  // A schedule that replaces another first waits for the handle's work in flight (the old
  // lists may be in use); the first one, made in create while the set-up kernels run on s0,
  // has nothing to wait for, so create's host work goes on beside them.
  const bool first = h->tile_mem == nullptr;
  if (!first) {
    CK(cudaStreamSynchronize(h->s0));
    CK(cudaStreamSynchronize(h->s2));
    CK(cudaStreamSynchronize(h->s3));
  }
  // Captured graphs hold the previous lists; they go before the block they point into.
  for (cudaGraphExec_t *g : {&h->graph, &h->graph_tc, &h->loop64, &h->loop_tc})
    if (*g) { cudaGraphExecDestroy(*g); *g = nullptr; }
  h->loop_state = 0;
  dev_free(h->tile_mem, h->tile_bytes);
  h->tile_mem = nullptr;
  h->tile_bytes = 0;
  h->tiles = h->tc_tiles = nullptr;
  h->lpart = h->tc_part = nullptr;
  h->fp_cta_off = nullptr;
  h->tc_sched = nullptr;
  h->red_fp = h->red_tc = nullptr;
  h->n_tiles = h->n_tc_tiles = 0;
  Arena ar;
  ar.add(&h->tiles, tiles.size()); ar.add(&h->lpart, lpart_tot);
  ar.add(&h->tc_tiles, tc_tiles.size());
  ar.add(&h->fp_cta_off, fp_cta_off.size()); ar.add(&h->tc_sched, 2);
  ar.add(&h->tc_part, tcpart_tot);
  ar.add(&h->red_fp, red_fp.size()); ar.add(&h->red_tc, red_tc.size());
  CK(dev_alloc(ar.used, &h->tile_mem, &h->tile_bytes));
  CK(cudaMemsetAsync(h->tile_mem, 0, ar.used, h->s3));
  for (auto &r : ar.reqs) *r.first = static_cast<char *>(h->tile_mem) + r.second;
  if (!tiles.empty())
    CK(cudaMemcpyAsync(h->tiles, tiles.data(), tiles.size() * sizeof(LadderTile),
                       cudaMemcpyHostToDevice, h->s3));
  if (!tc_tiles.empty())
    CK(cudaMemcpyAsync(h->tc_tiles, tc_tiles.data(), tc_tiles.size() * sizeof(LadderTile),
                       cudaMemcpyHostToDevice, h->s3));
  if (!fp_cta_off.empty())
    CK(cudaMemcpyAsync(h->fp_cta_off, fp_cta_off.data(), fp_cta_off.size() * sizeof(int32_t),
                       cudaMemcpyHostToDevice, h->s3));
  h->tc_grid = (int)std::min<size_t>(tc_tiles.size(), kTcGrid);
  if (!red_fp.empty())
    CK(cudaMemcpyAsync(h->red_fp, red_fp.data(), red_fp.size() * sizeof(RedItem),
                       cudaMemcpyHostToDevice, h->s3));
  if (!red_tc.empty())
    CK(cudaMemcpyAsync(h->red_tc, red_tc.data(), red_tc.size() * sizeof(RedItem),
                       cudaMemcpyHostToDevice, h->s3));
  h->n_red_fp = (int)red_fp.size();
  h->n_red_tc = (int)red_tc.size();
  CK(cudaEventRecord(h->ev_fork2, h->s3));
  CK(cudaStreamWaitEvent(h->s0, h->ev_fork2, 0));
  if (!first) CK(cudaStreamSynchronize(h->s0));
  h->n_tiles = (int)tiles.size();
  h->n_cls[0] = h->n_cls[1] = h->n_cls[2] = 0;
  for (const LadderTile &t : tiles) h->n_cls[cls_of(t.nb)]++;
  h->n_tc_tiles = (int)tc_tiles.size();
  h->schedule = sch;
  return CCDGPU_OK;
}

using TcKernel = void (*)(const LadderTile *, int, int32_t *, const __nv_bfloat16 *, int64_t,
                         const __nv_bfloat16 *, int64_t, const __nv_bfloat16 *, int64_t,
                         const __nv_bfloat16 *, int64_t, const int32_t *, const int32_t *,
                         double *, double *, const Control *, int32_t *, const ChanInfo *,
                         const VGenRow *, const uint32_t *, const double *);
TcKernel tc_kernel_of(int nt, bool gen) {
  if (nt == 2) return gen ? pp_ladder_tc_kernel<2, true> : pp_ladder_tc_kernel<2, false>;
  return gen ? pp_ladder_tc_kernel<3, true> : pp_ladder_tc_kernel<3, false>;
}

// Host work lists of build(), kept per thread between creates: their pages are touched once
// (first-touch page faults of ~20 MB of fresh vectors were most of a warm create's host time
// on the largest bases), later creates only clear them.
struct BuildScratch {
  std::vector<int32_t> rowmap, mirror, kcol, pp_swap, hh_swap, list;
  std::vector<int2> pk_idx, pp_pairs, hh_pairs, vrows, mod_ph, mod_hp, mod_dims;
  std::vector<QuadCol> quad_cols;
  std::vector<QuadItem> quad_items;
  std::vector<ElemRange> ranges;
  std::vector<int64_t> o_t, o_m, o_m_scratch, list_cnt;
  std::vector<int4> gv_items, gvt_items, mlook;
  std::vector<uint64_t> mod_chan;
  std::vector<int32_t> mod_gen_chan;
};
thread_local BuildScratch t_build_scratch;

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

void ready_loop_graphs(ccdgpu_handle *h);

int build(ccdgpu_handle *h, const ccdgpu_problem *P) {
  const auto t_build = std::chrono::steady_clock::now();
  const uint64_t nch = P->n_channels, nsp = P->n_sp, np = P->n_particles;
  h->nch = nch; h->nsp = nsp; h->np = np; h->npart = nsp - np;
  const ccdgpu_channel_dims *D = P->chan_dims, *MD = P->chan_mod_dims;
  // V_ON_THE_FLY: V_pppp is generated on the device from the model, P->v_pppp is not read.
  const bool on_the_fly =
      h->opt.v_mode == CCDGPU_V_ON_THE_FLY || h->opt.v_mode == CCDGPU_V_IN_LADDER;
  const ccdgpu_model *M = P->model;
  const bool model_ok = M && M->qn && M->kind >= CCDGPU_MODEL_PAIRING &&
                        M->kind <= CCDGPU_MODEL_ELECTRON_GAS &&
                        M->qn_stride >= (M->kind == CCDGPU_MODEL_PAIRING ? 2 : 5);
  if (on_the_fly && !model_ok) return CCDGPU_ERR_INVALID_ARGUMENT;
  if (!on_the_fly && !P->v_pppp) return CCDGPU_ERR_INVALID_ARGUMENT;
  // No V_hhhh, V_hhpp and modified-channel V at all (all four NULL): generated on the device
  // from the model, like V_pppp in the on-the-fly mode.
  const int n_vblocks = (P->v_hhhh ? 1 : 0) + (P->v_hhpp ? 1 : 0) + (P->v_hpph_mod ? 1 : 0) +
                        (P->v_hphp_mod ? 1 : 0);
  if (n_vblocks != 0 && n_vblocks != 4) return CCDGPU_ERR_INVALID_ARGUMENT;
  const bool gen_v = n_vblocks == 0;
  if (gen_v && !model_ok) return CCDGPU_ERR_INVALID_ARGUMENT;
  // No loadMaps tables at all: the library derives them on the device from the channel maps.
  int n_maps = 0;
  for (int k = 0; k < 8; k++) n_maps += P->maps[k] ? 1 : 0;
  if (n_maps != 0 && n_maps != 8) return CCDGPU_ERR_INVALID_ARGUMENT;
  const bool derive_tables = n_maps == 0;

  BuildScratch &bs = t_build_scratch;
  std::vector<int64_t> &o_t = bs.o_t, &o_m = bs.o_m;
  o_t.assign(nch + 1, 0);
  o_m.assign(nch + 1, 0);
  for (uint64_t c = 0; c < nch; c++) {
    o_t[c + 1] = o_t[c] + (int64_t)(D[c].pp * D[c].hh);
    o_m[c + 1] = o_m[c] + (int64_t)(MD[c].ph * MD[c].hp);
  }
  h->n_t = o_t[nch];
  h->n_m = o_m[nch];
  if (h->n_t != h->n_m) return CCDGPU_ERR_BAD_TABLE;  // pphh <-> phhp must be a bijection
  if (h->n_t >= (int64_t)INT32_MAX / 2) return CCDGPU_ERR_UNSUPPORTED;
  const int64_t n_t = h->n_t;

  // ---- per-channel metadata (O(sum pp) host work) ----
  // Active channels (pp, hh > 0) and their pair offsets; then two passes over the channels,
  // run in parallel (each writes its own ranges): pairs, swap partners and validation, then the
  // packed-row and K index lists, whose offsets need every channel's counts from the first.
  std::vector<ChanInfo> chans;
  std::vector<uint64_t> act_chan;  // reference channel of each active channel
  std::vector<int64_t> a_pp_off(1, 0), a_hh_off(1, 0);
  for (uint64_t c = 0; c < nch; c++) {
    const int64_t pp = D[c].pp, hh = D[c].hh;
    if (!pp || !hh) continue;
    if (hh > 8 * kMaxCG || pp > (1 << 20)) return CCDGPU_ERR_UNSUPPORTED;
    if (!P->chan_maps[c].pp || !P->chan_maps[c].hh) return CCDGPU_ERR_INVALID_ARGUMENT;
    act_chan.push_back(c);
    a_pp_off.push_back(a_pp_off.back() + pp);
    a_hh_off.push_back(a_hh_off.back() + hh);
  }
  const int n_act = (int)act_chan.size();
  std::vector<int32_t> &rowmap = bs.rowmap, &mirror = bs.mirror, &kcol = bs.kcol;
  std::vector<int2> &pk_idx = bs.pk_idx, &pp_pairs = bs.pp_pairs, &hh_pairs = bs.hh_pairs,
                    &vrows = bs.vrows;
  std::vector<int32_t> &pp_swap = bs.pp_swap, &hh_swap = bs.hh_swap;
  pp_pairs.resize(a_pp_off[n_act]);
  pp_swap.resize(a_pp_off[n_act]);
  pk_idx.resize(a_pp_off[n_act]);
  hh_pairs.resize(a_hh_off[n_act]);
  hh_swap.resize(a_hh_off[n_act]);
  std::vector<int32_t> a_pr(n_act), a_pk(n_act);
  std::atomic<int> bad{0};
  const int host_threads = std::max(1, std::min(omp_get_max_threads(), 16));
#pragma omp parallel num_threads(host_threads)
  {
    SwapIndex swap_index(nsp);
#pragma omp for schedule(dynamic, 4)
    for (int ai = 0; ai < n_act; ai++) {
      const uint64_t c = act_chan[ai];
      const ccdgpu_pair *pm = P->chan_maps[c].pp, *hm = P->chan_maps[c].hh;
      const int64_t pp = D[c].pp, hh = D[c].hh, off = a_pp_off[ai], hoff = a_hh_off[ai];
      if (!swap_index.build(pm, pp, pp_swap.data() + off)) {
        bad = CCDGPU_ERR_BAD_TABLE;
        continue;
      }
      int pr = 0, pk = 0;
      for (int64_t k = 0; k < pp; k++) {
        const uint64_t a = pm[k].p, b = pm[k].q;
        if (a < np || b < np || a >= nsp || b >= nsp || pp_swap[off + k] < 0) {
          bad = CCDGPU_ERR_BAD_TABLE;
          break;
        }
        pp_pairs[off + k] = make_int2((int)a, (int)b);
        pk += a < b;
        pr += a <= b;
      }
      a_pr[ai] = pr;
      a_pk[ai] = pk;
      for (int64_t k = 0; k < hh; k++) {
        const uint64_t i = hm[k].p, j = hm[k].q;
        const int sw = (i < np && j < np) ? find_pair(hm, hh, j, i) : -1;
        if (sw < 0) {
          bad = CCDGPU_ERR_BAD_TABLE;
          break;
        }
        hh_pairs[hoff + k] = make_int2((int)i, (int)j);
        hh_swap[hoff + k] = sw;
      }
    }
  }
  if (bad) return bad;
  std::vector<int64_t> a_row_off(n_act + 1, 0), a_pk_off(n_act + 1, 0);
  for (int ai = 0; ai < n_act; ai++) {
    a_row_off[ai + 1] = a_row_off[ai] + a_pr[ai];
    a_pk_off[ai + 1] = a_pk_off[ai] + a_pk[ai];
  }
  rowmap.resize(a_row_off[n_act]);
  mirror.resize(a_row_off[n_act]);
  // Row items of the stored-V tiling kernels (not needed when V_pppp is generated).
  vrows.resize(on_the_fly ? 0 : a_row_off[n_act]);
  kcol.resize(a_pk_off[n_act]);
#pragma omp parallel for num_threads(host_threads) schedule(dynamic, 4)
  for (int ai = 0; ai < n_act; ai++) {
    const int64_t pp = D[act_chan[ai]].pp, off = a_pp_off[ai];
    int32_t *rm = rowmap.data() + a_row_off[ai], *mr = mirror.data() + a_row_off[ai];
    int2 *vr = on_the_fly ? nullptr : vrows.data() + a_row_off[ai];
    int32_t *kc = kcol.data() + a_pk_off[ai];
    int pr = 0, pk = 0;
    for (int64_t k = 0; k < pp; k++) {
      const int a = pp_pairs[off + k].x, b = pp_pairs[off + k].y;
      int2 q = make_int2(-1, -1);
      if (a < b) { q.x = pk; kc[pk++] = (int32_t)k; }
      if (a <= b) {
        q.y = pr;
        rm[pr] = (int32_t)k;
        mr[pr] = a < b ? pp_swap[off + k] : -1;
        if (vr) vr[pr] = make_int2(ai, pr);
        pr++;
      }
      pk_idx[off + k] = q;
    }
  }
  std::vector<HHTile> hh_tiles;
  std::vector<HHRed> hh_red;
  int64_t x_tot = 0, tkt = 0, tmt = 0, xt = 0, vt = 0, part_tot = 0;
  int64_t vraw_tot = 0;
  int64_t vtc = 0, tkttc = 0, tmttc = 0, xttc = 0;
  std::vector<int64_t> vraw_off;
  int maxhh = 1;
  for (int ai = 0; ai < n_act; ai++) {
    const uint64_t c = act_chan[ai];
    const int64_t pp = D[c].pp, hh = D[c].hh;
    const int pr = a_pr[ai], pk = a_pk[ai];
    ChanInfo ci{};
    ci.pp = (int)pp; ci.hh = (int)hh;
    ci.nb = ladder_nb((int)hh);
    ci.bm = ladder_bm(ci.nb);
    ci.row_off = a_row_off[ai];
    ci.pk_off = a_pk_off[ai];
    ci.pp_off = a_pp_off[ai]; ci.hh_off = a_hh_off[ai]; ci.x_off = x_tot;
    ci.pr = pr; ci.pk = pk;
    ci.nkc = (int)ceil_div(pk, kBK);
    ci.nkh = (int)ceil_div(hh, kBK);
    ci.nmt = (int)ceil_div(pr, ci.bm);
    const int hh_rows = hh <= 16 ? kHHRows : kHHRowsL;  // K slice of the hh ladder
    ci.nhht = (int)ceil_div(pp, hh_rows);
    ci.t_off = o_t[c];
    ci.tkt_base = tkt; ci.tmt_base = tmt; ci.xt_base = xt; ci.vkt_base = vt;
    ci.part_off = part_tot;
    ci.hht0 = (int64_t)hh_tiles.size();
    ci.nbt = tc_nb(ci.hh);
    ci.nkct = (int)ceil_div(pk, kTcKC);
    ci.nkht = (int)ceil_div(hh, kTcKC);
    ci.vtc_base = vtc; ci.tkt_tc_base = tkttc; ci.tmt_tc_base = tmttc; ci.xt_tc_base = xttc;
    vtc += (int64_t)ci.nkct * kTcGroup * ceil_div(pr, 8);
    tmttc += (int64_t)ci.nkht * kTcGroup * ceil_div(pr, 8);
    tkttc += (int64_t)ci.nkct * (ci.nbt / 8) * kTcGroup;
    xttc += (int64_t)ci.nkht * (ci.nbt / 8) * kTcGroup;
    const int nb = ci.nb;
    x_tot += hh * hh;
    tkt += (int64_t)ci.nkc * kBK * ladder_bs(nb);
    // Full row tiles at their A stride, then the compact last one.
    const int64_t arows_tot = (int64_t)(ci.nmt - 1) * ladder_arows_full(ci.nb) +
                              ladder_arows(ci.nb, ci.pr - (ci.nmt - 1) * ci.bm);
    tmt += (int64_t)ci.nkh * arows_tot * kBK;
    xt += (int64_t)ci.nkh * kBK * ladder_bs(nb);
    vt += (int64_t)ci.nkc * arows_tot * kBK;
    part_tot += (int64_t)ci.nhht * hh * hh;
    vraw_off.push_back(vraw_tot);
    if (!on_the_fly) vraw_tot += (int64_t)ci.pr * pp;  // packed rows (a <= b) only
    maxhh = std::max<int>(maxhh, (int)hh);
    // hh ladder: hh <= 16, one warp unit per K slice (the whole P); wider hh, one CTA unit per
    // K slice of kHHRowsL rows (every P row tile, hh_slice_kernel).
    for (int t = 0; t < ci.nhht; t++)
      hh_tiles.push_back({ai, t * hh_rows, t,
                          (int)std::min<int64_t>(hh_rows, pp - (int64_t)t * hh_rows), 0, 0});
    for (int64_t i0 = 0; i0 < hh * hh; i0 += 256) hh_red.push_back({ai, (int32_t)i0});
    chans.push_back(ci);
  }
  const int64_t pp_tot = a_pp_off[n_act], hh_tot = a_hh_off[n_act];
  h->n_act = n_act;
  h->n_hh_tiles = (int)hh_tiles.size();
  h->n_hh_red = (int)hh_red.size();
  // Channels with hh <= 16 first (their own launch), then the rest; largest units
  // (rows x hh^2) first within each, so the short ones fill in behind them.
  // A stable sort by (class, -cost): the units come channel by channel as runs of equal cost
  // (the full slices, then a shorter last one), so the runs are stably sorted and expanded,
  // which gives the same order as sorting the units themselves.
  {
    struct Run {
      int32_t first, n;
      bool wide;
      int64_t cost;
    };
    std::vector<Run> runs;
    for (int32_t i = 0; i < (int32_t)hh_tiles.size(); i++) {
      const HHTile &t = hh_tiles[i];
      const int64_t hh = chans[t.ch].hh, cost = (int64_t)t.rows * hh * hh;
      if (!runs.empty() && hh_tiles[runs.back().first].ch == t.ch && runs.back().cost == cost)
        runs.back().n++;
      else
        runs.push_back(Run{i, 1, hh > 16, cost});
    }
    std::stable_sort(runs.begin(), runs.end(), [](const Run &x, const Run &y) {
      if (x.wide != y.wide) return !x.wide;
      return x.cost > y.cost;
    });
    std::vector<HHTile> sorted;
    sorted.reserve(hh_tiles.size());
    for (const Run &r : runs)
      sorted.insert(sorted.end(), hh_tiles.begin() + r.first, hh_tiles.begin() + r.first + r.n);
    hh_tiles.swap(sorted);
  }
  for (const HHTile &t : hh_tiles) h->n_hh_small += chans[t.ch].hh <= 16 ? 1 : 0;
  for (const ChanInfo &a : chans)
    if (a.hh > 16) h->hh_slice_smem = std::max(h->hh_slice_smem, hh_slice_smem(a.hh));
  // Per orbital w, the pair elements whose first index is w, ascending (particles: pp
  // elements, holes: hh elements): a counting sort.  The pp elements (first index a particle)
  // are split into one contiguous range per host thread: per-thread bucket counts, then each
  // thread places its range from its own start in every bucket, so a bucket keeps ascending
  // element order.  The hh elements (first index a hole, buckets of their own) follow serially.
  std::vector<int64_t> list_off(nsp + 1, 0);
  std::vector<int32_t> &list = bs.list;
  {
    std::vector<int64_t> &cnt = bs.list_cnt;  // [thread][orbital]: counts, then start offsets
    cnt.assign((size_t)host_threads * nsp, 0);
    int team = 1;
#pragma omp parallel num_threads(host_threads)
    {
#pragma omp single
      team = omp_get_num_threads();
      const int t = omp_get_thread_num();
      const int64_t lo = pp_tot * t / team, hi = pp_tot * (t + 1) / team;
      int64_t *c = cnt.data() + (size_t)t * nsp;
      for (int64_t e = lo; e < hi; e++) c[pp_pairs[e].x]++;
#pragma omp barrier
#pragma omp single
      {
        for (int64_t e = 0; e < hh_tot; e++) list_off[hh_pairs[e].x + 1]++;
        for (uint64_t w = 0; w < nsp; w++) {
          int64_t s = 0;
          for (int u = 0; u < team; u++) s += cnt[(size_t)u * nsp + w];
          list_off[w + 1] += s;
        }
        for (uint64_t w = 0; w < nsp; w++) list_off[w + 1] += list_off[w];
        list.resize(list_off[nsp]);
        for (uint64_t w = 0; w < nsp; w++) {
          int64_t at = list_off[w];
          for (int u = 0; u < team; u++) {
            const int64_t n = cnt[(size_t)u * nsp + w];
            cnt[(size_t)u * nsp + w] = at;
            at += n;
          }
        }
      }
      for (int64_t e = lo; e < hi; e++) list[c[pp_pairs[e].x]++] = (int32_t)e;
    }
    std::vector<int64_t> &cur = bs.o_m_scratch;
    cur.assign(list_off.begin(), list_off.end() - 1);
    for (int64_t e = 0; e < hh_tot; e++) list[cur[hh_pairs[e].x]++] = (int32_t)e;
  }
  h->n_list = list_off[nsp];

  // Modified channels: small ones (one warp each) first, then one group per padded size
  // (32, 48, 64, 80; one CTA per channel).
  std::vector<ModInfo> mods, mods_pad[4];
  std::vector<int2> &mod_dims = bs.mod_dims;
  mod_dims.resize(nch);
  int64_t y_tot = 0;
  std::vector<const double *> src_hpph, src_hphp;
  std::vector<int64_t> cnt_hpph, cnt_hphp;
  std::vector<ModGen> mod_gen;        // generated V: modified channels in channel order
  std::vector<int32_t> &mod_gen_chan = bs.mod_gen_chan;  // ... and their channel slots
  mod_gen_chan.clear();
  std::vector<int2> &mod_ph = bs.mod_ph, &mod_hp = bs.mod_hp;  // ... their ph' (b, j), hp' (i, a) pairs
  mod_ph.clear();
  mod_hp.clear();
  for (uint64_t c = 0; c < nch; c++) {
    const int64_t ph = MD[c].ph, hp = MD[c].hp;
    mod_dims[c] = make_int2((int)ph, (int)hp);
    if (!ph || !hp) continue;
    if (ph > kTcMaxNB || hp > kTcMaxNB) return CCDGPU_ERR_UNSUPPORTED;  // ring register tiles
    ModInfo m{};
    m.ph = (int)ph; m.hp = (int)hp; m.m_off = o_m[c]; m.y_off = y_tot;
    if (gen_v) {
      // The pairs themselves are copied in parallel after this loop.
      if (!P->chan_mod_maps[c].ph || !P->chan_mod_maps[c].hp) return CCDGPU_ERR_INVALID_ARGUMENT;
      const int64_t ph0 = mod_gen.empty() ? 0 : mod_gen.back().ph_off + mod_gen.back().ph;
      const int64_t hp0 = mod_gen.empty() ? 0 : mod_gen.back().hp_off + mod_gen.back().hp;
      mod_gen.push_back(ModGen{(int)ph, (int)hp, m.m_off, m.y_off, ph0, hp0});
      mod_gen_chan.push_back((int32_t)c);
    } else {
      if (!P->v_hpph_mod[c] || !P->v_hphp_mod[c]) return CCDGPU_ERR_INVALID_ARGUMENT;
      src_hpph.push_back(P->v_hpph_mod[c]); cnt_hpph.push_back(ph * hp);
      src_hphp.push_back(P->v_hphp_mod[c]); cnt_hphp.push_back(hp * hp);
    }
    y_tot += hp * hp;
    const int64_t w = std::max(ph, hp);
    if (w <= kRingSmall) mods.push_back(m);
    else mods_pad[w <= 32 ? 0 : w <= 48 ? 1 : w <= 64 ? 2 : 3].push_back(m);
  }
  if (!mod_gen.empty()) {
    mod_ph.resize(mod_gen.back().ph_off + mod_gen.back().ph);
    mod_hp.resize(mod_gen.back().hp_off + mod_gen.back().hp);
    const std::vector<int32_t> &mod_chan = mod_gen_chan;
    std::atomic<int> bad_mod{0};
#pragma omp parallel for num_threads(host_threads) schedule(dynamic, 16)
    for (int64_t g = 0; g < (int64_t)mod_gen.size(); g++) {
      const ModGen &mg = mod_gen[g];
      const ccdgpu_pair *phm = P->chan_mod_maps[mod_chan[g]].ph, *hpm = P->chan_mod_maps[mod_chan[g]].hp;
      for (int64_t k = 0; k < mg.ph; k++) {
        if (phm[k].p < np || phm[k].p >= nsp || phm[k].q >= np) bad_mod = 1;
        mod_ph[mg.ph_off + k] = make_int2((int)phm[k].p, (int)phm[k].q);
      }
      for (int64_t k = 0; k < mg.hp; k++) {
        if (hpm[k].p >= np || hpm[k].q < np || hpm[k].q >= nsp) bad_mod = 1;
        mod_hp[mg.hp_off + k] = make_int2((int)hpm[k].p, (int)hpm[k].q);
      }
    }
    if (bad_mod) return CCDGPU_ERR_BAD_TABLE;
  }
  // Largest channels first within a group, so that the short ones fill in behind them.
  auto by_work = [](const ModInfo &x, const ModInfo &y) {
    return (int64_t)x.ph * x.hp * x.hp > (int64_t)y.ph * y.hp * y.hp;
  };
  h->n_mod_small = (int)mods.size();
  for (int k = 0; k < 4; k++) {
    std::stable_sort(mods_pad[k].begin(), mods_pad[k].end(), by_work);
    h->n_mod_pad[k] = (int)mods_pad[k].size();
    mods.insert(mods.end(), mods_pad[k].begin(), mods_pad[k].end());
  }
  h->n_mod_mid = h->n_mod_pad[0];
  h->n_mod = (int)mods.size();
  h->host_mods = mods;

  std::vector<int64_t> o_h(np + 1, 0), o_p(h->npart + 1, 0);
  for (uint64_t k = 0; k < np; k++) o_h[k + 1] = o_h[k] + (int64_t)P->three_body_dims[k].hpp;
  for (uint64_t a = 0; a < h->npart; a++)
    o_p[a + 1] = o_p[a] + (int64_t)P->three_body_dims[np + a].phh;
  h->n_h = o_h[np];
  h->n_p = o_p[h->npart];
  if (h->n_h != n_t || h->n_p != n_t) return CCDGPU_ERR_BAD_TABLE;
  // Three-body V of the table path: from the host, or generated with the other V blocks when
  // the problem carries none of them and the handle runs the table path (the fused path reads
  // none: its one-body sums come from the hh ladder's row dots).
  const bool gen_v3 = gen_v && !P->v_h_hpp && !P->v_phh_p && h->opt.path == CCDGPU_PATH_TABLES;
  h->have_3body = (P->v_h_hpp && P->v_phh_p) || gen_v3;

  h->host_chans = chans;

  std::vector<ElemRange> &ranges = bs.ranges;
  ranges.clear();
  const int64_t per = (int64_t)kAsmThreads * kAsmPerThread;
  for (int ai = 0; ai < h->n_act; ai++) {
    const ChanInfo &a = chans[ai];
    const int64_t n = (int64_t)a.pp * a.hh;
    for (int64_t e = 0; e < n; e += per) ranges.push_back({ai, 0, a.t_off + e, a.t_off + std::min(n, e + per)});
  }
  h->n_ranges = (int)ranges.size();
  // Fused assembly: quads (strict packed row a < b, strict hole pair i < j) per channel, their
  // static tables, and work items of up to kQuadPerItem quads of one channel.
  std::vector<QuadCol> &quad_cols = bs.quad_cols;
  std::vector<QuadItem> &quad_items = bs.quad_items;
  quad_cols.clear();
  quad_items.clear();
  // Rows: the packed rows with a < b (pk of them per channel), filled in parallel below;
  // columns (i < j) and work items here.
  int64_t qrows_tot = 0;
  for (int ai = 0; ai < h->n_act; ai++) {
    ChanInfo &a = chans[ai];
    a.qrow_off = qrows_tot;
    qrows_tot += a.pk;
    a.qcol_off = (int64_t)quad_cols.size();
    for (int j = 0; j < a.hh; j++) {
      const int2 pij = hh_pairs[a.hh_off + j];
      if (pij.x >= pij.y) continue;  // i = j: zero column; i > j: the mirror of (j, i)
      QuadCol c{};
      c.c_ij = j; c.c_ji = hh_swap[a.hh_off + j]; c.i = pij.x; c.j = pij.y;
      c.eij = P->sp_energy[pij.x] + P->sp_energy[pij.y];
      quad_cols.push_back(c);
    }
    a.hk = (int)((int64_t)quad_cols.size() - a.qcol_off);
    const int64_t nq = (int64_t)a.pk * a.hk;
    if (nq >= ((int64_t)1 << 31) / 2) return CCDGPU_ERR_UNSUPPORTED;
    for (int64_t q = 0; q < nq; q += kQuadPerItem)
      quad_items.push_back({ai, (int32_t)q, (int32_t)std::min<int64_t>(nq, q + kQuadPerItem),
                            a.hk, a.t_off, a.qrow_off, a.qcol_off});
  }
  h->n_quad_rows = qrows_tot;  // built on the device (quad_rows_kernel)

  h->host_chans = chans;
  h->n_quad_items = (int)quad_items.size();
  // Persistent assembly grid: kAsmCTAsPerSM resident CTAs per SM at most (one CTA if there is no quad,
  // for the energy and the stop rule).
  h->n_asm_blocks = h->n_act ? std::max(1, std::min(h->n_quad_items, kAsmCTAsPerSM * 148)) : 0;

  // Work estimate (reference GEMM flops) for roofline reporting.
  double fl = 0, lf = 0, vb = 0, vbp = 0;
  for (const ChanInfo &a : chans) {
    lf += 2.0 * a.pp * a.pp * a.hh;
    fl += 2.0 * a.pp * a.pp * a.hh + 4.0 * a.pp * a.hh * (double)a.hh;
    vb += 8.0 * a.pp * a.pp;
    vbp += 8.0 * a.pr * (double)a.pk;
  }
  for (const ModInfo &m : mods) fl += 4.0 * m.ph * (double)m.hp * m.hp;
  h->flops = fl; h->ladder_flops = lf; h->v_bytes = vb; h->v_packed_bytes = vbp;
  // Bytes one pp-ladder launch must move: packed V, the T operand rows (c<d for V T, a<=b
  // for T X), X, and D written in full.
  double lb = vbp;
  for (const ChanInfo &a : chans)
    lb += 8.0 * ((double)a.pk * a.hh + (double)a.pr * a.hh + (double)a.hh * a.hh + (double)a.pp * a.hh);
  h->ladder_bytes = lb;
  double lbt = 0;
  for (const ChanInfo &a : chans)
    lbt += 2.0 * h->nt * ((double)a.pr * a.pk + (double)a.pk * a.hh + (double)a.pr * a.hh +
                          (double)a.hh * a.hh) + 8.0 * a.pp * (double)a.hh;
  h->ladder_bytes_tc = lbt;
  h->n_tkt = tkt;
  h->n_tmt = tmt;

  // Tensor-core ladder with V generated in the kernel (electron gas, on-the-fly V, momenta
  // |n_i| <= 6 so that q^2 <= 432): per packed row u (rowmap order) the codes of a and b, per K
  // index w (kcol order) the code of c (momentum bytes biased by 64, spin in byte 3), and the
  // direct term by q^2.
  std::vector<VGenRow> vg_rows;
  std::vector<uint32_t> vg_cols;
  std::vector<double> vg_tab;
  if (h->opt.v_mode == CCDGPU_V_IN_LADDER && h->nt && model_ok &&
      M->kind == CCDGPU_MODEL_ELECTRON_GAS) {
    int nmax = 0;
    for (uint64_t o = 0; o < nsp; o++)
      for (int i = 0; i < 3; i++) nmax = std::max(nmax, std::abs(M->qn[o * M->qn_stride + i]));
    if (nmax <= 6) {
      h->tc_gen = true;
      auto code = [&](int o) {
        const int32_t *q = M->qn + (int64_t)o * M->qn_stride;
        return (uint32_t)(q[0] + 64) | ((uint32_t)(q[1] + 64) << 8) |
               ((uint32_t)(q[2] + 64) << 16) | ((uint32_t)(q[3] > 0 ? kVGenSpin : 0) << 24);
      };
      vg_rows.resize(rowmap.size());
      vg_cols.resize(kcol.size());
      for (const ChanInfo &a : chans) {
        for (int u = 0; u < a.pr; u++) {
          const int2 ab = pp_pairs[a.pp_off + rowmap[a.row_off + u]];
          vg_rows[a.row_off + u] = VGenRow{code(ab.x), code(ab.y)};
        }
        for (int w = 0; w < a.pk; w++)
          vg_cols[a.pk_off + w] = code(pp_pairs[a.pp_off + kcol[a.pk_off + w]].x);
      }
      // w(q^2) = e^2 / L^3 * 4 pi / (2 pi / L)^2 q^2, zero for q = 0 (ElectronGasSPBasis.cpp:
      // 453-466 as a function of q^2).
      const double L = M->params[0], e_sq = M->params[1];
      vg_tab.assign(kTcGenTab, 0.0);
      for (int q2 = 1; q2 <= 3 * 12 * 12; q2++) {  // beyond: spins differ, zero
        const double rel = (2 * M_PI / L) * (2 * M_PI / L) * q2;
        vg_tab[q2] = e_sq / (L * L * L) * 4 * M_PI / rel;
      }
      // The ladder then moves no V bytes: the T and X operand images and D.
      double lbg = 0;
      for (const ChanInfo &a : chans)
        lbg += 2.0 * h->nt * ((double)a.pk * a.hh + (double)a.pr * a.hh + (double)a.hh * a.hh) +
               8.0 * a.pp * (double)a.hh;
      h->ladder_bytes_tc = lbg;
    }
  }

  // ---- one device allocation ----
  h->create_ms[0] = ms_since(t_build);
  Arena ar;
  ar.add(&h->chans, chans.size()); ar.add(&h->mods, mods.size());
  ar.add(&h->hh_tiles, hh_tiles.size()); ar.add(&h->hh_red, hh_red.size());
  ar.add(&h->ranges, ranges.size());
  ar.add(&h->pp_pairs, pp_pairs.size()); ar.add(&h->hh_pairs, hh_pairs.size());
  ar.add(&h->pp_swap, pp_swap.size()); ar.add(&h->hh_swap, hh_swap.size());
  ar.add(&h->list_off, list_off.size()); ar.add(&h->list, list.size());
  ar.add(&h->rowmap, rowmap.size()); ar.add(&h->mirror, mirror.size());
  ar.add(&h->pk_idx, pk_idx.size());
  ar.add(&h->part, part_tot);

  ar.add(&h->eps, nsp);
  // Generated V images are written in full (padding included) by the V generators.
  ar.add(&h->v_pphh, n_t); ar.add(&h->v_hhhh, x_tot);
  if (on_the_fly) ar.add_unset(&h->v_t, vt);
  else ar.add(&h->v_t, vt);
  ar.add(&h->v_hpph, h->n_m); ar.add(&h->v_hphp, y_tot);
  ar.add(&h->flat, (size_t)8 * n_t); ar.add(&h->inv4, n_t); ar.add(&h->d_ring, n_t); ar.add(&h->o_h, o_h.size()); ar.add(&h->o_p, o_p.size());
  ar.add(&h->t[0], n_t); ar.add(&h->t[1], n_t); ar.add(&h->dmat, n_t);
  ar.add(&h->old_phhp, h->n_m); ar.add(&h->r_phhp, h->n_m);
  ar.add(&h->x, x_tot); ar.add(&h->x_t, xt); ar.add(&h->t_kt, tkt); ar.add(&h->t_mt, tmt);
  ar.add(&h->s, hh_tot); ar.add(&h->r, pp_tot); ar.add(&h->xh, np); ar.add(&h->yp, h->npart);
  ar.add(&h->quad_items, quad_items.size());
  ar.add(&h->quad_rows, h->n_quad_rows); ar.add(&h->quad_cols, quad_cols.size());
  ar.add(&h->kcol, kcol.size());  // V tiling at create
  ar.add(&h->epart, std::max(h->n_ranges, h->n_asm_blocks)); ar.add(&h->ctl, 1); ar.add(&h->e_out, 1); ar.add(&h->err, 1);
  ar.add(&h->ticket, 1);
  if (h->nt) {
    auto round_up = [](int64_t n) { return std::max<int64_t>(256, (n + 255) / 256 * 256); };
    h->n_vtc = round_up(vtc); h->n_tkttc = round_up(tkttc);
    h->n_tmttc = round_up(tmttc); h->n_xttc = round_up(xttc);
    if (h->tc_gen) {
      h->n_vtc = 0;  // V planes generated in the ladder
      ar.add(&h->vg_rows, vg_rows.size()); ar.add(&h->vg_cols, vg_cols.size());
      ar.add(&h->vg_tab, vg_tab.size());
    } else if (on_the_fly) {
      ar.add_unset(&h->v_tc, (size_t)h->nt * h->n_vtc);
    } else {
      ar.add(&h->v_tc, (size_t)h->nt * h->n_vtc);
    }
    ar.add(&h->tkt_tc, (size_t)h->nt * h->n_tkttc);
    ar.add(&h->tmt_tc, (size_t)h->nt * h->n_tmttc); ar.add(&h->xt_tc, (size_t)h->nt * h->n_xttc);
  }
  if (h->have_3body) {
    ar.add(&h->v_h_hpp, h->n_h); ar.add(&h->v_phh_p, h->n_p);
    ar.add(&h->old_h1pp_h2, h->n_h); ar.add(&h->old_h2pp_h1, h->n_h); ar.add(&h->diff_h2pp_h1, h->n_h);
    ar.add(&h->old_p1_p2hh, h->n_p); ar.add(&h->old_p2_p1hh, h->n_p); ar.add(&h->diff_p2_p1hh, h->n_p);
    ar.add(&h->gath, (size_t)8 * n_t);
  }
  int rc;
#define TRY(x) do { rc = (x); if (rc) return rc; } while (0)
  TRY(ar.commit(h));
  // Scratch for the raw inputs, released at the end of create.
  Arena sc;
  double *vraw = nullptr, *hhpp_raw = nullptr, *hpph_raw = nullptr;
  RawIndex *raw_idx = nullptr;
  int32_t *counts = nullptr;
  int2 *d_vrows = nullptr, *d_mod_dims = nullptr;
  int4 *d_gv_items = nullptr, *d_gvt_items = nullptr;
  // Generated V_pppp: one item per operand-image chunk (channel, row tile, K chunk).
  // Counted per channel, then filled in parallel, each channel at its offset.
  std::vector<int4> &gv_items = bs.gv_items, &gvt_items = bs.gvt_items;
  gv_items.clear();
  gvt_items.clear();
  if (on_the_fly) {
    // With bf16 images both images come from the tensor-core chunks (gen_v_both_chunks_kernel).
    const bool tc_images = h->nt && !h->tc_gen;
    std::vector<int64_t> go(h->n_act + 1, 0), gto(h->n_act + 1, 0);
    for (int ai = 0; ai < h->n_act; ai++) {
      const ChanInfo &a = chans[ai];
      go[ai + 1] = go[ai] + (tc_images ? 0 : (int64_t)a.nmt * a.nkc);
      gto[ai + 1] = gto[ai] + (tc_images ? (int64_t)ceil_div(a.pr, kTcBM) * a.nkct : 0);
    }
    gv_items.resize(go[h->n_act]);
    gvt_items.resize(gto[h->n_act]);
#pragma omp parallel for num_threads(host_threads) schedule(dynamic, 4)
    for (int ai = 0; ai < h->n_act; ai++) {
      const ChanInfo &a = chans[ai];
      int4 *g = gv_items.data() + go[ai];
      if (!tc_images)
        for (int mt = 0; mt < a.nmt; mt++)
          for (int kc = 0; kc < a.nkc; kc++) *g++ = make_int4(ai, mt, kc, 0);
      int4 *gt = gvt_items.data() + gto[ai];
      if (tc_images)
        for (int mt = 0; mt < (int)ceil_div(a.pr, kTcBM); mt++)
          for (int kc = 0; kc < a.nkct; kc++) *gt++ = make_int4(ai, mt, kc, 0);
    }
  }
  int64_t *d_vraw_off = nullptr, *d_o_m = nullptr;
  // Derived tables: per-pair block offsets and the modified-channel lookup of (particle, hole)
  // pairs, built here from the ph' / hp' maps (O(npart * np)).
  int32_t *d_hblk = nullptr, *d_pblk = nullptr;
  int4 *d_mlook = nullptr;
  std::vector<int4> &mlook = bs.mlook;
  mlook.clear();
  // With generated V the ph' / hp' pairs go to the device anyway: the lookup is built there
  // (mod_lookup_kernel); otherwise here.
  const bool mlook_dev = derive_tables && gen_v;
  const uint64_t n_mlook = (nsp - np) * np;
  if (mlook_dev) {
    sc.add(&d_mlook, n_mlook);
  } else if (derive_tables) {
    const uint64_t npart = nsp - np;
    mlook.assign(npart * np, make_int4(-1, -1, -1, -1));
    std::vector<uint64_t> &mc = bs.mod_chan;
    mc.clear();
    for (uint64_t c = 0; c < nch; c++) {
      if (!MD[c].ph || !MD[c].hp) continue;
      if (!P->chan_mod_maps[c].ph || !P->chan_mod_maps[c].hp) return CCDGPU_ERR_INVALID_ARGUMENT;
      mc.push_back(c);
    }
    // In a valid problem every (particle, hole) slot is named by exactly one ph' entry and one
    // hp' entry, so the channels fill their slots in parallel (relaxed atomic stores, so that
    // an invalid problem's duplicates race harmlessly); a second pass checks that each entry's
    // slot holds that entry, which fails for every duplicate but one.
    std::atomic<int> bad_m{0};
    int32_t *ml = reinterpret_cast<int32_t *>(mlook.data());
    auto each_entry = [&](int64_t g, auto &&f) {
      const uint64_t c = mc[g];
      const ccdgpu_pair *phm = P->chan_mod_maps[c].ph, *hpm = P->chan_mod_maps[c].hp;
      for (uint64_t k = 0; k < MD[c].ph; k++) {
        const uint64_t a = phm[k].p, i = phm[k].q;
        if (a < np || a >= nsp || i >= np) bad_m = 1;
        else f(ml + 4 * ((a - np) * np + i), (int)c, (int)k);
      }
      for (uint64_t k = 0; k < MD[c].hp; k++) {
        const uint64_t i = hpm[k].p, a = hpm[k].q;
        if (i >= np || a < np || a >= nsp) bad_m = 1;
        else f(ml + 4 * ((a - np) * np + i) + 2, (int)c, (int)k);
      }
    };
#pragma omp parallel num_threads(host_threads)
    {
#pragma omp for schedule(dynamic, 16)
      for (int64_t g = 0; g < (int64_t)mc.size(); g++)
        each_entry(g, [](int32_t *m, int c, int k) {
          __atomic_store_n(m, c, __ATOMIC_RELAXED);
          __atomic_store_n(m + 1, k, __ATOMIC_RELAXED);
        });
#pragma omp for schedule(dynamic, 16)
      for (int64_t g = 0; g < (int64_t)mc.size(); g++)
        each_entry(g, [&](int32_t *m, int c, int k) {
          if (__atomic_load_n(m, __ATOMIC_RELAXED) != c ||
              __atomic_load_n(m + 1, __ATOMIC_RELAXED) != k)
            bad_m = 1;
        });
    }
    if (bad_m) return CCDGPU_ERR_BAD_TABLE;
    sc.add(&d_mlook, mlook.size());
  } else {
    sc.add(&raw_idx, (size_t)8 * n_t);
  }
  if (derive_tables || gen_v3) {  // block offsets inside hpp(k) and phh(a)
    sc.add(&d_hblk, np * np);
    sc.add(&d_pblk, (nsp - np) * (nsp - np));
  }
  ModGen *d_mod_gen = nullptr;
  int2 *d_mod_ph = nullptr, *d_mod_hp = nullptr;
  int32_t *d_mod_chan = nullptr;
  if (gen_v) {
    sc.add(&d_mod_gen, mod_gen.size()); sc.add(&d_mod_ph, mod_ph.size());
    sc.add(&d_mod_hp, mod_hp.size()); sc.add(&d_mod_chan, mod_gen_chan.size());
  }
  sc.add(&vraw, vraw_tot); sc.add(&hhpp_raw, gen_v ? 0 : n_t);
  sc.add(&hpph_raw, gen_v ? 0 : h->n_m);
  sc.add(&counts, (size_t)5 * n_t); sc.add(&d_vrows, vrows.size());
  sc.add(&d_gv_items, gv_items.size()); sc.add(&d_gvt_items, gvt_items.size());
  sc.add(&d_vraw_off, vraw_off.size()); sc.add(&d_mod_dims, mod_dims.size()); sc.add(&d_o_m, o_m.size());
  // The model on the device (on-the-fly V, E_ref and normal ordering): quantum numbers and
  // (electron gas) the direct Coulomb term by momentum transfer, computed here with the
  // reference's expression (ElectronGasSPBasis.cpp:424-448).  Kept for the handle's lifetime.
  ModelDev md{};
  std::vector<UploadPiece> batch;  // host -> device copies made together, after the lists
  std::unique_lock<std::mutex> staging_hold;  // staging buffers with copies still in flight
  std::vector<double> vq;
  std::vector<uint32_t> ocode;
  int32_t *d_qn = nullptr;
  double *d_vq = nullptr;
  uint32_t *d_ocode = nullptr;
  if (model_ok) {
    md.kind = M->kind;
    md.stride = M->qn_stride;
    md.g = M->params[0];
    md.Lb = M->params[0];
    if (M->kind == CCDGPU_MODEL_ELECTRON_GAS) {
      int nmax = 0;
      for (uint64_t o = 0; o < nsp; o++)
        for (int i = 0; i < 3; i++) nmax = std::max(nmax, std::abs(M->qn[o * M->qn_stride + i]));
      md.R = 2 * nmax;
      md.W = md.R + 1;  // components of the transfer by magnitude (see ModelDev)
      const double L = M->params[0], e_sq = M->params[1];
      vq.assign((size_t)md.W * md.W * md.W, 0.0);
      for (int dx = 0; dx <= md.R; dx++)
        for (int dy = 0; dy <= md.R; dy++)
          for (int dz = 0; dz <= md.R; dz++) {
            const int d[3] = {dx, dy, dz};
            const double prefactor = e_sq / (L * L * L);
            double rel = 0.0, mu = 0.0;
            for (int i = 0; i < 3; i++) {
              const double term = 2 * M_PI * d[i] / L;
              rel += term * term;
            }
            const double v = rel < 1.e-5 ? 0.0 : prefactor * 4 * M_PI / (rel + mu * mu);
            vq[((size_t)dx * md.W + dy) * md.W + dz] = v;
          }
      if (nmax <= 63) {
        ocode.resize(nsp);
        for (uint64_t o = 0; o < nsp; o++) {
          const int32_t *q = M->qn + o * M->qn_stride;
          ocode[o] = (uint32_t)(q[0] + 64) | ((uint32_t)(q[1] + 64) << 8) |
                     ((uint32_t)(q[2] + 64) << 16) | ((uint32_t)(q[3] & 0xff) << 24);
        }
      }
    }
    Arena mr;
    mr.add(&d_qn, (size_t)nsp * M->qn_stride);
    mr.add(&d_vq, vq.size());
    mr.add(&d_ocode, ocode.size());
    mr.add(&h->eps_io, 2 * nsp + 1);
    TRY(mr.commit(h));
    batch.push_back(UploadPiece{reinterpret_cast<char *>(d_qn),
                                reinterpret_cast<const char *>(M->qn),
                                (size_t)nsp * M->qn_stride * sizeof(int32_t)});
    batch.push_back(UploadPiece{reinterpret_cast<char *>(d_vq),
                                reinterpret_cast<const char *>(vq.data()), vq.size() * 8});
    batch.push_back(UploadPiece{reinterpret_cast<char *>(d_ocode),
                                reinterpret_cast<const char *>(ocode.data()), ocode.size() * 4});
    md.qn = d_qn;
    md.vq = d_vq;
    md.ocode = ocode.empty() ? nullptr : d_ocode;
    h->md = md;
    h->has_model = true;
  }
  const size_t n_allocs = h->allocs.size();
  TRY(sc.commit(h));

  // The host lists go up together with the model's (copy_pieces_to_device below); they stay
  // alive until then.
  auto put = [&](auto *dst, const auto &v) -> int {
    if (!v.empty())
      batch.push_back(UploadPiece{reinterpret_cast<char *>(dst),
                                  reinterpret_cast<const char *>(v.data()),
                                  v.size() * sizeof(v[0])});
    return CCDGPU_OK;
  };
  TRY(put(h->chans, chans)); TRY(put(h->mods, mods));
  TRY(put(h->hh_tiles, hh_tiles)); TRY(put(h->hh_red, hh_red)); TRY(put(h->ranges, ranges)); TRY(put(h->quad_items, quad_items));
  TRY(put(h->quad_cols, quad_cols));

  TRY(put(h->kcol, kcol));
  if (h->tc_gen) {
    TRY(put(h->vg_rows, vg_rows)); TRY(put(h->vg_cols, vg_cols)); TRY(put(h->vg_tab, vg_tab));
  }
  TRY(put(h->pp_pairs, pp_pairs)); TRY(put(h->hh_pairs, hh_pairs));
  TRY(put(h->pp_swap, pp_swap)); TRY(put(h->hh_swap, hh_swap));
  TRY(put(h->list_off, list_off)); TRY(put(h->list, list));
  TRY(put(h->rowmap, rowmap)); TRY(put(h->mirror, mirror)); TRY(put(h->pk_idx, pk_idx));
  TRY(put(h->o_h, o_h)); TRY(put(h->o_p, o_p));
  TRY(put(d_vrows, vrows)); TRY(put(d_vraw_off, vraw_off));
  TRY(put(d_gv_items, gv_items)); TRY(put(d_gvt_items, gvt_items));
  TRY(put(d_mod_dims, mod_dims)); TRY(put(d_o_m, o_m));
  batch.push_back(UploadPiece{reinterpret_cast<char *>(h->eps),
                              reinterpret_cast<const char *>(P->sp_energy), nsp * 8});

  // V blocks and tables, uploaded in their reference layouts (runs of adjacent blocks).
  {
    std::vector<const double *> sp, sx, sh;
    std::vector<int64_t> np2, nx, nh;
    std::vector<const ccdgpu_chain_index *> sm[8];
    std::vector<int64_t> nm;
    for (size_t ai = 0; ai < chans.size(); ai++) {
      const uint64_t c = act_chan[ai];
      const ChanInfo &a = chans[ai];
      if ((!on_the_fly && !P->v_pppp[c]) || (!gen_v && (!P->v_hhpp[c] || !P->v_hhhh[c])))
        return CCDGPU_ERR_INVALID_ARGUMENT;
      if (!on_the_fly)  // the rows a <= b of V_pppp, the only ones the ladder reads
        for (int u = 0; u < a.pr; u++) {
          sp.push_back(P->v_pppp[c] + (int64_t)rowmap[a.row_off + u] * a.pp);
          np2.push_back(a.pp);
        }
      if (!gen_v) {
        sx.push_back(P->v_hhpp[c]); nx.push_back((int64_t)a.pp * a.hh);
        sh.push_back(P->v_hhhh[c]); nh.push_back((int64_t)a.hh * a.hh);
      }
      for (int k = 0; k < 8 && !derive_tables; k++) {
        if (!P->maps[k][c]) return CCDGPU_ERR_INVALID_ARGUMENT;
        sm[k].push_back(P->maps[k][c]);
      }
      nm.push_back((int64_t)a.pp * a.hh);
    }
    TRY(upload_runs(h, vraw, sp, np2));
    TRY(upload_runs(h, hhpp_raw, sx, nx));
    TRY(upload_runs(h, h->v_hhhh, sh, nh));
    static_assert(sizeof(RawIndex) == sizeof(ccdgpu_chain_index), "ChainIndex layout");
    for (int k = 0; k < 8 && !derive_tables; k++)
      TRY(upload_runs(h, reinterpret_cast<ccdgpu_chain_index *>(raw_idx) + (size_t)k * n_t, sm[k], nm));
    if (derive_tables && !mlook_dev) TRY(put(d_mlook, mlook));
    if (gen_v) {
      TRY(put(d_mod_gen, mod_gen));
      TRY(put(d_mod_ph, mod_ph));
      TRY(put(d_mod_hp, mod_hp));
      TRY(put(d_mod_chan, mod_gen_chan));
    }
    TRY(upload_runs(h, hpph_raw, src_hpph, cnt_hpph));
    TRY(upload_runs(h, h->v_hphp, src_hphp, cnt_hphp));
    if (h->have_3body && !gen_v3) {
      std::vector<const double *> s5, s6;
      std::vector<int64_t> n5, n6;
      for (uint64_t k = 0; k < np; k++) {
        const int64_t n = o_h[k + 1] - o_h[k];
        if (n && !P->v_h_hpp[k]) return CCDGPU_ERR_INVALID_ARGUMENT;
        s5.push_back(P->v_h_hpp[k]); n5.push_back(n);
      }
      for (uint64_t a = 0; a < h->npart; a++) {
        const int64_t n = o_p[a + 1] - o_p[a];
        if (n && !P->v_phh_p[a]) return CCDGPU_ERR_INVALID_ARGUMENT;
        s6.push_back(P->v_phh_p[a]); n6.push_back(n);
      }
      TRY(upload_runs(h, h->v_h_hpp, s5, n5));
      TRY(upload_runs(h, h->v_phh_p, s6, n6));
    }
    // The last use of the staging buffers in create: the lists' copies stay in flight (the
    // staging lock is held until the set-up's final synchronisation).
    TRY(copy_pieces_to_device(h, batch, &staging_hold));
  }
  // Device layout transforms.
  h->create_ms[1] = ms_since(t_build) - h->create_ms[0];
  if (h->n_quad_rows) {
    quad_rows_kernel<<<(unsigned)h->n_act, 256, 0, h->s0>>>(h->chans, h->rowmap, h->mirror,
                                                           h->pk_idx, h->pp_pairs, h->eps,
                                                           (int)np, h->quad_rows);
    CK(cudaGetLastError());
  }
  if (gen_v && !mod_gen.empty()) {
    gen_v_mod_kernel<<<(unsigned)mod_gen.size(), 256, 0, h->s0>>>(d_mod_gen, d_mod_ph, d_mod_hp,
                                                                 md, h->v_hpph, h->v_hphp);
    CK(cudaGetLastError());
  } else if (h->n_mod) {
    transpose_hpph_kernel<<<h->n_mod, 256, 0, h->s0>>>(h->mods, hpph_raw, h->v_hpph);
    CK(cudaGetLastError());
  }
  if (h->n_ranges) {
    if (gen_v) {
      gen_v_pphh_kernel<<<h->n_ranges, 256, 0, h->s0>>>(h->ranges, h->chans, h->pp_pairs,
                                                        h->hh_pairs, md, h->v_pphh);
      CK(cudaGetLastError());
      gen_v_hhhh_kernel<<<(unsigned)chans.size(), 256, 0, h->s0>>>(h->chans, h->hh_pairs, md,
                                                                   h->v_hhhh);
    } else {
      transpose_hhpp_kernel<<<h->n_ranges, 256, 0, h->s0>>>(h->ranges, h->chans, hhpp_raw,
                                                            h->v_pphh);
    }
    CK(cudaGetLastError());
    if (derive_tables || gen_v3) {
      pair_sizes_kernel<<<(unsigned)chans.size(), 256, 0, h->s0>>>(
          h->chans, h->pp_pairs, h->hh_pairs, (int)np, (int)h->npart, d_hblk, d_pblk);
      CK(cudaGetLastError());
      row_scan_kernel<<<(unsigned)np, 256, 0, h->s0>>>(d_hblk, (int)np);
      CK(cudaGetLastError());
      row_scan_kernel<<<(unsigned)h->npart, 256, 0, h->s0>>>(d_pblk, (int)h->npart);
      CK(cudaGetLastError());
    }
    if (gen_v3) {
      gen_v3_kernel<<<(unsigned)chans.size(), 256, 0, h->s0>>>(
          h->chans, h->pp_pairs, h->hh_pairs, md, h->o_h, h->o_p, d_hblk, d_pblk, (int)np,
          (int)h->npart, h->v_h_hpp, h->v_phh_p, h->err);
      CK(cudaGetLastError());
    }
    if (mlook_dev) {
      CK(cudaMemsetAsync(d_mlook, 0xff, n_mlook * sizeof(int4), h->s0));  // every field -1
      if (!mod_gen.empty()) {
        mod_lookup_kernel<<<(unsigned)mod_gen.size(), 128, 0, h->s0>>>(
            d_mod_gen, d_mod_chan, d_mod_ph, d_mod_hp, (int)np, d_mlook, h->err);
        CK(cudaGetLastError());
      }
    }
    if (derive_tables) {
      DeriveGeometry dg{h->o_h, h->o_p, d_o_m, d_mod_dims, d_hblk, d_pblk, d_mlook,
                        (int32_t)np, (int32_t)h->npart};
      derive_tables_kernel<<<h->n_ranges, 256, 0, h->s0>>>(h->ranges, h->chans, h->pp_pairs,
                                                           h->hh_pairs, dg, n_t, h->flat, counts,
                                                           h->err);
    } else {
      TableGeometry geo{h->o_h, h->o_p, d_o_m, d_mod_dims, nch, np, h->npart};
      convert_tables_kernel<<<h->n_ranges, 256, 0, h->s0>>>(h->ranges, raw_idx, n_t, geo,
                                                            h->flat, counts, h->err);
    }
    CK(cudaGetLastError());
    const int nb = (int)std::min<int64_t>(ceil_div(5 * n_t, 256), 148 * 32);
    check_counts_kernel<<<std::max(nb, 1), 256, 0, h->s0>>>(counts, 5 * n_t, h->err);
    CK(cudaGetLastError());
    ring_maps_kernel<<<h->n_ranges, 256, 0, h->s0>>>(h->ranges, h->chans, h->pp_swap, h->hh_swap,
                                                     h->flat, n_t, h->inv4, h->err);
    CK(cudaGetLastError());
  }
  if (a_row_off[n_act] > 0) {
    if (on_the_fly) {
      // FP64 tiles, and the bf16 images unless the tensor-core ladder generates its own V: one
      // CTA per image chunk; with bf16 images, one CTA per tensor-core chunk writes both.
      if (!gv_items.empty()) {
        auto kern64 = md.ocode ? gen_v_chunks_kernel<true> : gen_v_chunks_kernel<false>;
        kern64<<<(unsigned)gv_items.size(), 256, 0, h->s0>>>(
            h->chans, d_gv_items, h->rowmap, h->kcol, h->pp_pairs, md, h->v_t);
        CK(cudaGetLastError());
      }
      if (h->nt && !h->tc_gen && !gvt_items.empty()) {
        auto kern = md.ocode ? (h->nt == 3 ? gen_v_both_chunks_kernel<3, true>
                                           : gen_v_both_chunks_kernel<2, true>)
                             : (h->nt == 3 ? gen_v_both_chunks_kernel<3, false>
                                           : gen_v_both_chunks_kernel<2, false>);
        kern<<<(unsigned)gvt_items.size(), 256, 0, h->s0>>>(h->chans, d_gvt_items, h->rowmap,
                                                           h->kcol, h->pp_pairs, md, h->v_t,
                                                           h->v_tc, h->n_vtc);
      }
    } else {
      tile_v_kernel<<<(unsigned)vrows.size(), 128, 0, h->s0>>>(h->chans, d_vrows, h->rowmap,
                                                               h->kcol, d_vraw_off, vraw, h->v_t);
    }
    CK(cudaGetLastError());
    if (h->nt && !on_the_fly) {
      tile_v_tc_kernel<<<(unsigned)vrows.size(), 128, 0, h->s0>>>(
          h->chans, d_vrows, h->rowmap, h->kcol, d_vraw_off, vraw, h->v_tc, h->n_vtc, h->nt);
      CK(cudaGetLastError());
    }
  }
  // Host work that needs no result of the set-up kernels runs while they do: kernel
  // attributes, the ladder schedules and, for device-loop handles, the loop graph's capture
  // (nothing of it executes until a solve launches it).  Then the set-up's error word is read.
  const auto t_sched = std::chrono::steady_clock::now();
#undef TRY
  h->h_ctl = ctl_acquire();
  if (!h->h_ctl) return CCDGPU_ERR_OUT_OF_MEMORY;

  h->ladder_smem = (size_t)kStages * (kMaxAS * kBK + kBK * kMaxBS) * 8 + 2 * kStages * 8;
  h->ladder_smem_thin = (size_t)kStages * (kMaxAS * kBK + kBK * 8) * 8 + 2 * kStages * 8;
  CK(cudaFuncSetAttribute(pp_ladder_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)h->ladder_smem_thin));
  CK(cudaFuncSetAttribute(pp_ladder_kernel<0>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  CK(cudaFuncSetAttribute(pp_ladder_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)h->ladder_smem));
  CK(cudaFuncSetAttribute(pp_ladder_kernel<1>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  CK(cudaFuncSetAttribute(pp_ladder_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)h->ladder_smem));
  CK(cudaFuncSetAttribute(pp_ladder_kernel<2>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  h->hh_smem = 0;  // static shared memory only
  // The attribute belongs to the kernel, not to this handle: set the device's opt-in maximum
  // (the same value for every handle), so that handles of different channel sizes coexist.
  int smem_optin = 0;
  CK(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->opt.device));
  if (ring16_smem(80) > (size_t)smem_optin) return CCDGPU_ERR_UNSUPPORTED;
  CK(cudaFuncSetAttribute(hh_slice_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)hh_slice_smem(8 * kMaxCG)));
  CK(cudaFuncSetAttribute(ring16_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)ring16_smem(32)));
  CK(cudaFuncSetAttribute(ring16_kernel<48>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)ring16_smem(48)));
  CK(cudaFuncSetAttribute(ring16_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)ring16_smem(64)));
  CK(cudaFuncSetAttribute(ring16_kernel<80>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)ring16_smem(80)));
  ccdgpu_schedule sch{};
  sch.thin_split_mul = 1;
  sch.wide_split_mul = 3;
  sch.tc_split_mul = 2;
  if (int rc2 = make_ladder_tiles(h, sch)) return rc2;
  if (h->nt) {
    h->tc_smem = tc_smem_bytes(h->nt);
    CK(cudaFuncSetAttribute(tc_kernel_of(h->nt, h->tc_gen),
                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->tc_smem));
  }
  if (h->opt.path == CCDGPU_PATH_FUSED && h->opt.use_graph && h->opt.device_loop) {
    ready_loop_graphs(h);
    if (h->loop_state != 1) h->loop_state = 0;  // retried by the first solve, on an idle stream
  }
  h->create_ms[3] = ms_since(t_sched);
  int32_t e = 0;
  CK(cudaMemcpyAsync(&e, h->err, sizeof(e), cudaMemcpyDeviceToHost, h->s0));
  CK(cudaStreamSynchronize(h->s0));
  h->create_ms[2] = ms_since(t_build) - h->create_ms[0] - h->create_ms[1];
  // Release the scratch allocation.
  for (size_t i = n_allocs; i < h->allocs.size(); i++) dev_free(h->allocs[i].p, h->allocs[i].bytes);
  h->allocs.resize(n_allocs);
  if (e & kErrBadIndex) return CCDGPU_ERR_BAD_TABLE;
  // The fused path relies on the structure of the ring tables; the table path does not.
  if ((e & kErrRingMaps) && h->opt.path == CCDGPU_PATH_FUSED) return CCDGPU_ERR_BAD_TABLE;
  if (e & ~kErrRingMaps) return CCDGPU_ERR_CUDA;
  if (e) CK(cudaMemsetAsync(h->err, 0, sizeof(int32_t), h->s0));
  return CCDGPU_OK;
}

// ---- launches -------------------------------------------------------------------------

// Launch with the programmatic-stream-serialization attribute (PDL): the kernel may begin
// launching while its stream predecessor drains; it waits in griddepcontrol.wait before
// touching the predecessor's results (skip_iteration / pdl_enter in every kernel).
thread_local bool t_pdl = true;  // cleared while retrying a loop-graph capture without PDL

template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), unsigned grid, unsigned block, size_t smem,
                       cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = t_pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// gate: 0 = kernel of an FP64 iteration, 1 = of a mixed-precision iteration (which also writes
// the bf16 operand images of the tensor-core ladder).
// only: -1 everything, 0 units of hh <= 16, 1 the other units (2: neither); the reduction
// runs when only < 0.
int launch_hh_ladder(ccdgpu_handle *h, cudaStream_t st, int gate, int only = -1) {
  const int nt = gate ? h->nt : 0;
  if (h->n_hh_small && only <= 0) {
    h->launches++;
    CK(launch_pdl(hh_mma_kernel<2>, (int)ceil_div(h->n_hh_small, kHHWarps), kHHWarps * 32, 0, st,
                  (const HHTile *)h->hh_tiles, h->n_hh_small, (const ChanInfo *)h->chans,
                  (const double *)h->v_pphh, (const double *)h->t[0], (const double *)h->t[1],
                  h->part, h->r, (const Control *)h->ctl, gate));
  }
  const int nbig = h->n_hh_tiles - h->n_hh_small;
  if (nbig && (only < 0 || only == 1)) {
    h->launches++;
    CK(launch_pdl(hh_slice_kernel, nbig, kHHSliceThreads, h->hh_slice_smem, st,
                  (const HHTile *)(h->hh_tiles + h->n_hh_small), (const ChanInfo *)h->chans,
                  (const double *)h->v_pphh, (const double *)h->t[0], (const double *)h->t[1],
                  h->part, h->r, (const Control *)h->ctl, gate));
  }
  if (h->n_hh_red && (only < 0 || only == 2)) {
    h->launches++;
    CK(launch_pdl(hh_reduce_kernel, h->n_hh_red, 256, 0, st, (const HHRed *)h->hh_red,
                  (const ChanInfo *)h->chans, (const double *)h->v_hhhh, (const double *)h->part,
                  h->x, h->x_t, h->s, h->xt_tc, h->n_xttc, nt, (const Control *)h->ctl, gate));
  }
  return CCDGPU_OK;
}
int launch_pp_ladder_tc(ccdgpu_handle *h, cudaStream_t st) {
  if (!h->n_tc_tiles) return CCDGPU_OK;
  h->launches++;
  // Persistent: two CTAs per SM (shared memory and 2 x 128 tensor-memory columns each).
  CK(launch_pdl(tc_kernel_of(h->nt, h->tc_gen), h->tc_grid, tc_threads(h->tc_gen), h->tc_smem,
                st, (const LadderTile *)h->tc_tiles, h->n_tc_tiles, h->tc_sched,
                (const __nv_bfloat16 *)h->v_tc, h->n_vtc, (const __nv_bfloat16 *)h->tkt_tc,
                h->n_tkttc, (const __nv_bfloat16 *)h->tmt_tc, h->n_tmttc,
                (const __nv_bfloat16 *)h->xt_tc, h->n_xttc, (const int32_t *)h->rowmap,
                (const int32_t *)h->mirror, h->dmat, h->tc_part, (const Control *)h->ctl, h->err,
                (const ChanInfo *)h->chans, (const VGenRow *)h->vg_rows,
                (const uint32_t *)h->vg_cols, (const double *)h->vg_tab));
  if (h->n_red_tc) {
    CK(launch_pdl(ladder_reduce_kernel, h->n_red_tc, 256, 0, st, (const RedItem *)h->red_tc,
                  (const LadderTile *)h->tc_tiles, (const int32_t *)h->rowmap,
                  (const int32_t *)h->mirror, h->dmat, (const double *)h->tc_part,
                  (const Control *)h->ctl, 1));
    h->launches++;
  }
  return CCDGPU_OK;
}
// The three column classes run concurrently: mid and wide go to stream s2 (wide first, they
// are the longest tiles), thin to `st`; s2 is joined back into `st` before returning.
int launch_pp_ladder(ccdgpu_handle *h, cudaStream_t st) {
  if (h->nt && h->n_ranges) {
    // A mixed handle's FP64 ladder first refreshes its operand tiles if mixed iterations ran.
    CK(launch_pdl(retile_kernel, h->n_ranges, 256, 0, st, (const ElemRange *)h->ranges,
                  (const ChanInfo *)h->chans, (const int2 *)h->pk_idx, (const double *)h->t[0],
                  (const double *)h->t[1], h->t_kt, h->t_mt, h->ctl, 0));
    CK(launch_pdl(retile_done_kernel, 1, 32, 0, st, h->ctl));
    h->launches += 2;
  }
  // The classes run one after another on `st`: each is persistent over every SM (its tiles
  // balanced for CTAs that all start together), so concurrent classes only delay each other's
  // CTAs.
  cudaStream_t s2 = st;
  if (h->n_cls[1] || h->n_cls[2]) {
    if (h->n_cls[2]) {
      pp_ladder_kernel<2><<<h->fp_grid[2], ladder_threads(2), h->ladder_smem, s2>>>(
          h->tiles, h->fp_cta_off + h->fp_off_base[2], h->v_t, h->t_kt, h->t_mt, h->x_t,
          h->rowmap, h->mirror, h->dmat, h->lpart, h->ctl, h->err, 0);
      h->launches++;
      CK(cudaGetLastError());
    }
    if (h->n_cls[1]) {
      pp_ladder_kernel<1><<<h->fp_grid[1], ladder_threads(1), h->ladder_smem, s2>>>(
          h->tiles, h->fp_cta_off + h->fp_off_base[1], h->v_t, h->t_kt, h->t_mt, h->x_t,
          h->rowmap, h->mirror, h->dmat, h->lpart, h->ctl, h->err, 0);
      h->launches++;
      CK(cudaGetLastError());
    }
  }
  if (h->n_cls[0]) {
    CK(launch_pdl(pp_ladder_kernel<0>, h->fp_grid[0], kLadderThreads, h->ladder_smem_thin, st,
                  (const LadderTile *)h->tiles, (const int32_t *)(h->fp_cta_off + h->fp_off_base[0]),
                  (const double *)h->v_t, (const double *)h->t_kt, (const double *)h->t_mt,
                  (const double *)h->x_t, (const int32_t *)h->rowmap, (const int32_t *)h->mirror,
                  h->dmat, h->lpart, (const Control *)h->ctl, h->err, 0));
    h->launches++;
  }
  if (h->n_red_fp) {
    CK(launch_pdl(ladder_reduce_kernel, h->n_red_fp, 256, 0, st, (const RedItem *)h->red_fp,
                  (const LadderTile *)h->tiles, (const int32_t *)h->rowmap,
                  (const int32_t *)h->mirror, h->dmat, (const double *)h->lpart,
                  (const Control *)h->ctl, 0));
    h->launches++;
  }
  return CCDGPU_OK;
}

// T' from the phhp slab in both paths.  fused: R scattered into pphh order for the fused
// assembly; else the table path's t2Diff_phhp slab.
// only: -1 every class, else 0 small, 1 mid, 2 large.
int launch_phhp_gather(ccdgpu_handle *h, cudaStream_t st, int gate) {
  if (!h->n_m) return CCDGPU_OK;
  h->launches++;
  const unsigned blocks = (unsigned)ceil_div(h->n_m, (int64_t)256 * kGatherPer);
  return cuda_status(launch_pdl(phhp_gather_kernel, blocks, 256, 0, st, (const int32_t *)h->inv4,
                                h->n_m, (const double *)h->t[0], (const double *)h->t[1],
                                h->old_phhp, (const Control *)h->ctl, gate));
}
int launch_ring(ccdgpu_handle *h, cudaStream_t st, int gate, bool fused, int only = -1) {
  const int32_t *inv = fused ? h->inv4 : nullptr;
  double *out = fused ? h->d_ring : h->r_phhp;
  // Fused path: T' (the phhp slab) gathered from the current amplitudes first; the profile's
  // small class includes it.
  if (fused && (only < 0 || only == 0))
    if (int rc = launch_phhp_gather(h, st, gate)) return rc;
  if (h->n_mod_small && (only < 0 || only == 0)) {
    CK(launch_pdl(ring_small_kernel, (int)ceil_div(h->n_mod_small, kRingSmallWarps),
                  kRingSmallWarps * 32, 0, st, (const ModInfo *)h->mods, h->n_mod_small,
                  (const double *)h->v_hpph, (const double *)h->v_hphp,
                  (const double *)h->old_phhp, inv, out, (const Control *)h->ctl, gate));
    h->launches++;
  }
  // Groups by padded size; only = 1 launches the 32 group, only = 2 the wider ones.
  const ModInfo *mp = h->mods + h->n_mod_small;
  for (int k = 0; k < 4; k++) {
    const int n = h->n_mod_pad[k];
    if (n && (only < 0 || only == (k == 0 ? 1 : 2))) {
      auto go = [&](auto kern, int pad) {
        return launch_pdl(kern, n, 32 * ring16_warps(pad), ring16_smem(pad), st, mp,
                          (const double *)h->v_hpph, (const double *)h->v_hphp,
                          (const double *)h->old_phhp, inv, out, (const Control *)h->ctl, gate);
      };
      switch (k) {
        case 0: CK(go(ring16_kernel<32>, 32)); break;
        case 1: CK(go(ring16_kernel<48>, 48)); break;
        case 2: CK(go(ring16_kernel<64>, 64)); break;
        default: CK(go(ring16_kernel<80>, 80)); break;
      }
      h->launches++;
    }
    mp += n;
  }
  return CCDGPU_OK;
}
int launch_onebody_fused(ccdgpu_handle *h, cudaStream_t st, int gate) {
  const int warps_per_block = 8;
  const int blocks = (int)ceil_div((int64_t)h->nsp, warps_per_block);
  h->launches++;
  return cuda_status(launch_pdl(onebody_fused_kernel, blocks, warps_per_block * 32, 0, st,
                                (int)h->np, (int)h->nsp, h->list_off, h->list, h->s, h->r, h->xh,
                                h->yp, h->ctl, gate));
}
int launch_assemble_fused(ccdgpu_handle *h, cudaStream_t st, int gate) {
  if (!h->n_asm_blocks) return CCDGPU_OK;
  h->launches++;
  return cuda_status(launch_pdl(
      h->loop_capture ? assemble_fused_kernel<true> : assemble_fused_kernel<false>,
      h->n_asm_blocks, kAsmThreads, 0, st, (const QuadItem *)h->quad_items, h->n_quad_items,
      (const ChanInfo *)h->chans, (const QuadRow *)h->quad_rows,
      (const QuadCol *)h->quad_cols, (const double *)h->v_pphh, (const double *)h->dmat,
      (const double *)h->d_ring, (const double *)h->xh, (const double *)h->yp, h->t[0], h->t[1], h->t_kt, h->t_mt, h->epart,
      h->ticket, h->ctl, h->tkt_tc, h->n_tkttc, h->tmt_tc, h->n_tmttc, gate ? h->nt : 0,
      (cudaGraphConditionalHandle)(h->loop_capture ? h->loop_cond : 0), h->loop_capture, gate));
}
int launch_energy(ccdgpu_handle *h, cudaStream_t st, int flags) {
  energy_kernel<<<1, kEnergyThreads, 0, st>>>(h->epart, h->n_ranges, h->ctl, flags, h->e_out, 0);
  h->launches++;
  return cuda_status(cudaGetLastError());
}
int launch_map_to(ccdgpu_handle *h, cudaStream_t st, const double *src, double *dst) {
  if (!h->n_ranges) return CCDGPU_OK;
  map_to_kernel<<<h->n_ranges, 256, 0, st>>>(h->ranges, h->chans, h->pk_idx, h->flat, h->n_t, src, dst,
                                               h->old_h2pp_h1, h->old_h1pp_h2, h->old_p1_p2hh,
                                               h->old_p2_p1hh, h->old_phhp, h->t_kt, h->t_mt,
                                               h->have_3body ? 1 : 0, h->tkt_tc, h->n_tkttc,
                                               h->tmt_tc, h->n_tmttc, h->nt);
  h->launches++;
  return cuda_status(cudaGetLastError());
}

// One fused iteration: ring on s1 beside hh ladder, one-body sums and pp ladder on s0, then the
// assembly.
// mixed: the pp ladder runs on the tensor cores (split bf16) instead of the FP64 pipe.
int enqueue_fused_iteration(ccdgpu_handle *h, bool mixed) {
  int rc;
  const int gate = mixed ? 1 : 0;
  auto ladder = [&](cudaStream_t st) {
    return mixed ? launch_pp_ladder_tc(h, st) : launch_pp_ladder(h, st);
  };
  if (h->profiling) {
    // ev: 0 start, 1 after hh ladder, 2 after one-body, 3 after pp ladder, 4/5 ring on s1,
    // 6 after assembly, 7 after the energy reduction.
    CK(cudaEventRecord(h->ev[0], h->s0));
    CK(cudaStreamWaitEvent(h->s1, h->ev[0], 0));
    CK(cudaEventRecord(h->ev[4], h->s1));
    if ((rc = launch_ring(h, h->s1, gate, true))) return rc;
    CK(cudaEventRecord(h->ev[5], h->s1));
    if ((rc = launch_hh_ladder(h, h->s0, gate))) return rc;
    CK(cudaEventRecord(h->ev[1], h->s0));
    if ((rc = launch_onebody_fused(h, h->s0, gate))) return rc;
    CK(cudaEventRecord(h->ev[2], h->s0));
    if ((rc = ladder(h->s0))) return rc;
    CK(cudaEventRecord(h->ev[3], h->s0));
    CK(cudaStreamWaitEvent(h->s0, h->ev[5], 0));
    CK(cudaEventRecord(h->ev[8], h->s0));
    if ((rc = launch_assemble_fused(h, h->s0, gate))) return rc;
    CK(cudaEventRecord(h->ev[6], h->s0));
    CK(cudaEventRecord(h->ev[7], h->s0));
    return CCDGPU_OK;
  }
  // The ring (s1) runs beside the hh ladder, the one-body sums and the pp ladder (s0); the
  // latency-bound small ring channels fill SMs the hh ladder leaves idle.  The one-body sums
  // stay on s0 ahead of the pp ladder: on a third stream their CTAs delayed the start of the
  // persistent ladder's CTAs (device trace).
  CK(cudaEventRecord(h->ev_fork, h->s0));
  CK(cudaStreamWaitEvent(h->s1, h->ev_fork, 0));
  if ((rc = launch_ring(h, h->s1, gate, true))) return rc;
  CK(cudaEventRecord(h->ev_join, h->s1));
  if ((rc = launch_hh_ladder(h, h->s0, gate))) return rc;
  // FP64 iterations: the one-body sums (read only by the assembly) run on s3 beside the FP64
  // ladder classes (FP64 iteration 2,836 -> 2,952 iter/s at EG N=54 |n|^2<=36).  Mixed
  // iterations keep them on s0 ahead of the tensor-core ladder (3,925 against 3,900 iter/s
  // beside it).
  cudaStream_t ob = mixed ? h->s0 : h->s3;
  if (!mixed) {
    CK(cudaEventRecord(h->ev_fork3, h->s0));
    CK(cudaStreamWaitEvent(h->s3, h->ev_fork3, 0));
  }
  if ((rc = launch_onebody_fused(h, ob, gate))) return rc;
  if (!mixed) CK(cudaEventRecord(h->ev_join3, h->s3));
  if ((rc = ladder(h->s0))) return rc;
  if (!mixed) CK(cudaStreamWaitEvent(h->s0, h->ev_join3, 0));
  CK(cudaStreamWaitEvent(h->s0, h->ev_join, 0));
  if ((rc = launch_assemble_fused(h, h->s0, gate))) return rc;  // + energy and stop rule
  if (h->loop_capture && !h->n_asm_blocks) {  // else the assembly set the loop condition
    h->launches++;
    CK(launch_pdl(loop_ctl_kernel, 1, 32, 0, h->s0, (const Control *)h->ctl, h->loop_cond,
                  h->loop_capture == 2 ? 1 : 0));
  }
  return CCDGPU_OK;
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
  if (e & kErrTimeout) {
    // Reported once: the handle stays usable (the timed-out iteration's amplitudes are
    // incomplete; ccdgpu_reset or ccdgpu_set_t2 starts over).  A tensor-core ladder CTA that
    // gave up may have left the tile counter and exit ticket behind: zero them for the next
    // launch.
    CK(cudaMemset(h->err, 0, sizeof(int32_t)));
    if (h->tc_sched) CK(cudaMemset(h->tc_sched, 0, 2 * sizeof(int32_t)));
    return CCDGPU_ERR_TIMEOUT;
  }
  if (h->h_ctl->error & kErrNonFinite) return CCDGPU_ERR_NONFINITE;
  return CCDGPU_OK;
}

int set_ctl(ccdgpu_handle *h, int active, double tol, int64_t max_iters, double mixing,
            bool reset_loop, int parity = -1, int phase = 0) {
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
    c.polish_iters = 0;
    std::memset(c.energies, 0, sizeof(c.energies));
  }
  c.phase = phase;
  c.polish_rel = h->opt.polish_threshold;
  c.active = active;
  c.tol = tol;
  c.max_iters = max_iters;
  c.mixing = mixing;
  CK(cudaMemcpyAsync(h->ctl, h->h_ctl, sizeof(Control), cudaMemcpyHostToDevice, h->s0));
  CK(cudaStreamSynchronize(h->s0));
  return CCDGPU_OK;
}

// The Control block of a new handle in one upload: what set_ctl(h, 0, 0.0, 100, 0.5, true)
// and ccdgpu_trace_arm(h, -1) would write over the zeroed device copy.
int init_ctl(ccdgpu_handle *h) {
  Control &c = *h->h_ctl;
  std::memset(&c, 0, sizeof(Control));
  c.e_prev = 100.0;
  c.e_diff = 1.0;
  c.polish_rel = h->opt.polish_threshold;
  c.max_iters = 100;
  c.mixing = 0.5;
  c.trace_iter = -1;
  for (int k = 0; k < kTraceKernels; k++) c.trace_first[k] = ~0ull;
  CK(cudaMemcpyAsync(h->ctl, h->h_ctl, sizeof(Control), cudaMemcpyHostToDevice, h->s0));
  CK(cudaStreamSynchronize(h->s0));
  return CCDGPU_OK;
}

int fused_ready_graph(ccdgpu_handle *h, bool mixed) {
  cudaGraphExec_t &exec = mixed ? h->graph_tc : h->graph;
  if (exec) return CCDGPU_OK;
  cudaGraph_t g = nullptr;
  const int64_t before = h->launches;
  CK(cudaStreamBeginCapture(h->s0, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_fused_iteration(h, mixed);
  (mixed ? h->kernels_per_graph_tc : h->kernels_per_graph) = h->launches - before;
  h->launches = before;
  cudaError_t e = cudaStreamEndCapture(h->s0, &g);
  if (rc) { if (g) cudaGraphDestroy(g); return rc; }
  CK(e);
  e = cudaGraphInstantiate(&exec, g, 0);
  cudaGraphDestroy(g);
  CK(e);
  return CCDGPU_OK;
}

// The device solve loop.  Graph: [WHILE c_mix { mixed iteration }] -> WHILE c64 { FP64
// iteration }; each body ends with the fused assembly, whose stop-rule CTA sets the body's
// condition (loop_ctl_kernel when a system has no assembly blocks).  Both
// conditions default to 1 at every launch; one launch runs until the stop rule fires or
// ctl->stop_at is reached.
int capture_loop_graph(ccdgpu_handle *h, bool mixed, cudaGraphExec_t *exec) {
  cudaGraph_t g = nullptr;
  CK(cudaGraphCreate(&g, 0));
  cudaGraphNode_t prev = nullptr;
  int rc = CCDGPU_OK;
  const int64_t before = h->launches;
  for (int pass = mixed ? 0 : 1; pass < 2 && !rc; pass++) {
    const bool body_mixed = pass == 0;
    cudaGraphConditionalHandle cond = 0;
    cudaError_t e = cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = cond;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, prev ? &prev : nullptr, prev ? 1 : 0, &p);
    if (e == cudaSuccess)
      e = cudaStreamBeginCaptureToGraph(h->s0, p.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      rc = cuda_status(e);
      break;
    }
    h->loop_capture = body_mixed ? 2 : 1;
    h->loop_cond = cond;
    const int64_t b0 = h->launches;
    rc = enqueue_fused_iteration(h, body_mixed);
    (body_mixed ? h->kernels_per_body_tc : h->kernels_per_body64) = h->launches - b0;
    h->loop_capture = 0;
    cudaGraph_t body = nullptr;
    e = cudaStreamEndCapture(h->s0, &body);
    if (!rc && e != cudaSuccess) rc = cuda_status(e);
    (void)cudaGetLastError();
    prev = node;
  }
  h->launches = before;
  if (!rc) {
    cudaError_t e = cudaGraphInstantiate(exec, g, 0);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      *exec = nullptr;
      rc = cuda_status(e);
    }
  }
  cudaGraphDestroy(g);
  return rc;
}

// Builds the loop graph a solve starts with (loop_tc for mixed handles, loop64 otherwise)
// once; any failure (for example a driver without conditional nodes, or without programmatic
// launches inside them, retried without) leaves the batched replay.
void ready_loop_graphs(ccdgpu_handle *h) {
  if (h->loop_state) return;
  const auto t0 = std::chrono::steady_clock::now();
  for (int attempt = 0; attempt < 2 && h->loop_state == 0; attempt++) {
    t_pdl = attempt == 0;
    const int rc = h->nt ? capture_loop_graph(h, true, &h->loop_tc)
                         : capture_loop_graph(h, false, &h->loop64);
    if (!rc) {
      h->loop_state = 1;
      h->loop_pdl = t_pdl;
    } else {
      if (h->loop64) cudaGraphExecDestroy(h->loop64);
      if (h->loop_tc) cudaGraphExecDestroy(h->loop_tc);
      h->loop64 = h->loop_tc = nullptr;
    }
  }
  t_pdl = true;
  if (h->loop_state == 0) h->loop_state = -1;
  h->loop_graph_ms = ms_since(t0);
}

// One table-path iteration: exactly the reference loop body.
int tables_iteration(ccdgpu_handle *h, double mixing, double *corr) {
  int rc;
  if ((rc = stage_onebody_tables(h, 0, 1))) return rc;     // calcT2Diff_p2_p1hh
  if ((rc = stage_onebody_tables(h, 1, 0))) return rc;     // calcT2Diff_h2pp_h1
  if ((rc = launch_ring(h, h->s0, 0, false))) return rc;   // calcT2Diff_phhp
  if ((rc = launch_hh_ladder(h, h->s0, 0))) return rc;     // calcT2Diff_pphh
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
  opt->polish_threshold = 1e-6;
  opt->use_graph = 1;
  opt->device_loop = 1;
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
  const auto t_create = std::chrono::steady_clock::now();
  *out = nullptr;
  if (!prob->sp_energy || !prob->chan_dims || !prob->chan_mod_dims || !prob->chan_maps ||
      !prob->three_body_dims || prob->n_particles == 0 || prob->n_particles >= prob->n_sp)
    return CCDGPU_ERR_INVALID_ARGUMENT;
  ccdgpu_handle *h = new (std::nothrow) ccdgpu_handle();
  if (!h) return CCDGPU_ERR_OUT_OF_MEMORY;
  if (opt) h->opt = *opt;
  else ccdgpu_default_options(&h->opt);
  switch (h->opt.precision) {
    case CCDGPU_PREC_FP64: h->nt = 0; break;
    case CCDGPU_PREC_MIXED_BF16: h->nt = 2; break;
    case CCDGPU_PREC_MIXED_BF16X3: h->nt = 3; break;
    default: delete h; return CCDGPU_ERR_UNSUPPORTED;
  }
  if (h->nt && h->opt.path != CCDGPU_PATH_FUSED) { delete h; return CCDGPU_ERR_UNSUPPORTED; }
  if (h->nt && !(h->opt.polish_threshold >= 0)) { delete h; return CCDGPU_ERR_INVALID_ARGUMENT; }
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) { (void)cudaGetLastError(); delete h; return CCDGPU_ERR_NO_DEVICE; }
  if (h->opt.device < 0 || h->opt.device >= ndev) { delete h; return CCDGPU_ERR_INVALID_ARGUMENT; }
  int rc = cuda_status(cudaSetDevice(h->opt.device));
  if (!rc) rc = cuda_status(acquire_set(h->sset));
  if (!rc) {
    h->s0 = h->sset.s[0]; h->s1 = h->sset.s[1]; h->s2 = h->sset.s[2]; h->s3 = h->sset.s[3];
    for (int i = 0; i < 10; i++) h->ev[i] = h->sset.ev[i];
    h->ev_fork = h->sset.ev[10]; h->ev_join = h->sset.ev[11];
    h->ev_fork2 = h->sset.ev[12]; h->ev_join2 = h->sset.ev[13];
    h->ev_fork3 = h->sset.ev[14]; h->ev_join3 = h->sset.ev[15];
  }
  if (!rc) rc = build(h, prob);
  if (!rc) rc = init_ctl(h);
  if (rc) { release(h); delete h; return rc; }
  h->create_ms[4] = ms_since(t_create);
  *out = h;
  return CCDGPU_OK;
}

void ccdgpu_release_cached_memory(void) {
  release_cache(-1);
  release_stream_pool();
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
  const std::pair<double *, int64_t> z[] = {
      {h->t[0], h->n_t}, {h->t[1], h->n_t}, {h->old_phhp, h->n_m}, {h->t_kt, h->n_tkt},
      {h->t_mt, h->n_tmt}, {h->old_h1pp_h2, h->n_h}, {h->old_h2pp_h1, h->n_h},
      {h->old_p1_p2hh, h->n_p}, {h->old_p2_p1hh, h->n_p}};
  for (const auto &b : z)
    if (b.first && b.second) CK(cudaMemsetAsync(b.first, 0, b.second * 8, h->s0));
  if (h->nt) {
    CK(cudaMemsetAsync(h->tkt_tc, 0, (size_t)h->nt * h->n_tkttc * 2, h->s0));
    CK(cudaMemsetAsync(h->tmt_tc, 0, (size_t)h->nt * h->n_tmttc * 2, h->s0));
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

int ccdgpu_mbpt2(ccdgpu_handle *h, int32_t init_t2, double *e_mbpt2) {
  if (!h) return CCDGPU_ERR_INVALID_ARGUMENT;
  CK(cudaSetDevice(h->opt.device));
  int rc = set_ctl(h, 0, h->h_ctl->tol, h->h_ctl->max_iters, h->h_ctl->mixing, false);
  if (rc) return rc;
  if (init_t2) {
    // The amplitudes become the current ones (parity 0, as after ccdgpu_set_t2).
    h->h_ctl->parity = 0;
    CK(cudaMemcpyAsync(h->ctl, h->h_ctl, sizeof(Control), cudaMemcpyHostToDevice, h->s0));
  }
  if (h->n_ranges) {
    mbpt2_kernel<<<h->n_ranges, 256, 0, h->s0>>>(h->ranges, h->chans, h->pp_pairs, h->hh_pairs,
                                                  h->v_pphh, h->eps, init_t2 ? h->t[1] : nullptr,
                                                  h->epart);
    CK(cudaGetLastError());
  }
  if ((rc = launch_energy(h, h->s0, 0))) return rc;
  if (init_t2 && (rc = launch_map_to(h, h->s0, h->t[1], h->t[0]))) return rc;
  double e = 0.0;
  CK(cudaMemcpyAsync(&e, h->e_out, 8, cudaMemcpyDeviceToHost, h->s0));
  CK(cudaStreamSynchronize(h->s0));
  if (e_mbpt2) *e_mbpt2 = h->n_ranges ? e : 0.0;
  return check_errors(h);
}

int ccdgpu_reference_energy(ccdgpu_handle *h, const double *sp_energy_bare, double *e_ref,
                            double *sp_energy_normal) {
  if (!h || !sp_energy_bare || !e_ref) return CCDGPU_ERR_INVALID_ARGUMENT;
  if (!h->has_model) return CCDGPU_ERR_UNSUPPORTED;
  CK(cudaSetDevice(h->opt.device));
  const int nsp = (int)h->nsp;
  std::vector<double> out((size_t)nsp + 1);
  CK(cudaMemcpyAsync(h->eps_io, sp_energy_bare, (size_t)nsp * 8, cudaMemcpyHostToDevice, h->s0));
  normal_order_kernel<<<(nsp + 128) / 128, 128, 0, h->s0>>>(h->md, h->eps_io, nsp, (int)h->np,
                                                            h->eps_io + nsp);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out.data(), h->eps_io + nsp, out.size() * 8, cudaMemcpyDeviceToHost, h->s0));
  CK(cudaStreamSynchronize(h->s0));
  *e_ref = out[nsp];
  if (sp_energy_normal) std::copy(out.begin(), out.begin() + nsp, sp_energy_normal);
  return CCDGPU_OK;
}

int ccdgpu_build_channels(const ccdgpu_channel_rule *rule, ccdgpu_channel_dims *dims,
                          ccdgpu_channel_dims *mod_dims, ccdgpu_pair *const lists[4],
                          ccdgpu_pair *const mod_lists[4], uint32_t *chan, uint32_t *mod_chan,
                          uint32_t *pos, uint32_t *mod_pos) {
  if (!rule || !rule->qn || !dims || !mod_dims || !lists || !mod_lists) return CCDGPU_ERR_INVALID_ARGUMENT;
  const uint64_t nsp = rule->n_sp, np = rule->n_particles, nch = rule->n_channels;
  if (np == 0 || np >= nsp || nch == 0 || rule->kind < CCDGPU_MODEL_PAIRING ||
      rule->kind > CCDGPU_MODEL_ELECTRON_GAS ||
      rule->qn_stride < (rule->kind == CCDGPU_MODEL_PAIRING ? 2 : 5) || rule->nmax < 0)
    return CCDGPU_ERR_INVALID_ARGUMENT;
  if (nsp > 65535 || nch * 4 >= (uint64_t(1) << 31)) return CCDGPU_ERR_UNSUPPORTED;
  const uint64_t npart = nsp - np, n = nsp * nsp;
  const uint64_t tot[4] = {npart * npart, np * np, np * npart, npart * np};  // pp, hh, hp, ph
  for (int k = 0; k < 4; k++)
    if (!lists[k] || !mod_lists[k]) return CCDGPU_ERR_INVALID_ARGUMENT;
  if (rule->device >= 0) CK(cudaSetDevice(rule->device));
  cudaStream_t st = nullptr;
  CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  // One device block: qn, the per-pair arrays and the per-(channel, kind) arrays.
  size_t used = 0;
  auto take = [&](size_t bytes) {
    const size_t o = used;
    used += (bytes + 255) & ~size_t(255);
    return o;
  };
  const size_t o_qn = take(nsp * rule->qn_stride * 4), o_c0 = take(n * 4), o_mc0 = take(n * 4),
               o_codes = take(n * 4), o_mcodes = take(n * 4), o_chan = take(n * 4),
               o_mchan = take(n * 4), o_pos = take(n * 4), o_mpos = take(n * 4),
               o_cnt = take(nch * 16), o_mcnt = take(nch * 16), o_fill = take(nch * 16),
               o_mfill = take(nch * 16), o_err = take(4), o_zero_end = used,
               o_inv = take(nch * 4), o_seg = take(nch * 16), o_mseg = take(nch * 16),
               o_segs = take(nch * 8 * sizeof(PairSegment));
  void *base = nullptr;
  size_t got = 0;
  int rc = CCDGPU_OK;
  std::vector<uint32_t> cnt(nch * 4), mcnt(nch * 4);
  std::vector<uint32_t> inv(nch), seg(nch * 4), mseg(nch * 4), codes(n), mcodes(n);
  std::vector<PairSegment> segs;
  int32_t err = 0;
  auto at = [&](size_t o) { return static_cast<char *>(base) + o; };
  auto run = [&]() -> int {
    CK(dev_alloc(used, &base, &got));
    CK(cudaMemsetAsync(at(o_cnt), 0, o_zero_end - o_cnt, st));
    CK(cudaMemcpyAsync(at(o_qn), rule->qn, nsp * rule->qn_stride * 4, cudaMemcpyHostToDevice, st));
    ChannelRuleDev r{reinterpret_cast<const int32_t *>(at(o_qn)), rule->kind, rule->qn_stride,
                     rule->nmax, rule->chan_tz_max, rule->mod_chan_tz_max, nsp, np, nch};
    const unsigned grid = (unsigned)std::min<uint64_t>((n + 255) / 256, 148 * 16);
    uint32_t *c0 = reinterpret_cast<uint32_t *>(at(o_c0)), *mc0 = reinterpret_cast<uint32_t *>(at(o_mc0));
    pair_channel_kernel<<<grid, 256, 0, st>>>(r, c0, mc0, reinterpret_cast<uint32_t *>(at(o_cnt)),
                                               reinterpret_cast<uint32_t *>(at(o_mcnt)),
                                               reinterpret_cast<int32_t *>(at(o_err)));
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(cnt.data(), at(o_cnt), nch * 16, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(mcnt.data(), at(o_mcnt), nch * 16, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&err, at(o_err), 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (err) return CCDGPU_ERR_INVALID_ARGUMENT;  // a pair outside the channel slots
    // Channel order, dimensions and segment starts (kinds one after another).
    std::vector<ccdgpu_channel_dims> d0(nch), md0(nch);
    for (uint64_t c = 0; c < nch; c++) {
      d0[c] = {cnt[c * 4 + 0], cnt[c * 4 + 1], cnt[c * 4 + 2], cnt[c * 4 + 3]};
      md0[c] = {mcnt[c * 4 + 0], mcnt[c * 4 + 1], mcnt[c * 4 + 2], mcnt[c * 4 + 3]};
    }
    const std::vector<uint64_t> order = ffd_channel_order(d0);
    for (uint64_t i = 0; i < nch; i++) {
      inv[order[i]] = (uint32_t)i;
      dims[i] = d0[order[i]];
      mod_dims[i] = md0[order[i]];
    }
    uint64_t base_k = 0;
    for (int k = 0; k < 4; k++) {
      uint64_t o = base_k, mo = base_k;
      for (uint64_t i = 0; i < nch; i++) {
        const uint64_t len = (&dims[i].pp)[k], mlen = (&mod_dims[i].pp)[k];
        if (len > (uint64_t)kMaxSegment || mlen > (uint64_t)kMaxSegment) return CCDGPU_ERR_UNSUPPORTED;
        seg[i * 4 + k] = (uint32_t)o;
        mseg[i * 4 + k] = (uint32_t)mo;
        if (len) segs.push_back(PairSegment{(uint32_t)o, (uint32_t)len, 0, 0});
        if (mlen) segs.push_back(PairSegment{(uint32_t)mo, (uint32_t)mlen, 1, 0});
        o += len;
        mo += mlen;
      }
      if (o - base_k != tot[k] || mo - base_k != tot[k]) return CCDGPU_ERR_INVALID_ARGUMENT;
      base_k += tot[k];
    }
    if (segs.size() > nch * 8) return CCDGPU_ERR_INVALID_ARGUMENT;
    CK(cudaMemcpyAsync(at(o_inv), inv.data(), nch * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(at(o_seg), seg.data(), nch * 16, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(at(o_mseg), mseg.data(), nch * 16, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(at(o_segs), segs.data(), segs.size() * sizeof(PairSegment),
                       cudaMemcpyHostToDevice, st));
    uint32_t *codes_d = reinterpret_cast<uint32_t *>(at(o_codes));
    uint32_t *mcodes_d = reinterpret_cast<uint32_t *>(at(o_mcodes));
    place_pairs_kernel<<<grid, 256, 0, st>>>(
        nsp, np, c0, mc0, reinterpret_cast<const uint32_t *>(at(o_inv)),
        reinterpret_cast<const uint32_t *>(at(o_seg)), reinterpret_cast<const uint32_t *>(at(o_mseg)),
        reinterpret_cast<uint32_t *>(at(o_fill)), reinterpret_cast<uint32_t *>(at(o_mfill)),
        codes_d, mcodes_d, reinterpret_cast<uint32_t *>(at(o_chan)),
        reinterpret_cast<uint32_t *>(at(o_mchan)));
    CK(cudaGetLastError());
    if (!segs.empty()) {
      sort_segments_kernel<<<(unsigned)segs.size(), 512, 0, st>>>(
          reinterpret_cast<const PairSegment *>(at(o_segs)), codes_d, mcodes_d,
          reinterpret_cast<uint32_t *>(at(o_pos)), reinterpret_cast<uint32_t *>(at(o_mpos)));
      CK(cudaGetLastError());
    }
    CK(cudaMemcpyAsync(codes.data(), codes_d, n * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(mcodes.data(), mcodes_d, n * 4, cudaMemcpyDeviceToHost, st));
    if (chan) CK(cudaMemcpyAsync(chan, at(o_chan), n * 4, cudaMemcpyDeviceToHost, st));
    if (mod_chan) CK(cudaMemcpyAsync(mod_chan, at(o_mchan), n * 4, cudaMemcpyDeviceToHost, st));
    if (pos) CK(cudaMemcpyAsync(pos, at(o_pos), n * 4, cudaMemcpyDeviceToHost, st));
    if (mod_pos) CK(cudaMemcpyAsync(mod_pos, at(o_mpos), n * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    // Codes -> pairs.
    uint64_t kb[4] = {0, tot[0], tot[0] + tot[1], tot[0] + tot[1] + tot[2]};
    for (int k = 0; k < 4; k++) {
#pragma omp parallel for schedule(static)
      for (int64_t j = 0; j < (int64_t)tot[k]; j++) {
        const uint32_t x = codes[kb[k] + j], y = mcodes[kb[k] + j];
        lists[k][j] = ccdgpu_pair{x / nsp, x % nsp};
        mod_lists[k][j] = ccdgpu_pair{y / nsp, y % nsp};
      }
    }
    return CCDGPU_OK;
  };
  rc = run();
  (void)cudaStreamSynchronize(st);
  if (base) dev_free(base, got);
  cudaStreamDestroy(st);
  if (rc) (void)cudaGetLastError();
  return rc;
}

int ccdgpu_get_t2(ccdgpu_handle *h, double *t2, uint64_t n) {
  if (!h || !t2 || n != (uint64_t)h->n_t) return CCDGPU_ERR_INVALID_ARGUMENT;
  CK(cudaSetDevice(h->opt.device));
  int rc = sync_ctl(h);
  if (rc) return rc;
  const double *src = h->t[h->h_ctl->parity];
  if (h->opt.path == CCDGPU_PATH_TABLES) src = h->t[1];
  return copy_from_device(h, reinterpret_cast<char *>(t2), reinterpret_cast<const char *>(src),
                          n * 8);
}

int ccdgpu_step(ccdgpu_handle *h, double mixing, double *e_corr) {
  if (!h) return CCDGPU_ERR_INVALID_ARGUMENT;
  CK(cudaSetDevice(h->opt.device));
  const bool inject = h->inject_next_step;
  h->inject_next_step = false;
  int rc = set_ctl(h, 0, h->h_ctl->tol, INT64_MAX / 2, mixing, false);
  if (rc) return rc;
  if (inject) {
    const int32_t one = 1;
    CK(cudaMemcpyAsync(&h->ctl->inject, &one, sizeof(one), cudaMemcpyHostToDevice, h->s0));
  }
  if (h->opt.path == CCDGPU_PATH_TABLES) rc = tables_iteration(h, mixing, nullptr);
  else rc = enqueue_fused_iteration(h, h->nt > 0);
  if (inject) {  // the fault applies to this iteration only
    const int32_t zero = 0;
    CK(cudaMemcpyAsync(&h->ctl->inject, &zero, sizeof(zero), cudaMemcpyHostToDevice, h->s0));
  }
  if (rc) return rc;
  if ((rc = sync_ctl(h))) return rc;
  if ((rc = check_errors(h))) return rc;
  if (e_corr) *e_corr = h->h_ctl->e_corr;
  return std::isfinite(h->h_ctl->e_corr) ? CCDGPU_OK : CCDGPU_ERR_NONFINITE;
}

}  // extern "C"

namespace {

// A solve in two halves, so that a batch can put every handle's device loop in flight before
// waiting for any of them.
struct SolveState {
  bool fused = false, mixed = false, graph = false, device_loop = false;
  double tol = 0;
  int64_t cap = 0, it0 = 0, pol0 = 0;
  std::chrono::steady_clock::time_point t0;
};
constexpr int64_t kLoopChunk = 128;  // iterations one device-loop launch may run

// Device loop: launch up to kLoopChunk iterations without the host (no synchronisation).
int loop_launch(ccdgpu_handle *h, SolveState &st) {
  Control &c = *h->h_ctl;
  st.it0 = c.iterations;
  st.pol0 = c.polish_iters;
  c.stop_at = c.iterations + kLoopChunk;
  CK(cudaMemcpyAsync(&h->ctl->stop_at, &c.stop_at, sizeof(int64_t), cudaMemcpyHostToDevice,
                     h->s0));
  cudaGraphExec_t &g = st.mixed && c.phase == 1 ? h->loop_tc : h->loop64;
  if (!g) {  // a mixed handle's FP64 loop, first needed now (the stream is idle here)
    t_pdl = h->loop_pdl;
    const int rc = capture_loop_graph(h, false, &g);
    t_pdl = true;
    if (rc) return rc;
  }
  CK(cudaGraphLaunch(g, h->s0));
  return CCDGPU_OK;
}

int solve_begin(ccdgpu_handle *h, double tol, int64_t max_iters, double mixing, SolveState &st) {
  if (!h || max_iters < 0 || !(tol >= 0)) return CCDGPU_ERR_INVALID_ARGUMENT;
  CK(cudaSetDevice(h->opt.device));
  st.fused = h->opt.path == CCDGPU_PATH_FUSED;
  st.mixed = st.fused && h->nt > 0;
  st.tol = tol;
  st.cap = max_iters + 1;
  // A mixed solve starts in phase 1 (tensor-core ladder) and finishes in phase 2 (FP64).
  int rc = set_ctl(h, 1, tol, max_iters, mixing, true, -1, st.mixed ? 1 : 0);
  if (rc) return rc;
  st.graph = st.fused && h->opt.use_graph && !h->profiling;
  if (st.graph && h->opt.device_loop) ready_loop_graphs(h);
  st.device_loop = st.graph && h->opt.device_loop && h->loop_state == 1;
  if (st.graph && !st.device_loop && (rc = fused_ready_graph(h, false))) return rc;
  if (st.graph && !st.device_loop && st.mixed && (rc = fused_ready_graph(h, true))) return rc;
  st.t0 = std::chrono::steady_clock::now();
  if (st.device_loop) return loop_launch(h, st);
  return CCDGPU_OK;
}

int solve_finish(ccdgpu_handle *h, SolveState &st, double mixing, ccdgpu_result *res) {
  CK(cudaSetDevice(h->opt.device));
  int rc;
  int64_t launched = 0;
  while (st.device_loop) {
    if ((rc = sync_ctl(h))) return rc;
    Control &c = *h->h_ctl;
    const int64_t fp = (c.polish_iters - st.pol0) + (st.mixed ? 0 : c.iterations - st.it0);
    h->launches += (c.iterations - st.it0 - fp) * h->kernels_per_body_tc + fp * h->kernels_per_body64;
    if (c.done || c.iterations >= st.cap || c.iterations == st.it0) break;
    if ((rc = loop_launch(h, st))) return rc;
  }
  while (!st.device_loop) {
    // Iterations are launched in batches; once the device-side stop rule fires the remaining
    // launches of the batch return immediately.
    const int64_t batch = (st.fused && !h->profiling)
                              ? std::min<int64_t>(launched < 8 ? 4 : 8, st.cap - launched)
                              : 1;
    // The phase can only change inside a batch from 1 to 2; mixed iterations that follow
    // the switch in the same batch are no-ops on the device.
    const bool mphase = st.mixed && h->h_ctl->phase == 1;
    for (int64_t b = 0; b < batch; b++) {
      if (st.graph) CK(cudaGraphLaunch(mphase ? h->graph_tc : h->graph, h->s0));
      else if (st.fused) { if ((rc = enqueue_fused_iteration(h, mphase))) return rc; }
      else {
        if ((rc = tables_iteration(h, mixing, nullptr))) return rc;
      }
    }
    launched += batch;
    if (st.graph)
      h->launches += batch * (mphase ? h->kernels_per_graph_tc : h->kernels_per_graph);
    if ((rc = sync_ctl(h))) return rc;
    if (h->profiling && st.fused && !st.graph) {
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
    if (h->h_ctl->done || launched >= st.cap) break;
  }
  auto t1 = std::chrono::steady_clock::now();
  // The result reflects the control block also when the solve failed (for example non-finite
  // amplitudes of a diverging iteration); the status says so.
  const Control &c = *h->h_ctl;
  if (res) {
    res->e_corr = c.e_corr;
    res->e_diff = c.e_diff;
    res->iterations = c.iterations;
    res->converged = std::fabs(c.e_diff) <= st.tol ? 1 : 0;
    res->polish_iterations = (int32_t)c.polish_iters;
    res->seconds = std::chrono::duration<double>(t1 - st.t0).count();
  }
  return check_errors(h);
}

}  // namespace

extern "C" {

int ccdgpu_solve(ccdgpu_handle *h, double tol, int64_t max_iters, double mixing, ccdgpu_result *res) {
  SolveState st;
  int rc = solve_begin(h, tol, max_iters, mixing, st);
  if (rc) return rc;
  return solve_finish(h, st, mixing, res);
}

int ccdgpu_solve_batch(ccdgpu_handle *const *hs, int32_t n, double tol, int64_t max_iters,
                       double mixing, ccdgpu_result *res) {
  if (!hs || n < 0) return CCDGPU_ERR_INVALID_ARGUMENT;
  for (int32_t i = 0; i < n; i++)
    for (int32_t j = 0; j < i; j++)
      if (!hs[i] || hs[i] == hs[j]) return CCDGPU_ERR_INVALID_ARGUMENT;
  std::vector<SolveState> st(n);
  int first_rc = CCDGPU_OK;
  std::vector<int> begun(n, 0);
  // Every handle's device loop goes in flight on its own streams before any is waited for.
  for (int32_t i = 0; i < n; i++) {
    const int rc = solve_begin(hs[i], tol, max_iters, mixing, st[i]);
    if (rc && !first_rc) first_rc = rc;
    begun[i] = rc == CCDGPU_OK;
  }
  for (int32_t i = 0; i < n; i++) {
    if (!begun[i]) continue;
    const int rc = solve_finish(hs[i], st[i], mixing, res ? &res[i] : nullptr);
    if (rc && !first_rc) first_rc = rc;
  }
  return first_rc;
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
  if (rc || (rc = launch_ring(h, h->s0, 0, false))) return rc;
  CK(cudaStreamSynchronize(h->s0));
  return CCDGPU_OK;
}
int ccdgpu_calc_t2diff_pphh(ccdgpu_handle *h) {
  if (!h) return CCDGPU_ERR_INVALID_ARGUMENT;
  int rc = set_ctl(h, 0, h->h_ctl->tol, h->h_ctl->max_iters, h->h_ctl->mixing, false);
  if (rc || (rc = launch_hh_ladder(h, h->s0, 0)) || (rc = launch_pp_ladder(h, h->s0))) return rc;
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
  if (chain == CCDGPU_CHAIN_OLD_PHHP && h->opt.path != CCDGPU_PATH_TABLES) {
    // The fused path gathers the slab at the head of each iteration's ring: bring it up to
    // the current amplitudes first.
    if ((rc = launch_phhp_gather(h, h->s0, -1))) return rc;
    CK(cudaStreamSynchronize(h->s0));
  }
  CK(cudaMemcpy(out, src, len * 8, cudaMemcpyDeviceToHost));
  return CCDGPU_OK;
}

int ccdgpu_get_profile(ccdgpu_handle *h, ccdgpu_profile *prof) {
  if (!h || !prof) return CCDGPU_ERR_INVALID_ARGUMENT;
  *prof = h->prof;
  prof->launches = h->launches;
  for (int k = 0; k < 5; k++) prof->ms_create[k] = h->create_ms[k];
  prof->ms_loop_graph = h->loop_graph_ms;
  return CCDGPU_OK;
}
int ccdgpu_enable_profiling(ccdgpu_handle *h, int32_t on) {
  if (!h) return CCDGPU_ERR_INVALID_ARGUMENT;
  h->profiling = on != 0;
  h->prof = ccdgpu_profile{};
  return CCDGPU_OK;
}
void *ccdgpu_stream(ccdgpu_handle *h) { return h ? (void *)h->s0 : nullptr; }

int ccdgpu_inject_wait_timeout(ccdgpu_handle *h) {
  if (!h) return CCDGPU_ERR_INVALID_ARGUMENT;
  h->inject_next_step = true;
  return CCDGPU_OK;
}

// Each pp-ladder class launched alone (FP64 thin, mid, wide; tensor-core ladder), `reps` times
// between CUDA events on the handle's stream; with the executed flops (packed: rows a<=b, K over
// c<d and hh) and the algorithmic bytes of each class.
int ccdgpu_kernel_profile(ccdgpu_handle *h, int32_t reps, double *ms, double *flops,
                          double *bytes) {
  if (!h || reps < 1 || !ms || !flops || !bytes) return CCDGPU_ERR_INVALID_ARGUMENT;
  CK(cudaSetDevice(h->opt.device));
  int rc = set_ctl(h, 0, h->h_ctl->tol, h->h_ctl->max_iters, h->h_ctl->mixing, false);
  if (rc) return rc;
  for (int k = 0; k < 7; k++) ms[k] = flops[k] = bytes[k] = 0;
  // Ring: Y = V_hphp + 0.5 V_hpph T' and R = T' Y; reads T', V_hpph, V_hphp and the inverse
  // ai_jb table, writes R.
  for (const ModInfo &m : h->host_mods) {
    const int k = (m.ph <= kRingSmall && m.hp <= kRingSmall) ? 0
                  : (m.ph <= 32 && m.hp <= 32) ? 1 : 2;
    flops[k] += 4.0 * m.ph * (double)m.hp * m.hp;
    bytes[k] += 28.0 * m.ph * m.hp + 8.0 * m.hp * m.hp;
  }
  // The small class is launched with the phhp gather ahead of it (fused path): per slab
  // element an index, one read of t and the slab store.
  bytes[0] += 20.0 * (double)h->n_m;
  // hh ladder: P = V_hhpp T over the pp rows and r = row dots; reads V_pphh and T, writes the
  // slice partials of P and r.  Reduction: reads the partials and V_hhhh, writes X (reference
  // layout and FP64 operand tiles) and s.
  for (const ChanInfo &a : h->host_chans) {
    const int k = a.hh <= 16 ? 3 : 4;
    const double hh2 = (double)a.hh * a.hh;
    flops[k] += 2.0 * a.pp * a.hh * (a.hh + 1.0);
    bytes[k] += 16.0 * a.pp * a.hh + 8.0 * a.nhht * hh2 + 8.0 * a.pp;
    flops[6] += (double)a.nhht * hh2;
    bytes[6] += 8.0 * a.nhht * hh2 + 24.0 * hh2 + 8.0 * a.hh;
  }
  // One-body: segmented sums of s and r (one value per pair) into x_k and y_a.
  flops[5] = (double)h->n_t * 0;  // no arithmetic worth counting
  bytes[5] = 16.0 * (double)(h->nsp) + 12.0 * (double)h->n_list;
  for (int k = 0; k < 7; k++) {
    auto launch = [&]() -> int {
      if (k <= 2) return launch_ring(h, h->s0, 0, true, k);
      if (k <= 4) return launch_hh_ladder(h, h->s0, 0, k - 3);
      if (k == 6) return launch_hh_ladder(h, h->s0, 0, 2);
      return launch_onebody_fused(h, h->s0, 0);
    };
    if ((rc = launch())) return rc;  // warm-up
    CK(cudaEventRecord(h->ev[0], h->s0));
    for (int i = 0; i < reps && !rc; i++) rc = launch();
    if (rc) return rc;
    CK(cudaEventRecord(h->ev[1], h->s0));
    CK(cudaEventSynchronize(h->ev[1]));
    float t = 0;
    CK(cudaEventElapsedTime(&t, h->ev[0], h->ev[1]));
    ms[k] = t / reps;
  }
  return check_errors(h);
}

int ccdgpu_ladder_profile(ccdgpu_handle *h, int32_t reps, double *ms, double *flops,
                          double *bytes) {
  if (!h || reps < 1 || !ms || !flops || !bytes) return CCDGPU_ERR_INVALID_ARGUMENT;
  CK(cudaSetDevice(h->opt.device));
  int rc = set_ctl(h, 0, h->h_ctl->tol, h->h_ctl->max_iters, h->h_ctl->mixing, false);
  if (rc) return rc;
  for (int k = 0; k < 4; k++) ms[k] = flops[k] = bytes[k] = 0;
  for (const ChanInfo &a : h->host_chans) {
    const int k = a.nb <= 8 ? 0 : a.nb <= 32 ? 1 : 2;
    const double f = 2.0 * a.pr * ((double)a.pk + a.hh) * a.hh;
    const double b = (double)a.pr * a.pk + ((double)a.pk + a.pr) * a.hh + (double)a.hh * a.hh;
    flops[k] += f;
    bytes[k] += 8.0 * b + 8.0 * a.pp * a.hh;
    if (h->nt) {
      flops[3] += f;
      bytes[3] += 2.0 * h->nt * (h->tc_gen ? b - (double)a.pr * a.pk : b) + 8.0 * a.pp * a.hh;
    }
  }
  for (int k = 0; k < 4; k++) {
    if (k < 3 && !h->n_cls[k]) continue;
    if (k == 3 && !h->n_tc_tiles) continue;
    auto launch = [&]() -> int {
      if (k == 3) return launch_pp_ladder_tc(h, h->s0);
      const size_t smem = k == 0 ? h->ladder_smem_thin : h->ladder_smem;
      auto kern = k == 0 ? pp_ladder_kernel<0> : k == 1 ? pp_ladder_kernel<1> : pp_ladder_kernel<2>;
      kern<<<h->fp_grid[k], ladder_threads(k), smem, h->s0>>>(
          h->tiles, h->fp_cta_off + h->fp_off_base[k], h->v_t, h->t_kt, h->t_mt, h->x_t,
          h->rowmap, h->mirror, h->dmat, h->lpart, h->ctl, h->err, 0);
      CK(cudaGetLastError());
      if (h->n_red_cls[k]) {
        const int off = k == 0 ? 0 : k == 1 ? h->n_red_cls[0] : h->n_red_cls[0] + h->n_red_cls[1];
        ladder_reduce_kernel<<<h->n_red_cls[k], 256, 0, h->s0>>>(
            h->red_fp + off, h->tiles, h->rowmap, h->mirror, h->dmat, h->lpart, h->ctl, 0);
        CK(cudaGetLastError());
      }
      return CCDGPU_OK;
    };
    if ((rc = launch())) return rc;  // warm-up
    CK(cudaEventRecord(h->ev[0], h->s0));
    for (int i = 0; i < reps && !rc; i++) rc = launch();
    if (rc) return rc;
    CK(cudaEventRecord(h->ev[1], h->s0));
    CK(cudaEventSynchronize(h->ev[1]));
    float t = 0;
    CK(cudaEventElapsedTime(&t, h->ev[0], h->ev[1]));
    ms[k] = t / reps;
  }
  return check_errors(h);
}

int ccdgpu_set_schedule(ccdgpu_handle *h, const ccdgpu_schedule *sch) {
  if (!h || !sch || sch->thin_split_mul < 1 || sch->wide_split_mul < 1 || sch->tc_split_mul < 1 ||
      sch->mid_split_mul < 0)
    return CCDGPU_ERR_INVALID_ARGUMENT;
  CK(cudaSetDevice(h->opt.device));
  return make_ladder_tiles(h, *sch);
}

int ccdgpu_get_schedule(const ccdgpu_handle *h, ccdgpu_schedule *sch) {
  if (!h || !sch) return CCDGPU_ERR_INVALID_ARGUMENT;
  *sch = h->schedule;
  return CCDGPU_OK;
}

// Times `reps` launches of the handle's pp ladders for each candidate schedule (CUDA events on
// the handle's stream; the ladders only overwrite the iteration's D) and keeps the fastest.
int ccdgpu_autotune(ccdgpu_handle *h, int32_t reps, ccdgpu_schedule *chosen, double *ms_fp64,
                    double *ms_tc) {
  if (!h || reps < 1) return CCDGPU_ERR_INVALID_ARGUMENT;
  CK(cudaSetDevice(h->opt.device));
  int rc = set_ctl(h, 0, h->h_ctl->tol, h->h_ctl->max_iters, h->h_ctl->mixing, false);
  if (rc) return rc;
  auto time_ladder = [&](bool tc, double *ms) -> int {
    int r = tc ? launch_pp_ladder_tc(h, h->s0) : launch_pp_ladder(h, h->s0);  // warm-up
    if (r) return r;
    CK(cudaEventRecord(h->ev[0], h->s0));
    for (int i = 0; i < reps && !r; i++) r = tc ? launch_pp_ladder_tc(h, h->s0) : launch_pp_ladder(h, h->s0);
    if (r) return r;
    CK(cudaEventRecord(h->ev[1], h->s0));
    CK(cudaEventSynchronize(h->ev[1]));
    float t = 0;
    CK(cudaEventElapsedTime(&t, h->ev[0], h->ev[1]));
    *ms = t / reps;
    return check_errors(h);
  };
  ccdgpu_schedule best = h->schedule;
  double best64 = 0, besttc = 0;
  // FP64 ladder: split factors of the thin and the mid/wide classes (mid as wide), then the
  // mid class's own.
  const int thin_c[] = {1, 2, 4}, wide_c[] = {1, 2, 3, 6, 12, 24, 48};
  bool first = true;
  best.mid_split_mul = 0;
  for (int tm : thin_c)
    for (int wm : wide_c) {
      ccdgpu_schedule c = best;
      c.thin_split_mul = tm;
      c.wide_split_mul = wm;
      if ((rc = make_ladder_tiles(h, c))) return rc;
      double ms = 0;
      if ((rc = time_ladder(false, &ms))) return rc;
      if (first || ms < best64) { best64 = ms; best.thin_split_mul = tm; best.wide_split_mul = wm; }
      first = false;
    }
  for (int mm : wide_c) {
    ccdgpu_schedule c = best;
    c.mid_split_mul = mm;
    if ((rc = make_ladder_tiles(h, c))) return rc;
    double ms = 0;
    if ((rc = time_ladder(false, &ms))) return rc;
    if (ms < best64) { best64 = ms; best.mid_split_mul = mm; }
  }
  // Tensor-core ladder: split factor.
  if (h->nt) {
    first = true;
    const int tc_c[] = {1, 2, 4, 8, 16};
    for (int tm : tc_c) {
      ccdgpu_schedule c = best;
      c.tc_split_mul = tm;
      if ((rc = make_ladder_tiles(h, c))) return rc;
      double ms = 0;
      if ((rc = time_ladder(true, &ms))) return rc;
      if (first || ms < besttc) { besttc = ms; best.tc_split_mul = tm; }
      first = false;
    }
  }
  if ((rc = make_ladder_tiles(h, best))) return rc;
  if (chosen) *chosen = best;
  if (ms_fp64) *ms_fp64 = best64;
  if (ms_tc) *ms_tc = besttc;
  return CCDGPU_OK;
}

int ccdgpu_trace_arm(ccdgpu_handle *h, int64_t iteration) {
  if (!h) return CCDGPU_ERR_INVALID_ARGUMENT;
  CK(cudaSetDevice(h->opt.device));
  int rc = sync_ctl(h);
  if (rc) return rc;
  Control &c = *h->h_ctl;
  c.trace_iter = iteration;
  for (int k = 0; k < kTraceKernels; k++) {
    c.trace_first[k] = ~0ull;
    c.trace_last[k] = 0;
    c.trace_end[k] = 0;
  }
  CK(cudaMemcpyAsync(h->ctl, h->h_ctl, sizeof(Control), cudaMemcpyHostToDevice, h->s0));
  CK(cudaStreamSynchronize(h->s0));
  return CCDGPU_OK;
}

int ccdgpu_trace_read(ccdgpu_handle *h, uint64_t *first, uint64_t *last, int32_t n) {
  if (!h || !first || !last || n < 0) return CCDGPU_ERR_INVALID_ARGUMENT;
  CK(cudaSetDevice(h->opt.device));
  int rc = sync_ctl(h);
  if (rc) return rc;
  for (int k = 0; k < n && k < kTraceKernels; k++) {
    first[k] = h->h_ctl->trace_first[k];
    last[k] = h->h_ctl->trace_last[k];
  }
  return CCDGPU_OK;
}
int ccdgpu_trace_read_end(ccdgpu_handle *h, uint64_t *end, int32_t n) {
  if (!h || !end || n < 0) return CCDGPU_ERR_INVALID_ARGUMENT;
  CK(cudaSetDevice(h->opt.device));
  int rc = sync_ctl(h);
  if (rc) return rc;
  for (int k = 0; k < n && k < kTraceKernels; k++) end[k] = h->h_ctl->trace_end[k];
  return CCDGPU_OK;
}
int ccdgpu_work_per_iteration(const ccdgpu_handle *h, double *flops, double *v_pppp_bytes,
                              double *ladder_flops) {
  if (!h) return CCDGPU_ERR_INVALID_ARGUMENT;
  if (flops) *flops = h->flops;
  if (v_pppp_bytes) *v_pppp_bytes = h->nt ? h->ladder_bytes_tc : h->ladder_bytes;
  if (ladder_flops) *ladder_flops = h->ladder_flops;
  return CCDGPU_OK;
}

}  // extern "C"
