// ccdgpu_calc_channel_t2diff_pphh_noalloc: the ladder term of one regular channel,
// computed without allocating any memory.
//
// Some callers cannot call cudaMalloc: a host that owns every byte of device memory through
// its own pool or budget and forbids a library to take more, or code that must not perturb
// the allocator state between calls.  This entry point serves them.  The caller passes all
// inputs and outputs as device buffers, and the split-K intermediate lives in a fixed
// file-scope device array that the library carries (kNoAllocScratchDoubles doubles, 2 MiB per
// GPU that loads the library, held until the process exits).
//
// Scratch layout (doubles): [0, 32) ticket counter (as int), [32, 32 + hh^2) X,
// then nslices * hh^2 partial products, nslices = ceil(pp / 64).
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "ccdgpu.h"

namespace {

constexpr int64_t kNoAllocScratchDoubles = int64_t(1) << 18;  // 2 MiB
constexpr int kSliceRows = 64;
constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

double *g_scratch_ptr[kMaxDevices] = {};
std::mutex g_setup_mutex;

// X = V_hhhh + 0.5 * V_hhpp T, split over 64-row slices of the pp index.  Each CTA writes the
// partial product of its slice; the last CTA (ticket) sums the slices in order and writes X.
__global__ void __launch_bounds__(kThreads)
noalloc_x_kernel(const double *__restrict__ v_hhpp, const double *__restrict__ t2,
                 const double *__restrict__ v_hhhh, int pp, int hh, double *scratch) {
  extern __shared__ double sm[];
  __shared__ int last;
  const int slice = blockIdx.x, k0 = slice * kSliceRows;
  const int rows = min(kSliceRows, pp - k0), tid = threadIdx.x, nout = hh * hh;
  double *Vs = sm, *Ts = sm + kSliceRows * hh;  // Vs[k][kl] = V_hhpp[kl][k0+k], Ts[k][ij]
  for (int e = tid; e < rows * hh; e += kThreads) {
    const int k = e / hh, c = e - k * hh;
    Vs[e] = v_hhpp[(int64_t)c * pp + k0 + k];
    Ts[e] = t2[(int64_t)(k0 + k) * hh + c];
  }
  __syncthreads();
  double *x = scratch + 32, *part = x + nout;
  for (int idx = tid; idx < nout; idx += kThreads) {
    const int kl = idx / hh, ij = idx - kl * hh;
    double a = 0.0;
    for (int k = 0; k < rows; ++k) a += Vs[k * hh + kl] * Ts[k * hh + ij];
    part[(int64_t)slice * nout + idx] = a;
  }
  __threadfence();
  __syncthreads();
  int *ticket = reinterpret_cast<int *>(scratch);
  if (tid == 0) last = (atomicAdd(ticket, 1) == (int)gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int idx = tid; idx < nout; idx += kThreads) {
    double p = 0.0;
    for (int s = 0; s < (int)gridDim.x; ++s) p += __ldcg(part + (int64_t)s * nout + idx);
    x[idx] = 0.5 * p + v_hhhh[idx];
  }
}

// D = 0.5 T X, then D = 0.5 V_pppp T + D (the two dgemm calls of calc.cpp:167-201).
__global__ void __launch_bounds__(kThreads)
noalloc_d_kernel(const double *__restrict__ v_pppp, const double *__restrict__ t2, int pp, int hh,
                 const double *scratch, double *__restrict__ d) {
  const double *x = scratch + 32;
  const int64_t n = (int64_t)pp * hh;
  for (int64_t e = blockIdx.x * (int64_t)kThreads + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * kThreads) {
    const int row = (int)(e / hh), col = (int)(e - (int64_t)row * hh);
    double tx = 0.0;
    for (int k = 0; k < hh; ++k) tx += t2[(int64_t)row * hh + k] * x[k * hh + col];
    double vt = 0.0;
    for (int k = 0; k < pp; ++k) vt += v_pppp[(int64_t)row * pp + k] * t2[(int64_t)k * hh + col];
    d[e] = 0.5 * vt + 0.5 * tx;
  }
}

// Device address of the scratch array for the current device, looked up once per device.
int scratch_for_current_device(double **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    (void)cudaGetLastError();
    return CCDGPU_ERR_NO_DEVICE;
  }
  if (dev < 0 || dev >= kMaxDevices) return CCDGPU_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    double *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&p), g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      (void)cudaGetLastError();
      return CCDGPU_ERR_CUDA;
    }
    // Dynamic shared memory of the X kernel at the largest supported hh (72).
    if (cudaFuncSetAttribute(noalloc_x_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             2 * kSliceRows * 72 * (int)sizeof(double)) != cudaSuccess) {
      (void)cudaGetLastError();
      return CCDGPU_ERR_CUDA;
    }
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return CCDGPU_OK;
}

}  // namespace

extern "C" int ccdgpu_calc_channel_t2diff_pphh_noalloc(const double *v_pppp, const double *v_hhpp,
                                                       const double *v_hhhh, const double *t2,
                                                       double *d, int64_t pp, int64_t hh,
                                                       void *stream) {
  if (!v_pppp || !v_hhpp || !v_hhhh || !t2 || !d || pp < 1 || hh < 1)
    return CCDGPU_ERR_INVALID_ARGUMENT;
  const int64_t nslices = (pp + kSliceRows - 1) / kSliceRows;
  if (hh > 72 || pp > (int64_t(1) << 20) || 32 + (nslices + 1) * hh * hh > kNoAllocScratchDoubles)
    return CCDGPU_ERR_UNSUPPORTED;  // beyond the fixed scratch capacity
  double *scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // The ticket counter must start at zero; the rest of the scratch is fully overwritten.
  cudaError_t e = cudaMemsetAsync(scratch, 0, 32 * sizeof(double), st);
  if (e == cudaSuccess) {
    const size_t smem = (size_t)2 * kSliceRows * hh * sizeof(double);
    noalloc_x_kernel<<<(unsigned)nslices, kThreads, smem, st>>>(v_hhpp, t2, v_hhhh, (int)pp,
                                                                (int)hh, scratch);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    const int64_t blocks = (pp * hh + kThreads - 1) / kThreads;
    noalloc_d_kernel<<<(unsigned)(blocks < 4096 ? blocks : 4096), kThreads, 0, st>>>(
        v_pppp, t2, (int)pp, (int)hh, scratch, d);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? CCDGPU_ERR_OUT_OF_MEMORY : CCDGPU_ERR_CUDA;
  }
  return CCDGPU_OK;
}
