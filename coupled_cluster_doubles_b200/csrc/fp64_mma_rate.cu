// FP64 throughput on sm_100a: DFMA against the FP64 mma.sync shapes (m8n8k4, m16n8k16), every
// MMA fed from shared memory with operands that change each iteration, plus a fragment-layout
// and accuracy check of both shapes against a long-double CPU product.  Standalone (not part of
// the library):
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -o fp64_mma_rate fp64_mma_rate.cu
//   ./fp64_mma_rate
// Lane layouts used by the library's FP64 MMA kernels (g = lane / 4, t = lane % 4):
//   m8n8k4:   a = A[g][t], b = B[t][g], c = {C[g][2t], C[g][2t+1]}
//   m16n8k16: a_i = A[g + 8 (i % 2)][t + 4 (i / 2)], b_i = B[t + 4 i][g],
//             c = {C[g][2t], C[g][2t+1], C[g+8][2t], C[g+8][2t+1]}
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include <cuda_runtime.h>

constexpr int kIters = 256;
constexpr int kFrags = 8;  // distinct operand sets cycled through

__device__ __forceinline__ void mma884(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c[0]), "+d"(c[1]) : "d"(a), "d"(b));
}
__device__ __forceinline__ void mma16816(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
      "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
        "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// 16 doubles per lane per operand set in shared memory, lane-minor ([set][i][lane]: a warp's
// load of one i touches 32 consecutive doubles, conflict-free); src holds 4096 doubles.
__device__ void stage(const double *src, double (*s)[16][32]) {
  for (int i = threadIdx.x; i < kFrags * 16 * 32; i += blockDim.x)
    (&s[0][0][0])[i] = src[(i * 7) % 4096];
  __syncthreads();
}

// DFMA: 8 operands loaded per iteration, 128 dependent-free FMAs on them (loads are 1/16 of
// the instructions, so shared memory does not bound the rate).
__global__ void dfma_kernel(const double *src, double *out) {
  __shared__ double s[kFrags][16][32];
  stage(src, s);
  const int l = threadIdx.x & 31;
  double acc[8] = {};
  for (int it = 0; it < kIters; ++it) {
    double x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = s[it % kFrags][i][l];
#pragma unroll
    for (int r = 0; r < 16; ++r)
#pragma unroll
      for (int i = 0; i < 8; ++i) acc[i] = fma(x[i], x[(i + r) % 8], acc[i]);
  }
  double r = 0;
  for (int i = 0; i < 8; ++i) r += acc[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = r;
}

// DFMA in the a = a * m + x form: 16 independent accumulators, one multiplier and 8 addends
// loaded per iteration, 128 FMAs on them.
__global__ void dfma_axpy_kernel(const double *src, double *out) {
  __shared__ double s[kFrags][16][32];
  stage(src, s);
  const int l = threadIdx.x & 31;
  double acc[16] = {};
  for (int it = 0; it < kIters; ++it) {
    const double m = s[it % kFrags][8][l];
    double x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = s[it % kFrags][i][l];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
      for (int i = 0; i < 16; ++i) acc[i] = fma(acc[i], m, x[(i + r) & 7]);
  }
  double r = 0;
  for (int i = 0; i < 16; ++i) r += acc[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = r;
}

__global__ void m884_kernel(const double *src, double *out) {
  __shared__ double s[kFrags][16][32];
  stage(src, s);
  const int l = threadIdx.x & 31;
  double c[4][2] = {};
  for (int it = 0; it < kIters; ++it) {
    const double a = s[it % kFrags][0][l], b = s[it % kFrags][1][l];
#pragma unroll
    for (int q = 0; q < 4; ++q) mma884(c[q], a, b);  // 4 MMAs per iteration
  }
  double r = 0;
  for (int q = 0; q < 4; ++q) r += c[q][0] + c[q][1];
  out[blockIdx.x * blockDim.x + threadIdx.x] = r;
}

__global__ void m16816_kernel(const double *src, double *out) {
  __shared__ double s[kFrags][16][32];
  stage(src, s);
  const int l = threadIdx.x & 31;
  double c[4][4] = {};
  for (int it = 0; it < kIters; ++it) {
    double a[8], b[4];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = s[it % kFrags][i][l];
#pragma unroll
    for (int i = 0; i < 4; ++i) b[i] = s[it % kFrags][8 + i][l];
#pragma unroll
    for (int q = 0; q < 4; ++q) mma16816(c[q], a, b);  // 4 MMAs per iteration
  }
  double r = 0;
  for (int q = 0; q < 4; ++q) r += c[q][0] + c[q][1] + c[q][2] + c[q][3];
  out[blockIdx.x * blockDim.x + threadIdx.x] = r;
}

// One warp: C (16 x 8) = A (16 x 16) B (16 x 8) with m16n8k16, and C[0:8] = A[0:8][0:4] B[0:4]
// with m8n8k4 (into c8, 8 x 8).
__global__ void layout_kernel(const double *A, const double *B, double *C, double *c8) {
  const int l = threadIdx.x, g = l >> 2, t = l & 3;
  double a[8], b[4], c[4] = {0, 0, 0, 0};
  for (int i = 0; i < 8; ++i) a[i] = A[(g + 8 * (i % 2)) * 16 + t + 4 * (i / 2)];
  for (int i = 0; i < 4; ++i) b[i] = B[(t + 4 * i) * 8 + g];
  mma16816(c, a, b);
  C[g * 8 + 2 * t] = c[0];
  C[g * 8 + 2 * t + 1] = c[1];
  C[(g + 8) * 8 + 2 * t] = c[2];
  C[(g + 8) * 8 + 2 * t + 1] = c[3];
  double d[2] = {0, 0};
  mma884(d, A[g * 16 + t], B[t * 8 + g]);
  c8[g * 8 + 2 * t] = d[0];
  c8[g * 8 + 2 * t + 1] = d[1];
}

int main() {
  const int threads = 256;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  double *src, *out;
  cudaMalloc(&src, 4096 * sizeof(double));
  cudaMalloc(&out, sizeof(double) * sms * (2048 / threads) * threads);
  double hs[4096];
  srand(11);
  for (int i = 0; i < 4096; ++i) hs[i] = (rand() / (double)RAND_MAX - 0.5) * 1e-3;
  cudaMemcpy(src, hs, sizeof hs, cudaMemcpyHostToDevice);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  struct Case {
    const char *name;
    void (*k)(const double *, double *);
    double flops_per_warp;
  } cases[] = {
      {"dfma", dfma_kernel, 2.0 * 128 * 32 * kIters},
      {"dfma a=a*m+x", dfma_axpy_kernel, 2.0 * 128 * 32 * kIters},
      {"mma m8n8k4", m884_kernel, 2.0 * 8 * 8 * 4 * 4 * kIters},
      {"mma m16n8k16", m16816_kernel, 2.0 * 16 * 8 * 16 * 4 * kIters},
  };
  for (const Case &c : cases) {
    // One full wave: every SM holds as many blocks as fit, so no tail wave runs under-occupied.
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, c.k, threads, 0);
    const int blocks = sms * per_sm;
    float best = 1e30f;
    for (int rep = 0; rep < 5; ++rep) {
      cudaEventRecord(e0);
      c.k<<<blocks, threads>>>(src, out);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      float ms;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep >= 2 && ms < best) best = ms;
    }
    const double fl = c.flops_per_warp * (threads / 32) * (double)blocks;
    printf("%-14s %d blocks/SM  %8.3f ms  %6.2f TFLOP/s  (%s)\n", c.name, per_sm, best,
           fl / best / 1e9, cudaGetErrorString(cudaGetLastError()));
  }
  double hA[256], hB[128], hC[128], h8[64];
  for (int i = 0; i < 256; ++i) hA[i] = (rand() / (double)RAND_MAX - 0.5) * pow(10.0, rand() % 7 - 3);
  for (int i = 0; i < 128; ++i) hB[i] = (rand() / (double)RAND_MAX - 0.5) * pow(10.0, rand() % 7 - 3);
  double *dA, *dB, *dC, *d8;
  cudaMalloc(&dA, sizeof hA);
  cudaMalloc(&dB, sizeof hB);
  cudaMalloc(&dC, sizeof hC);
  cudaMalloc(&d8, sizeof h8);
  cudaMemcpy(dA, hA, sizeof hA, cudaMemcpyHostToDevice);
  cudaMemcpy(dB, hB, sizeof hB, cudaMemcpyHostToDevice);
  layout_kernel<<<1, 32>>>(dA, dB, dC, d8);
  cudaMemcpy(hC, dC, sizeof hC, cudaMemcpyDeviceToHost);
  cudaMemcpy(h8, d8, sizeof h8, cudaMemcpyDeviceToHost);
  double e16 = 0, s16 = 0, e8 = 0, s8 = 0;
  for (int m = 0; m < 16; ++m)
    for (int n = 0; n < 8; ++n) {
      long double r = 0, a = 0;
      for (int k = 0; k < 16; ++k) {
        r += (long double)hA[m * 16 + k] * hB[k * 8 + n];
        a += fabsl((long double)hA[m * 16 + k] * hB[k * 8 + n]);
      }
      e16 = fmax(e16, fabs((double)(hC[m * 8 + n] - r)));
      s16 = fmax(s16, (double)a);
      if (m < 8) {
        long double r8 = 0, a8 = 0;
        for (int k = 0; k < 4; ++k) {
          r8 += (long double)hA[m * 16 + k] * hB[k * 8 + n];
          a8 += fabsl((long double)hA[m * 16 + k] * hB[k * 8 + n]);
        }
        e8 = fmax(e8, fabs((double)(h8[m * 8 + n] - r8)));
        s8 = fmax(s8, (double)a8);
      }
    }
  printf("m16n8k16 layout: max |error| / max sum|ab| = %.3e\n", e16 / s16);
  printf("m8n8k4   layout: max |error| / max sum|ab| = %.3e\n", e8 / s8);
  const bool ok = e16 / s16 < 1e-14 && e8 / s8 < 1e-14;
  printf("%s\n", ok ? "layouts ok" : "LAYOUT MISMATCH");
  return ok ? 0 : 1;
}
