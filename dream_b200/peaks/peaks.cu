// peaks.cu -- microbenchmarks for the roofline denominators the DAS kernels are
// measured against on this GPU (built into libdream_peaks.so, run by
// `python bench.py --peaks`; not part of the beamformer library):
//
//   l2_sector_gather  one 4-byte load per thread at a random 32-byte sector of
//                     an L2-resident buffer: 32 sectors per warp request
//   l2_das_gather     the DAS access shape: each warp reads 32 words spread
//                     over a window of ~100 words at a random offset
//   fp32_fma, fp64_fma, int_add   arithmetic throughput over 8 independent chains
//                     per thread (int_add counts the XOR and the ADD of each step)
//
// Each kernel returns nothing useful; results are derived from CUDA-event
// time and the known operation counts.
#include <cuda_runtime.h>
#include <stdint.h>

namespace {

__device__ __forceinline__ uint32_t hash32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352dU;
  x ^= x >> 15;
  x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}

// Random sector gather: thread t, iteration r reads word 8*h(t,r) (one
// sector each). n_sectors is a power of two.
__global__ void l2_sector_gather(const float *__restrict__ buf, uint32_t sector_mask, int iters,
                                 float *__restrict__ sink) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  float acc = 0.0f;
#pragma unroll 8
  for (int r = 0; r < iters; r++) {
    uint32_t s = hash32(t * 0x9e3779b9U + (uint32_t)r * 0x85ebca6bU) & sector_mask;
    acc += __ldg(buf + (size_t)s * 8);
  }
  if (acc == 12345.678f) sink[t] = acc;
}

// DAS-shaped gather: each warp picks a random window start; lane l reads word
// start + 3*l + (r & 3) (stride ~3, as 32 z-adjacent pixels of one A-scan).
__global__ void l2_das_gather(const float *__restrict__ buf, uint32_t word_mask, int iters,
                              float *__restrict__ sink) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t w = t >> 5, lane = t & 31;
  float acc = 0.0f;
#pragma unroll 8
  for (int r = 0; r < iters; r++) {
    uint32_t start = (hash32(w * 0x9e3779b9U + (uint32_t)r * 0x85ebca6bU) & word_mask) & ~31u;
    acc += __ldg(buf + ((start + 3 * lane + (r & 3)) & word_mask));
  }
  if (acc == 12345.678f) sink[t] = acc;
}

__global__ void fp32_fma(int iters, float *__restrict__ sink) {
  float a[8];
#pragma unroll
  for (int j = 0; j < 8; j++) a[j] = threadIdx.x * 1e-3f + j;
  for (int r = 0; r < iters; r++) {
#pragma unroll
    for (int j = 0; j < 8; j++) a[j] = fmaf(a[j], 0.999f, 0.001f);
  }
  float s = 0.0f;
#pragma unroll
  for (int j = 0; j < 8; j++) s += a[j];
  if (s == 12345.678f) sink[threadIdx.x] = s;
}

__global__ void fp64_fma(int iters, float *__restrict__ sink) {
  double a[8];
#pragma unroll
  for (int j = 0; j < 8; j++) a[j] = threadIdx.x * 1e-3 + j;
  for (int r = 0; r < iters; r++) {
#pragma unroll
    for (int j = 0; j < 8; j++) a[j] = fma(a[j], 0.999, 0.001);
  }
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < 8; j++) s += a[j];
  if (s == 12345.678) sink[threadIdx.x] = (float)s;
}

__global__ void int_add(int iters, float *__restrict__ sink) {
  uint32_t a[8];
#pragma unroll
  for (int j = 0; j < 8; j++) a[j] = threadIdx.x + j;
  for (int r = 0; r < iters; r++) {
#pragma unroll
    for (int j = 0; j < 8; j++) a[j] = (a[j] ^ 0x5bd1e995u) + 0x9e3779b9u;  // two ALU operations, 8 chains
  }
  uint32_t s = 0;
#pragma unroll
  for (int j = 0; j < 8; j++) s += a[j];
  if (s == 0x12345678u) sink[threadIdx.x] = (float)s;
}

}  // namespace

extern "C" {

// kind: 0 l2_sector_gather, 1 l2_das_gather, 2 fp32_fma, 3 fp64_fma, 4 int_add.
// buf: device buffer of 2^log2_words floats (kinds 0, 1). Returns the kernel
// time in ms (CUDA events) or a negative value on error; *ops receives the
// operation count (loads, FMAs or adds).
double dream_peaks_run(int kind, const float *buf, int log2_words, int blocks, int threads, int iters,
                       float *sink, double *ops) {
  cudaEvent_t a, b;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) return -1.0;
  const uint32_t words = 1u << log2_words;
  cudaEventRecord(a);
  switch (kind) {
    case 0: l2_sector_gather<<<blocks, threads>>>(buf, (words / 8) - 1, iters, sink); break;
    case 1: l2_das_gather<<<blocks, threads>>>(buf, words - 1, iters, sink); break;
    case 2: fp32_fma<<<blocks, threads>>>(iters, sink); break;
    case 3: fp64_fma<<<blocks, threads>>>(iters, sink); break;
    case 4: int_add<<<blocks, threads>>>(iters, sink); break;
    default: return -2.0;
  }
  cudaEventRecord(b);
  if (cudaEventSynchronize(b) != cudaSuccess) return -3.0;
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  const double n = (double)blocks * threads * iters;
  *ops = (kind <= 1) ? n : (kind == 4 ? n * 16.0 : n * 8.0);
  return cudaGetLastError() == cudaSuccess ? (double)ms : -4.0;
}

}  // extern "C"
