// das_common.cuh -- device helpers shared by the DAS kernels (sm_100a).
//
// Exact arithmetic: every product, sum and square root that feeds a sample
// index goes through the round-to-nearest intrinsics, so nvcc never fuses a
// multiply and an add (an FMA would change the rounding and hence, at times,
// the selected sample). Square roots are the IEEE correctly rounded ones,
// which is what std::sqrt gives the reference CPU code.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <utility>

namespace dream {

enum Method : int { SAFT = 0, TFM = 1, RCA_COLTX = 2, RCA_ROWTX = 3 };

template <class T>
struct Ar;

template <>
struct Ar<double> {
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double sqrt(double a) { return __dsqrt_rn(a); }
};

template <>
struct Ar<float> {
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float sqrt(float a) { return __fsqrt_rn(a); }
};

// |g - r| / cp with the reference association ((dx*dx + dy*dy) + dz*dz).
template <class T>
__device__ __forceinline__ T leg_time(T gx, T gy, T gz, T one_over_cp) {
  using A = Ar<T>;
  T ss = A::add(A::add(A::mul(gx, gx), A::mul(gy, gy)), A::mul(gz, gz));
  return A::mul(A::sqrt(ss), one_over_cp);
}

// Truncation toward zero of p, for p already known to lie in (-1, K):
// that is floor(max(p, 0)). Adding 2^52 (2^23 for float) with round-toward-
// zero leaves floor(x) in the low mantissa bits for 0 <= x < 2^52 (2^23),
// which avoids the slow float->int conversion unit.
__device__ __forceinline__ int trunc_index(double p) {
  double v = __dadd_rz(fmax(p, 0.0), 4503599627370496.0);  // 2^52
  return __double2loint(v);
}
__device__ __forceinline__ int trunc_index(float p) {
  float v = __fadd_rz(fmaxf(p, 0.0f), 8388608.0f);  // 2^23
  return __float_as_int(v) - 0x4B000000;
}

// Bounds-checked builds (nvcc -DDREAM_DAS_CHECKED, `python -m dream_b200.build
// --checked`): every A-scan gather verifies its element index against the
// buffer's extent; a violation is counted in *bad and the load is skipped.
// The normal build compiles this to the plain load.
template <class T>
__device__ __forceinline__ bool gather_ok(int64_t i, int64_t n, unsigned long long *bad) {
#ifdef DREAM_DAS_CHECKED
  if (i < 0 || i >= n) {
    if (bad) atomicAdd(bad, 1ull);
    return false;
  }
#endif
  return true;
}

// Warp-aggregated add of a per-thread count to a global counter. Must be
// called by all 32 lanes of the warp.
__device__ __forceinline__ void add_count(unsigned long long *ctr, unsigned int v) {
  unsigned int s = __reduce_add_sync(0xffffffffu, v);
  if (ctr != nullptr && (threadIdx.x & 31) == 0 && s) atomicAdd(ctr, (unsigned long long)s);
}

// Raises a kernel's dynamic shared-memory limit once per (kernel, device):
// later launches (including ones being captured into a CUDA graph) then issue
// no attribute call.
template <class F>
inline cudaError_t ensure_smem(F *kernel, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, size_t> done;
  if (bytes <= 48 * 1024) return cudaSuccess;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  auto key = std::make_pair(reinterpret_cast<const void *>(kernel), dev);
  auto it = done.find(key);
  if (it != done.end() && it->second >= bytes) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) done[key] = bytes;
  return e;
}

}  // namespace dream
