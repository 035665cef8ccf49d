// conv_p.cu -- column-wise full linear convolution on the GPU: the conv_p /
// fftconv_p step of DREAM that turns spatial impulse responses into A-scans
// (extra_src/conv.cc:34-78, extra_src/fftconv_p.cc, extra_src/oct_conv_p.cc).
//
//   Y[:, n] (=|+=|-=) A[:, n] * B[:, n or 0]     Y has A_M + B_M - 1 rows
//
// Exactness. The reference's direct form adds zr[i+j] += xr[i]*yr[j] with i
// outer, so output k receives its products in ascending i (= descending j),
// each product rounded, then added. The kernels keep that order per output
// and never fuse the product into the add, so they reproduce conv()
// bit for bit; FFTW's fftconv_p differs from it by rounding only.
//
// Layout. A CTA owns 4 warps x 32 lanes x R consecutive outputs of one
// column; its window of A (outputs + B_M - 1 samples, zero outside the
// column) and B are staged in shared memory. Lane l of warp w holds outputs
// k = k_w + R*l + r. Stepping j downwards, lane l needs A[k_w + R*l + r - j]:
// a window of R samples that slides by one per step. Steps go in groups of
// R: the lane loads the group's R new A samples and R B samples (broadcasts)
// up front, then does R x R products and adds from registers, so the only
// serial latency is each output's FP64 add (8 cycles). A warp skips the
// steps in which all its outputs would only meet samples outside the column
// (the triangle ends of a long-by-long convolution).
//
// '+=' / '-=' add into existing values; out-of-column terms then contribute
// the exact neutral element (-0 for +=, +0 for -=), so a stored -0 stays -0
// exactly as in the reference, which never visits those terms.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "das_common.cuh"
#include "das_kernels.h"
#include "dream_conv.h"

namespace dream {
namespace {

constexpr int CONV_WARPS = 4;  // small CTAs: long pulses leave few tiles per column
constexpr int CONV_R = 8;                                   // outputs per lane
constexpr int CONV_T = CONV_WARPS * 32 * CONV_R;            // outputs per CTA
constexpr int64_t CONV_LMAX = 8192;                         // B samples staged in shared memory

// A-window slots: CONV_T + L samples plus 2R read ahead by the last groups.
__host__ __device__ constexpr int64_t conv_window(int64_t L) { return CONV_T + L + 2 * CONV_R; }

// Shared-memory position of window sample q: one pad slot per 16 samples, so
// the 32 lanes' reads at a stride of R samples fall in distinct banks (two
// wavefronts per warp, the minimum for 8-byte values).
__host__ __device__ constexpr int64_t conv_sw(int64_t q) { return q + (q >> 4); }

__host__ __device__ constexpr size_t conv_smem_bytes(int64_t L) {
  return (size_t)(L + conv_sw(conv_window(L)) + 1) * sizeof(double);  // B, then the A window
}

template <int MODE>
__device__ __forceinline__ double conv_acc(double acc, double prod) {
  return MODE == 2 ? __dsub_rn(acc, prod) : __dadd_rn(acc, prod);
}

// R steps of R outputs: acc[r] (op)= A[i0 + r + s0 + u] * B[L-1-s0-u] for
// u = 0..R-1 in that order, with the A samples in cur (t < R) and nxt.
// FULL groups have all R steps inside [s0, s_end).
template <int MODE, bool FULL>
__device__ __forceinline__ void conv_group(double (&acc)[CONV_R], const double (&cur)[CONV_R],
                                           const double (&nxt)[CONV_R], const double (&yv)[CONV_R], int64_t s0,
                                           int64_t s_end, int64_t i0, int64_t M, double neutral) {
#pragma unroll
  for (int u = 0; u < CONV_R; u++) {
    if (!FULL && s0 + u >= s_end) break;  // uniform across the warp
#pragma unroll
    for (int r = 0; r < CONV_R; r++) {
      const double xv = (r + u < CONV_R) ? cur[r + u] : nxt[r + u - CONV_R];
      double prod = __dmul_rn(xv, yv[u]);
      if (MODE != 0) {
        const int64_t i = i0 + r + s0 + u;
        if (i < 0 || i >= M) prod = neutral;
      }
      acc[r] = conv_acc<MODE>(acc[r], prod);
    }
  }
}

// Tile launched at grid position y, centre-out: the middle tiles, whose
// outputs have the longest sums, first (mid, mid+1, mid-1, mid+2, ...), so
// the block scheduler spreads them over all SMs before the short ones.
__device__ __forceinline__ int64_t centre_out_tile(int64_t y, int64_t n) {
  const int64_t m = n / 2, hi = n - 1 - m;  // tiles above the middle (hi <= m)
  if (y == 0) return m;
  if (y <= 2 * hi) return (y & 1) ? m + (y + 1) / 2 : m - y / 2;
  return m - (y - hi);
}

// Column n of the output convolves A column n % na with B column n / nb
// (na = N, nb = 1 for fftconv_p / conv_p; the full-matrix-capture synthesis
// pairs every receive column with every transmit column).
template <int MODE>
__global__ void __launch_bounds__(CONV_WARPS * 32) conv_p_kernel(const double *__restrict__ A, int64_t M, int64_t N,
                                                                  const double *__restrict__ B, int64_t L,
                                                                  int64_t ldb, double *__restrict__ Y, int64_t NY,
                                                                  int64_t na, int64_t nb) {
  extern __shared__ __align__(16) double conv_sm[];
  double *ys = conv_sm;      // [L]
  double *xs = conv_sm + L;  // xs[conv_sw(q)] = A[k_cta - (L - 1) + q] (0 outside the column)
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t k_cta = centre_out_tile(blockIdx.y, gridDim.y) * CONV_T;
  const int64_t base = k_cta - (L - 1);
  const int64_t W = conv_window(L);
  const double neutral = MODE == 2 ? 0.0 : -0.0;
  for (int64_t n = blockIdx.x; n < N; n += gridDim.x) {
    const double *x = A + (n % na) * M;
    const double *y = B + (n / nb) * ldb;
    double *z = Y + n * NY;
    __syncthreads();  // the previous column's window is no longer read
    for (int64_t q = tid; q < L; q += blockDim.x) ys[q] = y[q];
    for (int64_t q = tid; q < W; q += blockDim.x) {
      const int64_t i = base + q;
      xs[conv_sw(q)] = (i >= 0 && i < M) ? x[i] : 0.0;
    }
    __syncthreads();
    const int q0 = warp * 32 * CONV_R + CONV_R * lane;  // window start of this lane at step s = 0
    // step s = L-1-j: output k_r takes A[i], i = base + q0 + r + s (xs index q0 + r + s).
    // Steps where every output of the warp sees only samples outside the
    // column contribute nothing (neutral terms) and are skipped: the warp's
    // samples span i in [k_w - (L-1) + s, k_w + 32R - 1 - (L-1) + s].
    const int64_t k_w = k_cta + warp * 32 * CONV_R;
    const int64_t s_begin = std::max<int64_t>(0, (L - 1) - (k_w + 32 * CONV_R - 1));
    const int64_t s_end = std::min<int64_t>(L, M + (L - 1) - k_w);
    // group of R steps starting at s0: lane sample t (0 <= t < 2R) is
    // window sample q0 + s0 + t; the B samples are ys[L-1-s0-u]
    auto xsamp = [&](int64_t t) { return xs[conv_sw(q0 + t)]; };
    auto bsamp = [&](int64_t s) { return ys[std::max<int64_t>(L - 1 - s, 0)]; };  // clamped past the end, unused
    // A samples in three buffers (the group's, the next group's, the one after
    // being loaded), B samples in two; six groups per loop trip make every
    // buffer's role fixed, so nothing is copied between groups.
    double acc[CONV_R], X0[CONV_R], X1[CONV_R], X2[CONV_R], Y0[CONV_R], Y1[CONV_R];
#pragma unroll
    for (int r = 0; r < CONV_R; r++) {
      const int64_t k = k_cta + q0 + r;
      acc[r] = MODE == 0 ? 0.0 : (k < NY ? z[k] : 0.0);
      X0[r] = xsamp(s_begin + r);
      X1[r] = xsamp(s_begin + CONV_R + r);
      Y0[r] = bsamp(s_begin + r);
    }
    // One group: the following group's samples are loaded first (they do not
    // depend on the sums, so their latency overlaps this group's arithmetic),
    // then R x R products and adds; only each output's FP64 add is serial.
    auto group = [&](int64_t s0, const double(&cur)[CONV_R], const double(&nxt)[CONV_R], double(&load)[CONV_R],
                     const double(&yv)[CONV_R], double(&yload)[CONV_R]) {
#pragma unroll
      for (int u = 0; u < CONV_R; u++) {
        load[u] = xsamp(std::min<int64_t>(s0 + 2 * CONV_R + u, W - 1 - q0));
        yload[u] = bsamp(s0 + CONV_R + u);
      }
      if (s0 + CONV_R <= s_end)  // a full group: no exit test between the steps
        conv_group<MODE, true>(acc, cur, nxt, yv, s0, s_end, base + q0, M, neutral);
      else
        conv_group<MODE, false>(acc, cur, nxt, yv, s0, s_end, base + q0, M, neutral);
    };
    for (int64_t s0 = s_begin; s0 < s_end;) {
      group(s0, X0, X1, X2, Y0, Y1);
      if ((s0 += CONV_R) >= s_end) break;
      group(s0, X1, X2, X0, Y1, Y0);
      if ((s0 += CONV_R) >= s_end) break;
      group(s0, X2, X0, X1, Y0, Y1);
      if ((s0 += CONV_R) >= s_end) break;
      group(s0, X0, X1, X2, Y1, Y0);
      if ((s0 += CONV_R) >= s_end) break;
      group(s0, X1, X2, X0, Y0, Y1);
      if ((s0 += CONV_R) >= s_end) break;
      group(s0, X2, X0, X1, Y1, Y0);
      s0 += CONV_R;
    }
#pragma unroll
    for (int r = 0; r < CONV_R; r++) {
      const int64_t k = k_cta + q0 + r;
      if (k < NY) z[k] = acc[r];
    }
  }
}

// Pulses longer than the shared-memory budget: one output per thread, the
// same order of operations, operands from global memory (L1/L2).
template <int MODE>
__global__ void __launch_bounds__(256) conv_p_global_kernel(const double *__restrict__ A, int64_t M, int64_t N,
                                                             const double *__restrict__ B, int64_t L, int64_t ldb,
                                                             double *__restrict__ Y, int64_t NY, int64_t na,
                                                             int64_t nb) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t n = blockIdx.y; n < N; n += gridDim.y) {
    if (k >= NY) continue;
    const double *x = A + (n % na) * M;
    const double *y = B + (n / nb) * ldb;
    double acc = MODE == 0 ? 0.0 : Y[n * NY + k];
    const int64_t i_lo = std::max<int64_t>(0, k - (L - 1)), i_hi = std::min<int64_t>(M - 1, k);
    for (int64_t i = i_lo; i <= i_hi; i++) acc = conv_acc<MODE>(acc, __dmul_rn(__ldg(x + i), __ldg(y + (k - i))));
    Y[n * NY + k] = acc;
  }
}

template <int MODE>
cudaError_t launch_mode(const double *A, int64_t M, int64_t N, const double *B, int64_t L, int64_t ldb, double *Y,
                        int64_t NY, cudaStream_t st, int64_t na, int64_t nb) {
  const unsigned gy = (unsigned)std::min<int64_t>(N, 65535);
  if (L <= CONV_LMAX && (NY + CONV_T - 1) / CONV_T <= 65535) {
    const size_t smem = conv_smem_bytes(L);
    cudaError_t e = ensure_smem(conv_p_kernel<MODE>, smem);
    if (e != cudaSuccess) return e;
    // x: columns (fastest, so every column's middle tile launches before any
    // column's edge tiles), y: tiles in centre-out order
    dim3 grid((unsigned)std::min<int64_t>(N, 1 << 30), (unsigned)((NY + CONV_T - 1) / CONV_T));
    conv_p_kernel<MODE><<<grid, CONV_WARPS * 32, smem, st>>>(A, M, N, B, L, ldb, Y, NY, na, nb);
  } else {
    dim3 grid((unsigned)((NY + 255) / 256), gy);
    conv_p_global_kernel<MODE><<<grid, 256, 0, st>>>(A, M, N, B, L, ldb, Y, NY, na, nb);
  }
  return cudaGetLastError();
}

// Shapes after the reference's rules (python/include/py_fftconv_p.hpp:70-77,
// extra_src/oct_conv_p.cc:225-236): B a vector (either orientation) for every
// column, or a matrix with A_N columns.
int conv_shapes(int64_t A_M, int64_t A_N, int64_t &B_M, int64_t &B_N, int mode) {
  if (A_M < 0 || A_N < 0 || B_M < 0 || B_N < 0) return set_last_error(DREAM_ERR_ARGUMENT, "negative dimension");
  if (mode != DREAM_CONV_EQU && mode != DREAM_CONV_SUM && mode != DREAM_CONV_NEG)
    return set_last_error(DREAM_ERR_ARGUMENT, "Non-valid string in arg 4!");
  if (B_M != 1 && B_N != 1 && B_N != A_N)
    return set_last_error(DREAM_ERR_ARGUMENT,
                          "Argument 2 must be a vector or a matrix with the same number of columns as arg 1!");
  if (B_M == 1 || B_N == 1) {
    B_M = B_M * B_N;
    B_N = 1;
  }
  return 0;
}

int conv_device(const double *dA, int64_t A_M, int64_t A_N, const double *dB, int64_t B_M, int64_t B_N, double *dY,
                int mode, cudaStream_t st) {
  const int64_t NY = A_M + B_M - 1;
  if (A_N == 0 || NY <= 0) return 0;
  if (dY == nullptr) return set_last_error(DREAM_ERR_ARGUMENT, "NULL output pointer");
  if (A_M == 0 || B_M == 0) {  // no products: '=' clears, '+=' and '-=' leave Y as it is
    if (mode == DREAM_CONV_EQU) {
      cudaError_t e = cudaMemsetAsync(dY, 0, (size_t)NY * A_N * sizeof(double), st);
      if (e != cudaSuccess) return set_last_error(DREAM_ERR_CUDA, cudaGetErrorString(e));
    }
    return 0;
  }
  if (dA == nullptr || dB == nullptr) return set_last_error(DREAM_ERR_ARGUMENT, "NULL input pointer");
  const int64_t ldb = B_N > 1 ? B_M : 0;
  cudaError_t e = mode == DREAM_CONV_EQU   ? launch_mode<0>(dA, A_M, A_N, dB, B_M, ldb, dY, NY, st, A_N, 1)
                  : mode == DREAM_CONV_SUM ? launch_mode<1>(dA, A_M, A_N, dB, B_M, ldb, dY, NY, st, A_N, 1)
                                           : launch_mode<2>(dA, A_M, A_N, dB, B_M, ldb, dY, NY, st, A_N, 1);
  if (e != cudaSuccess) return set_last_error(DREAM_ERR_CUDA, std::string("conv_p launch: ") + cudaGetErrorString(e));
  return 0;
}

// Device buffers of the host-pointer entry, kept per device and grown on demand.
struct ConvBuffers {
  std::mutex mu;
  double *A = nullptr, *B = nullptr, *Y = nullptr;
  size_t cap_a = 0, cap_b = 0, cap_y = 0;
  cudaStream_t st = nullptr;
};

int grow(double *&p, size_t &cap, size_t bytes) {
  if (bytes <= cap) return 0;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_last_error(DREAM_ERR_ALLOC, "conv_p: device allocation failed");
  }
  cap = bytes;
  return 0;
}

}  // namespace
}  // namespace dream

using namespace dream;

extern "C" {

int dream_conv_p_run_device(const double *dA, int64_t A_M, int64_t A_N, const double *dB, int64_t B_M, int64_t B_N,
                            double *dY, int mode, void *stream) {
  DREAM_API_TRY
  int r = conv_shapes(A_M, A_N, B_M, B_N, mode);
  if (r) return r;
  return conv_device(dA, A_M, A_N, dB, B_M, B_N, dY, mode, (cudaStream_t)stream);
  DREAM_API_CATCH
}

int dream_conv_p_run(const double *A, int64_t A_M, int64_t A_N, const double *B, int64_t B_M, int64_t B_N, double *Y,
                     int mode, int device) {
  DREAM_API_TRY
  int r = conv_shapes(A_M, A_N, B_M, B_N, mode);
  if (r) return r;
  const int64_t NY = A_M + B_M - 1;
  if (A_N == 0 || NY <= 0) return 0;
  if (Y == nullptr || (A_M > 0 && A == nullptr) || (B_M > 0 && B == nullptr))
    return set_last_error(DREAM_ERR_ARGUMENT, "NULL host pointer");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return set_last_error(DREAM_ERR_ARGUMENT, "invalid CUDA device ordinal");
  static std::vector<ConvBuffers> bufs(64);
  if (device >= (int)bufs.size()) return set_last_error(DREAM_ERR_ARGUMENT, "invalid CUDA device ordinal");
  ConvBuffers &cb = bufs[device];
  std::lock_guard<std::mutex> lk(cb.mu);
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != device) cudaSetDevice(device);
  auto done = [&](int code) {
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
    return code;
  };
  cudaError_t e = cudaSuccess;
  if (cb.st == nullptr && (e = cudaStreamCreateWithFlags(&cb.st, cudaStreamNonBlocking)) != cudaSuccess)
    return done(set_last_error(DREAM_ERR_CUDA, cudaGetErrorString(e)));
  const size_t na = (size_t)A_M * A_N, nb = (size_t)B_M * B_N, ny = (size_t)NY * A_N;
  if ((r = grow(cb.A, cb.cap_a, std::max<size_t>(na, 1) * 8)) || (r = grow(cb.B, cb.cap_b, std::max<size_t>(nb, 1) * 8)) ||
      (r = grow(cb.Y, cb.cap_y, ny * 8)))
    return done(r);
  if (na) e = cudaMemcpyAsync(cb.A, A, na * 8, cudaMemcpyHostToDevice, cb.st);
  if (e == cudaSuccess && nb) e = cudaMemcpyAsync(cb.B, B, nb * 8, cudaMemcpyHostToDevice, cb.st);
  if (e == cudaSuccess && mode != DREAM_CONV_EQU) e = cudaMemcpyAsync(cb.Y, Y, ny * 8, cudaMemcpyHostToDevice, cb.st);
  if (e != cudaSuccess) return done(set_last_error(DREAM_ERR_CUDA, cudaGetErrorString(e)));
  if ((r = conv_device(cb.A, A_M, A_N, cb.B, B_M, B_N, cb.Y, mode, cb.st))) return done(r);
  e = cudaMemcpyAsync(Y, cb.Y, ny * 8, cudaMemcpyDeviceToHost, cb.st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(cb.st);
  if (e != cudaSuccess) return done(set_last_error(DREAM_ERR_CUDA, cudaGetErrorString(e)));
  return done(0);
  DREAM_API_CATCH
}

int dream_conv_p_fmc_device(const double *dHt, int64_t M, int64_t L_t, const double *dHr, int64_t L_r,
                            const double *dP, int64_t P_M, double *dDP, double *dY, void *stream) {
  DREAM_API_TRY
  if (M <= 0 || L_t < 0 || L_r < 0 || P_M <= 0)
    return set_last_error(DREAM_ERR_ARGUMENT, "fmc synthesis: M and the pulse length must be positive");
  const int64_t N = L_t * L_r;
  if (N == 0) return 0;
  if (dHt == nullptr || dHr == nullptr || dP == nullptr || dDP == nullptr || dY == nullptr)
    return set_last_error(DREAM_ERR_ARGUMENT, "NULL pointer");
  const cudaStream_t st = (cudaStream_t)stream;
  const int64_t NY1 = 2 * M - 1, NY2 = NY1 + P_M - 1;
  // double path: column t*L_r + r = Hr[:, r] (*) Ht[:, t]; then every column (*) the pulse
  cudaError_t e = launch_mode<0>(dHr, M, N, dHt, M, M, dDP, NY1, st, L_r, L_r);
  if (e == cudaSuccess) e = launch_mode<0>(dDP, NY1, N, dP, P_M, 0, dY, NY2, st, N, 1);
  if (e != cudaSuccess) return set_last_error(DREAM_ERR_CUDA, std::string("fmc synthesis launch: ") + cudaGetErrorString(e));
  return 0;
  DREAM_API_CATCH
}

}  // extern "C"
