// das_kernels.h -- launch descriptors shared by the C ABI (das_capi.cu) and
// the kernel translation units. Host-side only types.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace dream {

// Per-call constants, computed on the host exactly as the restated reference
// source computes them (see das_capi.cu: constants_*).
struct Consts64 {
  double Fs, ocp, delay_ms;
};
struct Consts32 {
  float Fs, ocp, delay_ms;
};

// Warp patch of the plain kernels under a grid hint: PLAIN_PATCH_F points
// along the grid's fast axis x (32 / PLAIN_PATCH_F) along the slow one.
constexpr int PLAIN_PATCH_F = 8;
constexpr int PLAIN_PATCH_S = 32 / PLAIN_PATCH_F;

struct PlainLaunch {
  int method;  // 0 SAFT, 1 TFM, 2 RCA col-tx, 3 RCA row-tx
  bool uni;
  const void *Y;
  int64_t K;
  const void *Ro;
  int64_t No;
  int64_t no0, no1;  // pixel range of this launch (patch-row range when n_fast > 0)
  int64_t n_fast;    // grid hint: points along the grid's fast axis (0: none)
  const void *Gt;
  int64_t Nt;
  const void *Gr;
  int64_t Nr;
  const void *delay_vec;  // device delays (us): 1 value, or No values when delay_multi
  bool delay_multi;
  Consts64 c64;
  Consts32 c32;
  double tri64[15];
  float tri32[15];
  int64_t Nx, Ny, Nz;
  void *Im;
  unsigned long long *oob;
  int64_t ny;               // elements in Y
  unsigned long long *bad;  // gather index violations (bounds-checked builds)
  int64_t *idx;             // non-NULL: write the sample indices instead of the image
};

cudaError_t launch_plain_f64(const PlainLaunch &L, cudaStream_t st);

// Records msg as this host thread's last error (dream_das_last_error) and
// returns code.
int set_last_error(int code, const std::string &msg);

// The status of the C++ exception being handled (call only inside a catch
// block): DREAM_ERR_ALLOC for std::bad_alloc, DREAM_ERR_ARGUMENT otherwise,
// with its message recorded. Every int-returning C ABI entry wraps its body in
// DREAM_API_TRY ... DREAM_API_CATCH, so no exception crosses the C boundary.
int api_exception() noexcept;
#define DREAM_API_TRY try {
#define DREAM_API_CATCH \
  }                     \
  catch (...) {         \
    return ::dream::api_exception(); \
  }
cudaError_t launch_plain_f32(const PlainLaunch &L, cudaStream_t st);

}  // namespace dream
