// das_capi.cu -- the C ABI declared in include/dream_das.h.
//
// A plan plays the role of the reference's cached DAS<T> / DAS_UNI<T> object
// (include/das.h:52-94, include/das_uni.h:50-64): it remembers the setup,
// owns the device buffers the host-pointer entry points stage through, an
// out-of-bounds counter and a stream. Argument checks follow the reference
// bindings (python/include/py_das.hpp:53-148, include/arg_parser.h:236-290).
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dream_das.h"
#include "das_fast.h"
#include <exception>
#include <new>

#include "das_kernels.h"

using namespace dream;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char *where) {
  g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
  return DREAM_ERR_CUDA;
}

#define CU(call)                                       \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

struct DeviceGuard {
  int prev = -1;
  bool ok = true;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) ok = cudaSetDevice(dev) == cudaSuccess;
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes) {
    if (bytes <= cap) return 0;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    if (bytes == 0) return 0;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(DREAM_ERR_ALLOC, std::string("device allocation of ") + std::to_string(bytes) +
                                       " bytes failed: " + cudaGetErrorString(e));
    }
    cap = bytes;
    return 0;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

int status_from_oob(uint64_t oob, int err_level) {
  if (oob == 0) return DREAM_STATUS_NONE;
  switch (err_level) {  // src/dream_error.cc:40-76
    case DREAM_ERR_LEVEL_IGNORE: return DREAM_STATUS_IGNORE_OUT_OF_BOUNDS;
    case DREAM_ERR_LEVEL_WARN: return DREAM_STATUS_WARN_OUT_OF_BOUNDS;
    case DREAM_ERR_LEVEL_STOP:
    case DREAM_ERR_LEVEL_PARALLEL_STOP: return DREAM_STATUS_OUT_OF_BOUNDS;
    default: return DREAM_STATUS_NONE;
  }
}

}  // namespace

int dream::set_last_error(int code, const std::string &msg) { return fail(code, msg); }

int dream::api_exception() noexcept {
  int code = DREAM_ERR_ARGUMENT;
  const char *msg = "unexpected C++ exception";
  try {
    throw;
  } catch (const std::bad_alloc &) {
    code = DREAM_ERR_ALLOC;
    msg = "host memory allocation failed";
  } catch (const std::exception &e) {
    msg = e.what();
  } catch (...) {
  }
  try {
    g_last_error = msg;
  } catch (...) {  // no memory even for the message: keep the old one
  }
  return code;
}

struct dream_das_plan {
  int das_type = 0;
  int64_t K = 0, No = 0, Nt = 0, Nr = 0;
  int precision = 0;
  int device = 0;
  bool uni = false;
  double tri[15] = {0};
  int64_t Nx = 0, Ny = 0, Nz = 0;
  cudaStream_t stream = nullptr;
  DevBuf bY, bRo, bGt, bGr, bDelay, bIm, bOob, bY16;
  int64_t n_fast = 0;          // grid hint (0: none)
  int tile_f = 0, tile_s = 0;  // user / autotuner tile (0: automatic)
  int jc = 0;                  // user / autotuner inner chunk (0: automatic)
  int64_t l2_block = 0;        // A-scan bytes per inner-element pass (0: automatic, < 0: never split)
  // inner-element shard: Y holds only inner elements [shard_lo, shard_hi) (0, 0: all of them)
  int64_t shard_lo = 0, shard_hi = 0;
  // host-pointer runs of FP32/BF16-storage plans: A-scan upload stream
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t chunk_ev[16] = {nullptr};  // [0, 15): upload chunks, [15]: fence on the previous call
  // geometry-bound operator
  bool bound = false;
  FastParams geo{};
  DevBuf bScatter;  // unweighted scatter of the weight gradient (bound operator)
  DevBuf bBad;  // gather index violations (bounds-checked builds only)
  int sm_count = 148;
  unsigned long long *h_oob = nullptr;  // pinned
  void *h_stage = nullptr;  // pinned staging of host image read-backs
  size_t h_stage_bytes = 0;
  std::atomic<bool> cancelled{false};
  std::atomic<int64_t> launches{0};
  std::mutex mu;
};

namespace {

size_t prec_size(int prec) { return prec == DREAM_PREC_F64 ? 8 : 4; }

bool is_fast(const dream_das_plan *p) {
  return p->precision == DREAM_PREC_F32_STORE || p->precision == DREAM_PREC_BF16_STORE;
}
// element sizes: Y as passed on the device, geometry, image
size_t y_dev_size(const dream_das_plan *p) {
  return p->precision == DREAM_PREC_F64 ? 8 : (p->precision == DREAM_PREC_BF16_STORE ? 2 : 4);
}
size_t geo_size(const dream_das_plan *p) { return p->precision == DREAM_PREC_F32 ? 4 : 8; }
size_t im_size(const dream_das_plan *p) { return p->precision == DREAM_PREC_F64 ? 8 : 4; }

int check_common(int das_type, int64_t K, int64_t No, int64_t Nt, int64_t Nr, int precision) {
  if (das_type < DREAM_DAS_SAFT || das_type > DREAM_DAS_RCA_ROWTX)
    return fail(DREAM_ERR_ARGUMENT, "Unknown delay-and-sum method!");
  if (K < 0 || No < 0 || Nt < 0 || Nr < 0) return fail(DREAM_ERR_ARGUMENT, "negative size");
  if (precision < DREAM_PREC_F64 || precision > DREAM_PREC_BF16_STORE)
    return fail(DREAM_ERR_ARGUMENT, "unknown precision");
  if (K > INT32_MAX) return fail(DREAM_ERR_ARGUMENT, "A-scan length must be below 2^31 samples");
  if (precision == DREAM_PREC_F32 && K > (int64_t(1) << 24))
    return fail(DREAM_ERR_ARGUMENT, "FP32 plans need A-scans of at most 2^24 samples");
  if (Nt > INT32_MAX || Nr > INT32_MAX) return fail(DREAM_ERR_ARGUMENT, "too many elements");
  return 0;
}

// RCA stripe edges are read as Gr[Nt], Gr[2*Nt-1], Gt[0], Gt[Nr-1]
// (extra_src/das.cc:464-467); these must lie inside the 3*Nr and 3*Nt arrays.
int check_rca_edges(int64_t Nt, int64_t Nr) {
  if (Nt < 1 || Nr < 1) return fail(DREAM_ERR_ARGUMENT, "RCA needs at least one column and one row");
  if (2 * Nt - 1 >= 3 * Nr || Nr - 1 >= 3 * Nt)
    return fail(DREAM_ERR_ARGUMENT,
                "RCA stripe edges would be read outside Gt/Gr (the reference reads "
                "Gr[num_cols], Gr[2*num_cols-1] and Gt[num_rows-1])");
  return 0;
}

int effective_method(const dream_das_plan *p) { return p->Nr == 0 ? DREAM_DAS_SAFT : p->das_type; }

int64_t terms_per_pixel(const dream_das_plan *p) {
  return effective_method(p) == DREAM_DAS_SAFT ? p->Nt : p->Nt * p->Nr;
}

int64_t num_columns(const dream_das_plan *p) { return terms_per_pixel(p); }

// Constants of DAS<double> / DAS<float> (extra_src/das.cc:316-318) and of the
// das_uni float kernels (opencl/das_uni_float.cl:47-49).
Consts64 constants_f64(double dt, double cp, double delay) {
  Consts64 c;
  c.Fs = (1.0 / dt) * 1000.0;
  c.ocp = 1.0 / cp;
  c.delay_ms = delay / 1000.0;
  return c;
}
Consts32 constants_das_f32(float dt, float cp, float delay) {
  Consts32 c;
  c.Fs = (float)((1.0 / (double)dt) * 1000.0);
  c.ocp = (float)(1.0 / (double)cp);
  c.delay_ms = (float)((double)delay / 1000.0);
  return c;
}
Consts32 constants_uni_f32(float dt, float cp, float delay) {
  Consts32 c;
  c.Fs = (1.0f / dt) * 1000.0f;
  c.ocp = 1.0f / cp;
  c.delay_ms = delay / 1000.0f;
  return c;
}

// (int)((max - min)/d + 1.0) in the plan precision (include/das_uni.h:70-78).
int64_t uni_count(double mn, double d, double mx, bool f32) {
  double q;
  if (f32) {
    float qf = ((float)mx - (float)mn) / (float)d;
    q = (double)qf + 1.0;
  } else {
    q = (mx - mn) / d + 1.0;
  }
  if (!(q >= 0.0) || q > 2147483647.0) return -1;
  return (int64_t)(int)q;
}

#ifdef DREAM_DAS_CHECKED
constexpr bool kChecked = true;
#else
constexpr bool kChecked = false;
#endif

// Device counter of gather indices outside Y (bounds-checked builds; NULL in
// the normal build, whose kernels never test the index).
unsigned long long *bad_counter(dream_das_plan *p) {
  if (!kChecked) return nullptr;
  if (p->bBad.p == nullptr) {
    if (p->bBad.ensure(sizeof(unsigned long long))) return nullptr;
    if (cudaMemset(p->bBad.p, 0, sizeof(unsigned long long)) != cudaSuccess) return nullptr;
  }
  return (unsigned long long *)p->bBad.p;
}

int launch_plain(dream_das_plan *p, PlainLaunch &L, cudaStream_t st) {
  L.ny = p->K * num_columns(p);
  L.bad = bad_counter(p);
  // 2-D warp patches for RCA volumes with a grid hint (das_uni: its own
  // grid). On the 128x128-element RCA volume (128x128x256 points) they take
  // plain FP32 from 194.8 to 180.7 ms; on the 64x64-element TFM frame
  // (512x512 points) they cost 4 % (FP64 2.43 -> 2.52 ms), so TFM and SAFT
  // keep warps of consecutive points.
  L.n_fast = 0;
  if (L.method == DREAM_DAS_RCA_COLTX || L.method == DREAM_DAS_RCA_ROWTX) {
    if (L.uni) {
      const int64_t nf = L.Ny > 1 ? L.Ny : L.Ny * L.Nz;
      if (nf >= 8 && L.No % nf == 0 && nf < L.No) L.n_fast = nf;
    } else if (p->n_fast >= 8 && p->n_fast < L.No) {
      L.n_fast = p->n_fast;
    }
  }
  // Pixel chunks keep a cancellation request observable between launches.
  const int64_t tpp = std::max<int64_t>(terms_per_pixel(p), 1);
  int64_t chunk = std::max<int64_t>(int64_t(1) << 16, (int64_t(1) << 33) / tpp);
  chunk = (chunk + 255) / 256 * 256;
  int64_t total = L.No;
  if (L.n_fast > 0) {  // the range is over rows of warp patches (at most 65535 per launch: the grid's y extent)
    total = (L.No / L.n_fast + PLAIN_PATCH_S - 1) / PLAIN_PATCH_S;
    chunk = std::min<int64_t>(65535, std::max<int64_t>(1, chunk / (PLAIN_PATCH_S * L.n_fast)));
  }
  for (int64_t s = 0; s < total; s += chunk) {
    if (p->cancelled.load()) return fail(DREAM_ERR_CANCELLED, "DAS cancelled");
    L.no0 = s;
    L.no1 = std::min(total, s + chunk);
    cudaError_t e = (p->precision == DREAM_PREC_F64) ? launch_plain_f64(L, st) : launch_plain_f32(L, st);
    if (e != cudaSuccess) return cuda_fail(e, "DAS kernel launch");
    p->launches++;
  }
  return 0;
}

// Fill a PlainLaunch for `das` (arbitrary geometry) on device pointers. The
// delay (one value or No values) is read by the kernel from device memory and
// converted to ms there, as DAS<T> does per pixel (extra_src/das.cc:131-136).
int prepare_das(dream_das_plan *p, PlainLaunch &L, const void *dY, const void *dRo, const void *dGt,
                const void *dGr, double dt, int delay_type, const void *ddelay, double cp, void *dIm,
                unsigned long long *doob) {
  memset(&L, 0, sizeof(L));
  L.method = effective_method(p);
  L.uni = false;
  L.Y = dY;
  L.K = p->K;
  L.Ro = dRo;
  L.No = p->No;
  L.Gt = dGt;
  L.Nt = p->Nt;
  L.Gr = dGr;
  L.Nr = (L.method == DREAM_DAS_SAFT) ? 0 : p->Nr;
  L.Im = dIm;
  L.oob = doob;
  if (delay_type != DREAM_DELAY_SINGLE && delay_type != DREAM_DELAY_MULTIPLE)
    return fail(DREAM_ERR_ARGUMENT, "unknown delay type");
  if (ddelay == nullptr) return fail(DREAM_ERR_ARGUMENT, "delay pointer is NULL");
  L.delay_vec = ddelay;
  L.delay_multi = delay_type == DREAM_DELAY_MULTIPLE;
  if (p->precision == DREAM_PREC_F64) L.c64 = constants_f64(dt, cp, 0.0);
  else L.c32 = constants_das_f32((float)dt, (float)cp, 0.0f);
  if (L.method >= DREAM_DAS_RCA_COLTX) {
    int r = check_rca_edges(p->Nt, p->Nr);
    if (r) return r;
  }
  if (p->No > 0 && (dRo == nullptr || dIm == nullptr)) return fail(DREAM_ERR_ARGUMENT, "NULL Ro or Im");
  if (p->No > 0 && p->K > 0 && terms_per_pixel(p) > 0 && dY == nullptr)
    return fail(DREAM_ERR_ARGUMENT, "NULL Y");
  if (p->Nt > 0 && dGt == nullptr) return fail(DREAM_ERR_ARGUMENT, "NULL Gt");
  if (L.Nr > 0 && dGr == nullptr) return fail(DREAM_ERR_ARGUMENT, "NULL Gr");
  return 0;
}

__global__ void add_u64_kernel(unsigned long long *ctr, unsigned long long v) { *ctr += v; }

// K == 0 (or no element pairs) has no in-bounds sample: the image is all
// zeros and every term is out of bounds.
int zero_length_ascans(dream_das_plan *p, void *dIm, unsigned long long *doob, cudaStream_t st) {
  if (p->No > 0) CU(cudaMemsetAsync(dIm, 0, p->No * im_size(p), st));
  unsigned long long oob = (unsigned long long)p->No * (unsigned long long)terms_per_pixel(p);
  if (doob && oob) {
    add_u64_kernel<<<1, 1, 0, st>>>(doob, oob);
    CU(cudaGetLastError());
    p->launches++;
  }
  return 0;
}

// Tile of the FP32/BF16-storage kernels: the user's, or the largest CTA
// whose outer-leg table (n_out x threads x 4 B) fits in 96 KB, at most 128
// points on a hinted grid (16 x 8: on the 64x64-element TFM frame 0.532 ms
// against 0.565 ms for 32 x 8) and 256 consecutive points otherwise.
void fast_tile(const dream_das_plan *p, int n_out, int &tf, int &ts, int &wf) {
  if (p->tile_f > 0) {
    tf = p->tile_f;
    ts = p->tile_s;
    wf = p->n_fast > 0 ? 8 : 32;
    return;
  }
  // frames of fewer points than two waves of 128-point tiles (the CG
  // configuration's 256x256): 8 x 32-point tiles, whose per-tile set-up serves
  // twice the points (0.091 against 0.096 ms for that frame's forward)
  const bool small = p->n_fast > 0 && p->No < (int64_t)p->sm_count * 8 * 128;
  int nthr = (p->n_fast > 0 && !small) ? 128 : 256;
  while (nthr > 32 && (size_t)n_out * nthr * 4 > 96 * 1024) nthr >>= 1;
  if (p->n_fast > 0) {
    wf = 8;
    tf = small ? 8 : (nthr >= 256 ? 32 : (nthr >= 64 ? 16 : 8));
    ts = nthr / tf;
  } else {
    wf = 32;
    tf = nthr;
    ts = 1;
  }
}

// Tiling of the FP32/BF16-storage kernels for plan p: tile shape, warp
// layout, register chunk and grid axes (F.method, Nt, Nr, No must be set).
int tile_params(const dream_das_plan *p, FastParams &F, int jc) {
  const int n_out = (F.method == DREAM_DAS_RCA_ROWTX) ? F.Nr : F.Nt;
  fast_tile(p, n_out, F.tile_f, F.tile_s, F.wf);
  F.jc = jc ? jc : (p->jc ? p->jc : 16);
  if (p->n_fast > 0) {
    F.n_fast = p->n_fast;
    F.n_slow = p->No / p->n_fast;
  } else {
    F.n_fast = p->No;
    F.n_slow = 1;
  }
  if (fast_smem_bytes(F, F.tile_f * F.tile_s) > 220 * 1024)
    return fail(DREAM_ERR_UNSUPPORTED, "too many elements on the outer loop for the FP32/BF16 storage kernels");
  return 0;
}

// The plan's inner-element shard (dream_das_set_inner_shard) applied to F:
// column layout of the shard's A-scans and the inner range; false when the
// range leaves nothing to do.
bool apply_shard(const dream_das_plan *p, FastParams &F) {
  if (p->shard_hi <= 0) return true;
  const int n_out = (F.method == DREAM_DAS_RCA_ROWTX) ? F.Nr : F.Nt;
  const int n_in = (F.method == DREAM_DAS_RCA_ROWTX) ? F.Nt : F.Nr;
  F.ycol_o = p->shard_hi - p->shard_lo;
  F.ycol_i0 = (int)p->shard_lo;
  F.ny = p->K * n_out * F.ycol_o;
  const int lo = std::max<int>(F.in_lo, (int)p->shard_lo);
  const int hi = std::min<int>(F.in_hi > 0 ? F.in_hi : n_in, (int)p->shard_hi);
  F.in_lo = lo;
  F.in_hi = hi;
  return lo < hi;
}

// A-scan columns the plan's Y holds: all of them, or the shard's.
int64_t plan_columns(const dream_das_plan *p) {
  if (p->shard_hi <= 0) return num_columns(p);
  const int64_t n_out = (effective_method(p) == DREAM_DAS_RCA_ROWTX) ? p->Nr : p->Nt;
  return n_out * (p->shard_hi - p->shard_lo);
}

// Slow-axis tiles per launch: about 2^34 terms, so a launch stays well below
// a second.
int64_t slow_tile_chunk(const FastParams &F, int64_t terms_per_pixel) {
  const int64_t per_tile_terms = (int64_t)F.tile_s * F.n_fast * terms_per_pixel;
  const int64_t chunk = std::max<int64_t>(1, (int64_t(1) << 34) / std::max<int64_t>(per_tile_terms, 1));
  return std::min<int64_t>(chunk, 65535);
}

int launch_fast_plan(dream_das_plan *p, const void *dY, const void *dRo, const void *dGt, const void *dGr,
                     double dt, int delay_type, const void *ddelay, double cp, const float *dW, float *dIm,
                     unsigned long long *doob, cudaStream_t st, int in_lo = 0, int in_hi = 0, int accumulate = 0,
                     int jc = 0) {
  if (delay_type != DREAM_DELAY_SINGLE && delay_type != DREAM_DELAY_MULTIPLE)
    return fail(DREAM_ERR_ARGUMENT, "unknown delay type");
  if (ddelay == nullptr) return fail(DREAM_ERR_ARGUMENT, "delay pointer is NULL");
  const int method = effective_method(p);
  if (method >= DREAM_DAS_RCA_COLTX) {
    int r = check_rca_edges(p->Nt, p->Nr);
    if (r) return r;
  }
  if (p->No == 0) return 0;
  if (p->K == 0 || terms_per_pixel(p) == 0) return zero_length_ascans(p, dIm, doob, st);
  if (dY == nullptr || dRo == nullptr || dGt == nullptr || dIm == nullptr ||
      (method != DREAM_DAS_SAFT && dGr == nullptr))
    return fail(DREAM_ERR_ARGUMENT, "NULL device pointer");
  FastParams F;
  memset(&F, 0, sizeof(F));
  F.method = method;
  F.Y = dY;
  F.ny = p->K * num_columns(p);
  F.bad = bad_counter(p);
  F.K = p->K;
  F.Ro = (const double *)dRo;
  F.No = p->No;
  F.Gt = (const double *)dGt;
  F.Nt = (int)p->Nt;
  F.Gr = (const double *)dGr;
  F.Nr = (method == DREAM_DAS_SAFT) ? 0 : (int)p->Nr;
  F.delay = (const double *)ddelay;
  F.delay_multi = delay_type == DREAM_DELAY_MULTIPLE;
  Consts64 c = constants_f64(dt, cp, 0.0);
  F.Fs = c.Fs;
  F.ocp = c.ocp;
  F.w = dW;
  F.Im = dIm;
  F.oob = doob;
  F.in_lo = in_lo;
  F.in_hi = in_hi;
  F.accumulate = accumulate;
  const bool bf16 = p->precision == DREAM_PREC_BF16_STORE;
  const int64_t tpp = std::max<int64_t>(terms_per_pixel(p), 1);
  if (method == DREAM_DAS_SAFT) {
    int64_t chunk = std::max<int64_t>(int64_t(1) << 16, (int64_t(1) << 33) / tpp);
    for (int64_t s0 = 0; s0 < p->No; s0 += chunk) {
      if (p->cancelled.load()) return fail(DREAM_ERR_CANCELLED, "DAS cancelled");
      F.no0 = s0;
      F.no1 = std::min(p->No, s0 + chunk);
      cudaError_t e = launch_fast(F, bf16, st);
      if (e != cudaSuccess) return cuda_fail(e, "DAS kernel launch");
      p->launches++;
    }
    return 0;
  }
  const int n_out = (method == DREAM_DAS_RCA_ROWTX) ? F.Nr : F.Nt;
  int r = tile_params(p, F, jc);
  if (r) return r;
  const int64_t slow_tiles = (F.n_slow + F.tile_s - 1) / F.tile_s;
  const int64_t chunk = slow_tile_chunk(F, tpp);
  // L2 blocking: A-scans larger than the budget are beamformed in passes over
  // ranges of inner elements (multiples of the 16-term register chunk), each
  // pass adding its terms into the image, so the A-scans of one pass stay in
  // L2 while every image point gathers from them.
  const int n_in = (method == DREAM_DAS_RCA_ROWTX) ? F.Nt : F.Nr;
  if (!apply_shard(p, F)) return 0;  // Y holds the columns of inner elements [shard_lo, shard_hi) only
  const int64_t col_bytes = (int64_t)n_out * p->K * (bf16 ? 2 : 4);  // A-scans of one inner element
  const int64_t y_bytes = col_bytes * n_in;
  // automatic: once the A-scans exceed 112 MB (most of the 126 MB L2), even
  // passes of at most 96 MB, widths multiples of the 16-term register chunk
  // (RCA 128x128, K 4096: FP32 268 MB in passes of 48/48/32 columns, 51.6 ->
  // 40.0 ms; BF16 134 MB in two of 64, 36.7 -> 34.5 ms; smaller passes lose
  // more to the per-pass leg set-up than they gain in L2 hits)
  const int64_t budget = p->l2_block > 0 ? p->l2_block : (int64_t(96) << 20);
  const int64_t split_above = p->l2_block > 0 ? budget : (int64_t(112) << 20);
  int pass_w = n_in;
  if (in_hi == 0 && p->l2_block >= 0 && y_bytes > split_above) {
    const int64_t n_pass = (y_bytes + budget - 1) / budget;
    pass_w = (int)std::max<int64_t>(16, ((n_in + n_pass - 1) / n_pass + 15) / 16 * 16);
    pass_w = std::min(pass_w, n_in);
  }
  const int lo0 = F.in_lo, hi0 = F.in_hi > 0 ? F.in_hi : n_in;
  for (int i0 = lo0; i0 < hi0; i0 += pass_w) {
    F.in_lo = i0;
    F.in_hi = std::min(hi0, i0 + pass_w);
    F.accumulate = accumulate || i0 > lo0;
    for (int64_t t0 = 0; t0 < slow_tiles; t0 += chunk) {
      if (p->cancelled.load()) return fail(DREAM_ERR_CANCELLED, "DAS cancelled");
      F.slow_tile0 = t0;
      F.slow_tile1 = std::min(slow_tiles, t0 + chunk);
      cudaError_t e = launch_fast(F, bf16, st);
      if (e != cudaSuccess) return cuda_fail(e, "DAS kernel launch");
      p->launches++;
    }
  }
  return 0;
}

}  // namespace

extern "C" {

const char *dream_das_version(void) { return "dream_b200 das 0.1 (sm_100a)"; }

const char *dream_das_last_error(void) { return g_last_error.c_str(); }

int dream_das_plan_create(dream_das_plan **plan, int das_type, int64_t a_scan_len, int64_t No,
                          int64_t num_t_elements, int64_t num_r_elements, int precision, int device) {
  DREAM_API_TRY
  if (plan == nullptr) return fail(DREAM_ERR_ARGUMENT, "plan pointer is NULL");
  *plan = nullptr;
  int r = check_common(das_type, a_scan_len, No, num_t_elements, num_r_elements, precision);
  if (r) return r;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
  if (device < 0 || device >= ndev) return fail(DREAM_ERR_ARGUMENT, "invalid CUDA device ordinal");
  DeviceGuard g(device);
  if (!g.ok) return fail(DREAM_ERR_CUDA, "cudaSetDevice failed");
  dream_das_plan *p = new dream_das_plan();
  p->das_type = das_type;
  p->K = a_scan_len;
  p->No = No;
  p->Nt = num_t_elements;
  p->Nr = (das_type == DREAM_DAS_SAFT) ? 0 : num_r_elements;
  p->precision = precision;
  p->device = device;
  e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMallocHost((void **)&p->h_oob, sizeof(unsigned long long));
  if (e != cudaSuccess) {
    dream_das_plan_destroy(p);
    return cuda_fail(e, "plan setup");
  }
  r = p->bOob.ensure(sizeof(unsigned long long));
  if (r) {
    dream_das_plan_destroy(p);
    return r;
  }
  cudaDeviceGetAttribute(&p->sm_count, cudaDevAttrMultiProcessorCount, device);
  *plan = p;
  return 0;
  DREAM_API_CATCH
}

int dream_das_setup_has_changed(const dream_das_plan *p, int das_type, int64_t a_scan_len, int64_t No,
                                int64_t num_t_elements, int64_t num_r_elements, int precision, int device) {
  DREAM_API_TRY
  if (p == nullptr) return 1;
  int64_t nr = (das_type == DREAM_DAS_SAFT) ? 0 : num_r_elements;
  return (p->uni || das_type != p->das_type || a_scan_len != p->K || No != p->No || num_t_elements != p->Nt ||
          nr != p->Nr || precision != p->precision || device != p->device)
             ? 1
             : 0;
  DREAM_API_CATCH
}

void dream_das_plan_destroy(dream_das_plan *p) {
  if (p == nullptr) return;
  {
    DeviceGuard g(p->device);
    if (p->stream) cudaStreamSynchronize(p->stream);
    p->bY.release();
    p->bRo.release();
    p->bGt.release();
    p->bGr.release();
    p->bDelay.release();
    p->bIm.release();
    p->bOob.release();
    p->bY16.release();
    p->bScatter.release();
    if (p->h_oob) cudaFreeHost(p->h_oob);
    if (p->h_stage) cudaFreeHost(p->h_stage);
    for (auto &ev : p->chunk_ev)
      if (ev) cudaEventDestroy(ev);
    if (p->copy_stream) cudaStreamDestroy(p->copy_stream);
    if (p->stream) cudaStreamDestroy(p->stream);
  }
  delete p;
}

void dream_das_cancel(dream_das_plan *p) {
  if (p) p->cancelled.store(true);
}

void dream_das_set_running(dream_das_plan *p) {
  if (p) p->cancelled.store(false);
}

int64_t dream_das_plan_num_points(const dream_das_plan *p) { return p ? p->No : -1; }

int64_t dream_das_plan_num_ascans(const dream_das_plan *p) { return p ? num_columns(p) : -1; }

int64_t dream_das_plan_launch_count(const dream_das_plan *p) { return p ? p->launches.load() : -1; }

int dream_das_checked_build(void) {
  DREAM_API_TRY return kChecked ? 1 : 0;
  DREAM_API_CATCH
}

int64_t dream_das_plan_bound_violations(dream_das_plan *p) {
  if (p == nullptr) return fail(DREAM_ERR_ARGUMENT, "plan is NULL");
  if (!kChecked || p->bBad.p == nullptr) return 0;
  std::lock_guard<std::mutex> lk(p->mu);
  DeviceGuard g(p->device);
  unsigned long long v = 0;
  CU(cudaDeviceSynchronize());
  CU(cudaMemcpy(&v, p->bBad.p, sizeof(v), cudaMemcpyDeviceToHost));
  return (int64_t)v;
}

int dream_das_set_grid_hint(dream_das_plan *p, int64_t n_fast) {
  DREAM_API_TRY
  if (p == nullptr) return fail(DREAM_ERR_ARGUMENT, "plan is NULL");
  if (n_fast < 0 || (n_fast > 0 && (p->No % n_fast) != 0))
    return fail(DREAM_ERR_ARGUMENT, "grid hint must divide the number of image points");
  std::lock_guard<std::mutex> lk(p->mu);
  if (n_fast != p->n_fast) p->tile_f = p->tile_s = 0;  // tile shapes depend on the hint
  p->n_fast = n_fast;
  return 0;
  DREAM_API_CATCH
}

int dream_das_set_tile(dream_das_plan *p, int tile_f, int tile_s) {
  DREAM_API_TRY
  if (p == nullptr) return fail(DREAM_ERR_ARGUMENT, "plan is NULL");
  std::lock_guard<std::mutex> lk(p->mu);
  if (tile_f == 0 && tile_s == 0) {
    p->tile_f = p->tile_s = 0;
    return 0;
  }
  const int n = tile_f * tile_s;
  bool ok = tile_f > 0 && tile_s > 0 && n >= 32 && n <= 256 && n % 32 == 0;
  if (p->n_fast > 0) ok = ok && tile_f % 8 == 0 && tile_s % 4 == 0;
  else ok = ok && tile_s == 1;
  if (!ok) return fail(DREAM_ERR_ARGUMENT, "invalid tile shape");
  p->tile_f = tile_f;
  p->tile_s = tile_s;
  return 0;
  DREAM_API_CATCH
}

int dream_das_set_l2_block(dream_das_plan *p, int64_t bytes) {
  DREAM_API_TRY
  if (p == nullptr) return fail(DREAM_ERR_ARGUMENT, "plan is NULL");
  std::lock_guard<std::mutex> lk(p->mu);
  p->l2_block = bytes;
  return 0;
  DREAM_API_CATCH
}

int dream_das_set_inner_shard(dream_das_plan *p, int64_t lo, int64_t hi) {
  DREAM_API_TRY
  if (p == nullptr) return fail(DREAM_ERR_ARGUMENT, "plan is NULL");
  if (!is_fast(p) || p->uni)
    return fail(DREAM_ERR_UNSUPPORTED, "inner-element shards need an F32_STORE or BF16_STORE das plan");
  const int method = effective_method(p);
  if (method == DREAM_DAS_SAFT) return fail(DREAM_ERR_UNSUPPORTED, "SAFT has no inner elements to shard");
  const int64_t n_in = (method == DREAM_DAS_RCA_ROWTX) ? p->Nt : p->Nr;
  if (lo == 0 && hi == 0) {
    p->shard_lo = p->shard_hi = 0;
    return 0;
  }
  if (lo < 0 || hi > n_in || lo >= hi) return fail(DREAM_ERR_ARGUMENT, "inner-element shard out of range");
  p->shard_lo = lo;
  p->shard_hi = hi;
  return 0;
  DREAM_API_CATCH
}

int dream_das_set_chunk(dream_das_plan *p, int jc) {
  DREAM_API_TRY
  if (p == nullptr) return fail(DREAM_ERR_ARGUMENT, "plan is NULL");
  if (jc != 0 && jc != 8 && jc != 16) return fail(DREAM_ERR_ARGUMENT, "chunk must be 0, 8 or 16");
  std::lock_guard<std::mutex> lk(p->mu);
  p->jc = jc;
  return 0;
  DREAM_API_CATCH
}

int dream_das_get_tile(const dream_das_plan *p, int *tile_f, int *tile_s) {
  DREAM_API_TRY
  if (p == nullptr || tile_f == nullptr || tile_s == nullptr) return fail(DREAM_ERR_ARGUMENT, "NULL argument");
  int wf = 0;
  const int n_out = (effective_method(p) == DREAM_DAS_RCA_ROWTX) ? (int)p->Nr : (int)p->Nt;
  fast_tile(p, n_out, *tile_f, *tile_s, wf);
  return 0;
  DREAM_API_CATCH
}

int dream_das_bind_geometry(dream_das_plan *p, const void *dRo, const void *dGt, const void *dGr, double dt,
                            int delay_type, const void *ddelay, double cp, void *stream) {
  DREAM_API_TRY
  if (p == nullptr) return fail(DREAM_ERR_ARGUMENT, "plan is NULL");
  if (p->precision != DREAM_PREC_F32_STORE || p->uni)
    return fail(DREAM_ERR_UNSUPPORTED, "the differentiable operator needs an F32_STORE plan");
  if (delay_type != DREAM_DELAY_SINGLE && delay_type != DREAM_DELAY_MULTIPLE)
    return fail(DREAM_ERR_ARGUMENT, "unknown delay type");
  const int method = effective_method(p);
  if (method == DREAM_DAS_SAFT) return fail(DREAM_ERR_UNSUPPORTED, "the operator supports TFM and RCA");
  if (method >= DREAM_DAS_RCA_COLTX) {
    int r = check_rca_edges(p->Nt, p->Nr);
    if (r) return r;
  }
  if ((p->No > 0 && dRo == nullptr) || dGt == nullptr || dGr == nullptr || ddelay == nullptr)
    return fail(DREAM_ERR_ARGUMENT, "NULL device pointer");
  std::lock_guard<std::mutex> lk(p->mu);
  (void)stream;  // nothing is precomputed: the operator's kernels form their legs per tile
  FastParams F;
  memset(&F, 0, sizeof(F));
  F.method = method;
  F.K = p->K;
  F.Ro = (const double *)dRo;
  F.No = p->No;
  F.Gt = (const double *)dGt;
  F.Nt = (int)p->Nt;
  F.Gr = (const double *)dGr;
  F.Nr = (int)p->Nr;
  F.delay = (const double *)ddelay;
  F.delay_multi = delay_type == DREAM_DELAY_MULTIPLE;
  Consts64 c = constants_f64(dt, cp, 0.0);
  F.Fs = c.Fs;
  F.ocp = c.ocp;
  p->geo = F;
  p->bound = true;
  return 0;
  DREAM_API_CATCH
}

// Forward (weighted gather) of the bound operator on pixel tiles.
static int op_gather(dream_das_plan *p, const float *dY, const float *dW, float *dIm, unsigned long long *d_oob,
                     cudaStream_t st) {
  FastParams F = p->geo;
  F.Y = dY;
  F.w = dW;
  F.Im = dIm;
  F.oob = d_oob;
  F.ny = p->K * num_columns(p);
  F.bad = bad_counter(p);
  int r = tile_params(p, F, 0);
  if (r) return r;
  if (!apply_shard(p, F)) return 0;
  const int64_t slow_tiles = (F.n_slow + F.tile_s - 1) / F.tile_s;
  const int64_t chunk = slow_tile_chunk(F, terms_per_pixel(p));
  for (int64_t t0 = 0; t0 < slow_tiles; t0 += chunk) {
    F.slow_tile0 = t0;
    F.slow_tile1 = std::min(slow_tiles, t0 + chunk);
    CU(launch_fast(F, false, st));
    p->launches++;
  }
  return 0;
}

// Adjoint (scatter) of the bound operator on pixel tiles: Ya zeroed, then
// every term added at the forward's index.
static int op_scatter(dream_das_plan *p, const float *X, const float *dW, float *Ya, cudaStream_t st) {
  const size_t ycount = (size_t)p->K * plan_columns(p);
  if (ycount) CU(cudaMemsetAsync(Ya, 0, ycount * 4, st));
  if (p->No == 0 || p->K == 0) return 0;
  FastParams F = p->geo;
  F.w = dW;
  int r = tile_params(p, F, 0);
  if (r) return r;
  // The scatter's own automatic tile on a hinted TFM grid: 8 x 32 points,
  // long along the slow axis, where a column's sample window grows slowest
  // relative to the tile's terms (64x64-element TFM frame 1.25 -> 1.20 ms,
  // 32x32-element CG configuration 0.130 -> 0.120 ms, against 16 x 8). RCA
  // volumes keep the forward's tile: 32 points along their slow axis spread a
  // stripe's leg beyond the window (128x128 frame: 108.7 against 81.7 ms).
  const int n_out = (F.method == DREAM_DAS_RCA_ROWTX) ? F.Nr : F.Nt;
  if (p->tile_f == 0 && p->n_fast > 0 && F.method == DREAM_DAS_TFM && (size_t)n_out * 256 * 4 <= 96 * 1024) {
    F.tile_f = 8;
    F.tile_s = 32;
    F.wf = 8;
  }
  if (!apply_shard(p, F)) return 0;
  const int64_t slow_tiles = (F.n_slow + F.tile_s - 1) / F.tile_s;
  const int64_t chunk = slow_tile_chunk(F, terms_per_pixel(p));
  for (int64_t t0 = 0; t0 < slow_tiles; t0 += chunk) {
    F.slow_tile0 = t0;
    F.slow_tile1 = std::min(slow_tiles, t0 + chunk);
    CU(launch_scatter(F, X, Ya, st));
    p->launches++;
  }
  return 0;
}

static int op_check(dream_das_plan *p) {
  if (p == nullptr) return fail(DREAM_ERR_ARGUMENT, "plan is NULL");
  if (!p->bound) return fail(DREAM_ERR_ARGUMENT, "no geometry bound (dream_das_bind_geometry)");
  if (p->cancelled.load()) return fail(DREAM_ERR_CANCELLED, "DAS cancelled");
  return 0;
}

int dream_das_op_forward(dream_das_plan *p, const float *dY, const float *dW, float *dIm, unsigned long long *d_oob,
                         void *stream) {
  DREAM_API_TRY
  int r = op_check(p);
  if (r) return r;
  std::lock_guard<std::mutex> lk(p->mu);
  DeviceGuard g(p->device);
  if (p->No == 0) return 0;
  if (p->K == 0) return zero_length_ascans(p, dIm, d_oob, (cudaStream_t)stream);
  return op_gather(p, dY, dW, dIm, d_oob, (cudaStream_t)stream);
  DREAM_API_CATCH
}

int dream_das_op_adjoint(dream_das_plan *p, const float *dX, const float *dW, float *dYa, void *stream) {
  DREAM_API_TRY
  int r = op_check(p);
  if (r) return r;
  if (dX == nullptr || dYa == nullptr) return fail(DREAM_ERR_ARGUMENT, "NULL device pointer");
  std::lock_guard<std::mutex> lk(p->mu);
  DeviceGuard g(p->device);
  return op_scatter(p, dX, dW, dYa, (cudaStream_t)stream);
  DREAM_API_CATCH
}

int dream_das_op_wgrad(dream_das_plan *p, const float *dG, const float *dY, float *dWgrad, void *stream) {
  DREAM_API_TRY
  int r = op_check(p);
  if (r) return r;
  if (dG == nullptr || dY == nullptr || dWgrad == nullptr) return fail(DREAM_ERR_ARGUMENT, "NULL device pointer");
  std::lock_guard<std::mutex> lk(p->mu);
  DeviceGuard g(p->device);
  // dW[c] = sum_n g[n] Y[k(n,c), c] = sum_k Y[k,c] (DAS^T g)[k,c]: the
  // unweighted scatter of g into the plan's scratch, then one column pass
  const size_t ycount = (size_t)p->K * plan_columns(p);
  if ((r = p->bScatter.ensure(std::max<size_t>(ycount, 1) * 4))) return r;
  cudaStream_t st = (cudaStream_t)stream;
  if ((r = op_scatter(p, dG, nullptr, (float *)p->bScatter.p, st))) return r;
  CU(launch_column_dot_scale(dY, (float *)p->bScatter.p, nullptr, dWgrad, p->K, plan_columns(p), st));
  p->launches++;
  return 0;
  DREAM_API_CATCH
}

int dream_das_op_backward(dream_das_plan *p, const float *dG, const float *dY, const float *dW, float *dYgrad,
                          float *dWgrad, void *stream) {
  DREAM_API_TRY
  int r = op_check(p);
  if (r) return r;
  if (dG == nullptr || dYgrad == nullptr || dWgrad == nullptr || dY == nullptr)
    return fail(DREAM_ERR_ARGUMENT, "NULL device pointer");
  std::lock_guard<std::mutex> lk(p->mu);
  DeviceGuard g(p->device);
  // one unweighted scatter S = DAS^T g into dYgrad, then per column
  // dW[c] = <Y[:,c], S[:,c]> and dYgrad[:,c] = w[c] S[:,c]
  cudaStream_t st = (cudaStream_t)stream;
  if ((r = op_scatter(p, dG, nullptr, dYgrad, st))) return r;
  CU(launch_column_dot_scale(dY, dYgrad, dW, dWgrad, p->K, plan_columns(p), st));
  p->launches++;
  return 0;
  DREAM_API_CATCH
}

}  // extern "C"

namespace dream {
// One batch frame: validated and turned into its launch descriptor (oob
// pointer left NULL). Shared by dream_das_batch_create and the allocation-free
// batch entry so that both accept exactly the same frames.
int batch_frame_params(const dream_das_frame &d, FastParams &F) {
  int r = check_common(d.das_type, d.a_scan_len, d.No, d.num_t_elements, d.num_r_elements, DREAM_PREC_F32_STORE);
  if (!r && (d.das_type == DREAM_DAS_SAFT || d.num_r_elements == 0))
    r = fail(DREAM_ERR_UNSUPPORTED, "batch frames must be TFM or RCA");
  if (!r && d.das_type >= DREAM_DAS_RCA_COLTX) r = check_rca_edges(d.num_t_elements, d.num_r_elements);
  if (!r && (d.n_fast < 0 || (d.n_fast > 0 && d.No % d.n_fast)))
    r = fail(DREAM_ERR_ARGUMENT, "grid hint must divide the number of image points");
  if (!r && (d.tile_f || d.tile_s) &&
      (d.tile_f * d.tile_s != 128 || (d.n_fast > 0 ? (d.tile_f % 8 || d.tile_s % 4) : d.tile_s != 1)))
    r = fail(DREAM_ERR_ARGUMENT, "invalid frame tile (tile_f * tile_s must be 128)");
  if (!r && d.jc != 0 && d.jc != 8 && d.jc != 16) r = fail(DREAM_ERR_ARGUMENT, "chunk must be 0, 8 or 16");
  if (!r && d.No > 0 && d.a_scan_len > 0 &&
      (d.Y == nullptr || d.Ro == nullptr || d.Gt == nullptr || d.Gr == nullptr || d.delay == nullptr || d.Im == nullptr))
    r = fail(DREAM_ERR_ARGUMENT, "NULL frame pointer");
  if (r) return r;
  memset(&F, 0, sizeof(F));
  F.method = d.das_type;
  F.Y = d.Y;
  F.K = d.a_scan_len;
  F.Ro = d.Ro;
  F.No = d.No;
  F.Gt = d.Gt;
  F.Nt = (int)d.num_t_elements;
  F.Gr = d.Gr;
  F.Nr = (int)d.num_r_elements;
  F.delay = d.delay;
  F.delay_multi = d.delay_type == DREAM_DELAY_MULTIPLE;
  Consts64 c = constants_f64(d.dt, d.cp, 0.0);
  F.Fs = c.Fs;
  F.ocp = c.ocp;
  F.Im = d.Im;
  if (d.n_fast > 0) {
    F.n_fast = d.n_fast;
    F.n_slow = d.No / d.n_fast;
    F.wf = 8;
    F.tile_f = d.tile_f ? d.tile_f : 16;
    F.tile_s = d.tile_s ? d.tile_s : 8;
  } else {
    F.n_fast = d.No;
    F.n_slow = 1;
    F.wf = 32;
    F.tile_f = 128;
    F.tile_s = 1;
  }
  F.jc = d.jc ? d.jc : 16;
  return 0;
}
}  // namespace dream

struct dream_das_batch {
  int device = 0;
  bool bf16 = false;
  int n_frames = 0;
  int64_t n_items = 0;
  size_t smem = 0;
  int grid = 0;
  DevBuf bFrames, bItems, bCtr;
  std::vector<FastParams> frames;  // host copy (oob pointer patched per run)
  unsigned long long *last_oob = nullptr;
  std::mutex mu;
};

extern "C" {

int dream_das_batch_create(dream_das_batch **out, const dream_das_frame *fr, int n_frames, int precision, int device) {
  DREAM_API_TRY
  if (out == nullptr || (fr == nullptr && n_frames > 0) || n_frames < 0) return fail(DREAM_ERR_ARGUMENT, "NULL argument");
  *out = nullptr;
  if (precision != DREAM_PREC_F32_STORE && precision != DREAM_PREC_BF16_STORE)
    return fail(DREAM_ERR_UNSUPPORTED, "batches use F32_STORE or BF16_STORE");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
  if (device < 0 || device >= ndev) return fail(DREAM_ERR_ARGUMENT, "invalid CUDA device ordinal");
  DeviceGuard g(device);
  auto *b = new dream_das_batch();
  b->device = device;
  b->bf16 = precision == DREAM_PREC_BF16_STORE;
  b->n_frames = n_frames;
  struct Group {
    double cost;
    int f;
    int64_t tf, ts;
  };
  std::vector<Group> groups;
  for (int f = 0; f < n_frames; f++) {
    const dream_das_frame &d = fr[f];
    FastParams F;
    int r = batch_frame_params(d, F);
    if (r) {
      dream_das_batch_destroy(b);
      return r;
    }
    b->smem = std::max(b->smem, fast_smem_bytes(F, 128));
    b->frames.push_back(F);
    if (d.No > 0 && d.a_scan_len > 0) {
      const int64_t tf = (F.n_fast + F.tile_f - 1) / F.tile_f, ts = (F.n_slow + F.tile_s - 1) / F.tile_s;
      groups.push_back({(double)d.num_t_elements * d.num_r_elements, f, tf, ts});
    }
  }
  if (b->smem > 220 * 1024) {
    dream_das_batch_destroy(b);
    return fail(DREAM_ERR_UNSUPPORTED, "a frame has too many outer elements for the batch kernel");
  }
  // largest per-tile cost first: the queue drains big tiles before small ones
  std::stable_sort(groups.begin(), groups.end(), [](const Group &a, const Group &c) { return a.cost > c.cost; });
  std::vector<int4> items;
  for (const Group &gr : groups)
    for (int64_t ts = 0; ts < gr.ts; ts++)
      for (int64_t tf = 0; tf < gr.tf; tf++) items.push_back(make_int4(gr.f, (int)tf, (int)ts, 0));
  b->n_items = (int64_t)items.size();
  if (b->n_items > INT32_MAX) {
    dream_das_batch_destroy(b);
    return fail(DREAM_ERR_ARGUMENT, "too many tiles in one batch");
  }
  int r;
  if ((r = b->bFrames.ensure(std::max<size_t>(1, b->frames.size()) * sizeof(FastParams))) ||
      (r = b->bItems.ensure(std::max<size_t>(1, items.size()) * sizeof(int4))) || (r = b->bCtr.ensure(sizeof(int)))) {
    dream_das_batch_destroy(b);
    return r;
  }
  if (!items.empty()) {
    e = cudaMemcpy(b->bItems.p, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      dream_das_batch_destroy(b);
      return cuda_fail(e, "copying the work list");
    }
  }
  int per_sm = batch_prepare(std::max<size_t>(b->smem, 1024), b->bf16);
  if (per_sm <= 0) {
    dream_das_batch_destroy(b);
    return fail(DREAM_ERR_CUDA, "batch kernel does not fit on an SM");
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  b->grid = (int)std::min<int64_t>((int64_t)sms * per_sm, std::max<int64_t>(1, b->n_items));
  b->last_oob = (unsigned long long *)1;  // force the first upload
  *out = b;
  return 0;
  DREAM_API_CATCH
}

int dream_das_batch_run(dream_das_batch *b, unsigned long long *d_oob, void *stream) {
  DREAM_API_TRY
  if (b == nullptr) return fail(DREAM_ERR_ARGUMENT, "batch is NULL");
  std::lock_guard<std::mutex> lk(b->mu);
  DeviceGuard g(b->device);
  cudaStream_t st = (cudaStream_t)stream;
  if (d_oob != b->last_oob) {
    // the frame table holds the counter pointer: upload it when it changes
    for (auto &F : b->frames) F.oob = d_oob;
    CU(cudaMemcpyAsync(b->bFrames.p, b->frames.data(), b->frames.size() * sizeof(FastParams),
                       cudaMemcpyHostToDevice, st));
    CU(cudaStreamSynchronize(st));
    b->last_oob = d_oob;
  }
  CU(launch_batch((const FastParams *)b->bFrames.p, (const int4 *)b->bItems.p, (int)b->n_items, (int *)b->bCtr.p,
                  std::max<size_t>(b->smem, 1024), b->bf16, b->grid, st));
  return 0;
  DREAM_API_CATCH
}

int64_t dream_das_batch_items(const dream_das_batch *b) { return b ? b->n_items : -1; }

int dream_das_batch_grid(const dream_das_batch *b) {
  DREAM_API_TRY return b ? b->grid : -1;
  DREAM_API_CATCH
}

void dream_das_batch_destroy(dream_das_batch *b) {
  if (b == nullptr) return;
  {
    DeviceGuard g(b->device);
    b->bFrames.release();
    b->bItems.release();
    b->bCtr.release();
  }
  delete b;
}

int dream_das_weighted_run_device(dream_das_plan *p, const void *dY, const void *dRo, const void *dGt,
                                  const void *dGr, double dt, int delay_type, const void *ddelay, double cp,
                                  const float *dW, float *dIm, unsigned long long *d_oob, void *stream) {
  DREAM_API_TRY
  if (p == nullptr) return fail(DREAM_ERR_ARGUMENT, "plan is NULL");
  if (!is_fast(p) || p->uni)
    return fail(DREAM_ERR_UNSUPPORTED, "weighted DAS needs an F32_STORE or BF16_STORE plan");
  if (dW == nullptr) return fail(DREAM_ERR_ARGUMENT, "weights pointer is NULL");
  if (p->cancelled.load()) return fail(DREAM_ERR_CANCELLED, "DAS cancelled");
  std::lock_guard<std::mutex> lk(p->mu);
  DeviceGuard g(p->device);
  return launch_fast_plan(p, dY, dRo, dGt, dGr, dt, delay_type, ddelay, cp, dW, dIm, d_oob, (cudaStream_t)stream);
  DREAM_API_CATCH
}

static int run_device_impl(dream_das_plan *p, const void *dY, const void *dRo, const void *dGt, const void *dGr,
                           double dt, int delay_type, const void *ddelay, double cp, void *dIm,
                           unsigned long long *doob, cudaStream_t st) {
  if (is_fast(p))
    return launch_fast_plan(p, dY, dRo, dGt, dGr, dt, delay_type, ddelay, cp, nullptr, (float *)dIm, doob, st);
  PlainLaunch L;
  int r = prepare_das(p, L, dY, dRo, dGt, dGr, dt, delay_type, ddelay, cp, dIm, doob);
  if (r) return r;
  if (p->No == 0) return 0;
  if (p->K == 0 || terms_per_pixel(p) == 0) return zero_length_ascans(p, dIm, doob, st);
  return launch_plain(p, L, st);
}

int dream_das_indices_device(dream_das_plan *p, const void *dRo, const void *dGt, const void *dGr, double dt,
                             int delay_type, const void *ddelay, double cp, int64_t *d_idx, int64_t *oob_count,
                             void *stream) {
  DREAM_API_TRY
  if (p == nullptr) return fail(DREAM_ERR_ARGUMENT, "plan is NULL");
  if (p->uni) return fail(DREAM_ERR_ARGUMENT, "uniform-grid plan passed to dream_das_indices_device");
  if (p->cancelled.load()) return fail(DREAM_ERR_CANCELLED, "DAS cancelled");
  if (delay_type != DREAM_DELAY_SINGLE && delay_type != DREAM_DELAY_MULTIPLE)
    return fail(DREAM_ERR_ARGUMENT, "unknown delay type");
  if (ddelay == nullptr) return fail(DREAM_ERR_ARGUMENT, "delay pointer is NULL");
  std::lock_guard<std::mutex> lk(p->mu);
  DeviceGuard g(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  // F32 plans: das_f's FP32 indices; every other precision: das's FP64 ones
  // (the indices the FP32/BF16-storage kernels select as well)
  const bool f32 = p->precision == DREAM_PREC_F32;
  PlainLaunch L;
  memset(&L, 0, sizeof(L));
  L.method = effective_method(p);
  L.K = p->K;
  L.Ro = dRo;
  L.No = p->No;
  L.Gt = dGt;
  L.Nt = p->Nt;
  L.Gr = dGr;
  L.Nr = (L.method == DREAM_DAS_SAFT) ? 0 : p->Nr;
  L.delay_vec = ddelay;
  L.delay_multi = delay_type == DREAM_DELAY_MULTIPLE;
  if (f32) L.c32 = constants_das_f32((float)dt, (float)cp, 0.0f);
  else L.c64 = constants_f64(dt, cp, 0.0);
  if (L.method >= DREAM_DAS_RCA_COLTX) {
    int r = check_rca_edges(p->Nt, p->Nr);
    if (r) return r;
  }
  const int64_t terms = terms_per_pixel(p);
  if (p->No == 0 || terms == 0) {
    if (oob_count) *oob_count = 0;
    return 0;
  }
  if (dRo == nullptr || dGt == nullptr || d_idx == nullptr || (L.Nr > 0 && dGr == nullptr))
    return fail(DREAM_ERR_ARGUMENT, "NULL device pointer");
  unsigned long long *doob = (unsigned long long *)p->bOob.p;
  CU(cudaMemsetAsync(doob, 0, sizeof(unsigned long long), st));
  if (p->K == 0) {  // every term out of bounds
    CU(cudaMemsetAsync(d_idx, 0xff, (size_t)p->No * terms * sizeof(int64_t), st));
    if (oob_count) *oob_count = p->No * terms;
    return 0;
  }
  L.idx = d_idx;
  L.oob = doob;
  const int64_t chunk = std::max<int64_t>(int64_t(1) << 16, ((int64_t(1) << 33) / terms + 255) / 256 * 256);
  for (int64_t s0 = 0; s0 < p->No; s0 += chunk) {
    if (p->cancelled.load()) return fail(DREAM_ERR_CANCELLED, "DAS cancelled");
    L.no0 = s0;
    L.no1 = std::min(p->No, s0 + chunk);
    cudaError_t e = f32 ? launch_plain_f32(L, st) : launch_plain_f64(L, st);
    if (e != cudaSuccess) return cuda_fail(e, "DAS index kernel launch");
    p->launches++;
  }
  if (oob_count) {
    unsigned long long h = 0;
    CU(cudaMemcpyAsync(&h, doob, sizeof(h), cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    *oob_count = (int64_t)h;
  }
  return 0;
  DREAM_API_CATCH
}

int dream_das_run_device(dream_das_plan *p, const void *dY, const void *dRo, const void *dGt, const void *dGr,
                         double dt, int delay_type, const void *ddelay, double cp, void *dIm, int err_level,
                         int64_t *oob_count, void *stream) {
  DREAM_API_TRY
  if (p == nullptr) return fail(DREAM_ERR_ARGUMENT, "plan is NULL");
  if (p->uni) return fail(DREAM_ERR_ARGUMENT, "uniform-grid plan passed to dream_das_run_device");
  if (p->cancelled.load()) return fail(DREAM_ERR_CANCELLED, "DAS cancelled");
  std::lock_guard<std::mutex> lk(p->mu);
  DeviceGuard g(p->device);
  cudaStream_t st = (cudaStream_t)stream;  // NULL: the default stream
  unsigned long long *doob = (unsigned long long *)p->bOob.p;
  CU(cudaMemsetAsync(doob, 0, sizeof(unsigned long long), st));
  int r = run_device_impl(p, dY, dRo, dGt, dGr, dt, delay_type, ddelay, cp, dIm, doob, st);
  if (r) return r;
  CU(cudaMemcpyAsync(p->h_oob, doob, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  uint64_t oob = *p->h_oob;
  if (oob_count) *oob_count = (int64_t)oob;
  return status_from_oob(oob, err_level);
  DREAM_API_CATCH
}

int dream_das_run_device_async(dream_das_plan *p, const void *dY, const void *dRo, const void *dGt,
                               const void *dGr, double dt, int delay_type, const void *ddelay, double cp,
                               void *dIm, unsigned long long *d_oob, void *stream) {
  DREAM_API_TRY
  if (p == nullptr) return fail(DREAM_ERR_ARGUMENT, "plan is NULL");
  if (p->uni) return fail(DREAM_ERR_ARGUMENT, "uniform-grid plan passed to dream_das_run_device_async");
  if (p->cancelled.load()) return fail(DREAM_ERR_CANCELLED, "DAS cancelled");
  std::lock_guard<std::mutex> lk(p->mu);
  DeviceGuard g(p->device);
  cudaStream_t st = (cudaStream_t)stream;  // NULL: the default stream
  return run_device_impl(p, dY, dRo, dGt, dGr, dt, delay_type, ddelay, cp, dIm, d_oob, st);
  DREAM_API_CATCH
}

// Image read-back to host memory Im: straight into Im when it is pinned,
// else into the plan's pinned staging buffer, which finish_read_back copies
// into Im once the stream has synchronised. (A copy to pageable memory is
// staged by the driver at a fraction of the link rate: 0.10 ms for the 1 MB
// image of a 512x512 frame, against 0.02 ms from pinned memory.)
static int start_read_back(dream_das_plan *p, void *Im, const void *dIm, size_t bytes, cudaStream_t st, void *&staged) {
  staged = nullptr;
  if (bytes == 0) return 0;
  cudaPointerAttributes attr{};
  const bool pinned = cudaPointerGetAttributes(&attr, Im) == cudaSuccess && attr.type == cudaMemoryTypeHost;
  cudaGetLastError();  // an unregistered pointer may leave an error on older runtimes
  if (!pinned) {
    if (p->h_stage_bytes < bytes) {
      if (p->h_stage) CU(cudaFreeHost(p->h_stage));
      p->h_stage = nullptr;
      p->h_stage_bytes = 0;
      CU(cudaMallocHost(&p->h_stage, bytes));
      p->h_stage_bytes = bytes;
    }
    staged = p->h_stage;
  }
  CU(cudaMemcpyAsync(staged ? staged : Im, dIm, bytes, cudaMemcpyDeviceToHost, st));
  return 0;
}

static void finish_read_back(void *Im, const void *staged, size_t bytes) {
  if (staged) memcpy(Im, staged, bytes);
}

// Inner-element boundaries of the pipelined upload: UPLOAD_CHUNKS ranges on
// multiples of 8 (at most 15). Every chunk's kernel recomputes the image
// points' outer legs, so more, shorter chunks cost more than they save at the
// ends of the pipeline: on the 64x64-element TFM frame from pinned memory,
// 4 chunks of 16 take 1.50 ms, 8 of 8 take 1.94 ms and 8/16/16/16/8 1.55 ms.
static std::vector<int> upload_chunks(int n_in) {
  constexpr int UPLOAD_CHUNKS = 4;
  const int n = std::max(1, std::min({UPLOAD_CHUNKS, 15, (n_in + 7) / 8}));
  std::vector<int> cuts{0};
  for (int c = 1; c < n; c++) {
    const int b = std::min(n_in, (c * n_in / n + 7) / 8 * 8);
    if (b > cuts.back()) cuts.push_back(b);
  }
  if (n_in > cuts.back()) cuts.push_back(n_in);
  return cuts;
}

int dream_das_run(dream_das_plan *p, const void *Y, const void *Ro, const void *Gt, const void *Gr, double dt,
                  int delay_type, const void *delay, double cp, void *Im, int err_level, int64_t *oob_count) {
  DREAM_API_TRY
  if (p == nullptr) return fail(DREAM_ERR_ARGUMENT, "plan is NULL");
  if (p->uni) return fail(DREAM_ERR_ARGUMENT, "uniform-grid plan passed to dream_das_run");
  if (p->shard_hi > 0)
    return fail(DREAM_ERR_UNSUPPORTED, "inner-element shards run through the device entry points");
  if (p->cancelled.load()) return fail(DREAM_ERR_CANCELLED, "DAS cancelled");
  if (delay == nullptr) return fail(DREAM_ERR_ARGUMENT, "delay pointer is NULL");
  std::lock_guard<std::mutex> lk(p->mu);
  DeviceGuard g(p->device);
  cudaStream_t st = p->stream;
  const size_t ys = is_fast(p) ? 4 : prec_size(p->precision);  // host Y element
  const size_t gs = geo_size(p), is = im_size(p);
  const int method = effective_method(p);
  const int64_t ncol = num_columns(p);
  const int64_t nr = (method == DREAM_DAS_SAFT) ? 0 : p->Nr;
  const bool multi = delay_type == DREAM_DELAY_MULTIPLE && p->No != 1;
  const int64_t ny = p->K * ncol;
  int r;
  if ((r = p->bY.ensure((size_t)ny * ys))) return r;
  if ((r = p->bRo.ensure((size_t)p->No * 3 * gs))) return r;
  if ((r = p->bGt.ensure((size_t)p->Nt * 3 * gs))) return r;
  if ((r = p->bGr.ensure((size_t)nr * 3 * gs))) return r;
  if ((r = p->bDelay.ensure((size_t)(multi ? p->No : 1) * gs))) return r;
  if ((r = p->bIm.ensure((size_t)p->No * is))) return r;
  // FP32/BF16-storage TFM and RCA: the A-scans are uploaded in chunks of
  // inner elements on a copy stream while the kernel beamforms the chunks
  // already resident, adding each chunk's terms into the image.
  const bool pipelined = is_fast(p) && method != DREAM_DAS_SAFT && p->No > 0 && p->K > 0 &&
                         (size_t)ny * 4 >= (size_t(8) << 20);
  if (ny > 0 && !pipelined) CU(cudaMemcpyAsync(p->bY.p, Y, (size_t)ny * ys, cudaMemcpyHostToDevice, st));
  if (p->No > 0) CU(cudaMemcpyAsync(p->bRo.p, Ro, (size_t)p->No * 3 * gs, cudaMemcpyHostToDevice, st));
  if (p->Nt > 0) CU(cudaMemcpyAsync(p->bGt.p, Gt, (size_t)p->Nt * 3 * gs, cudaMemcpyHostToDevice, st));
  if (nr > 0) CU(cudaMemcpyAsync(p->bGr.p, Gr, (size_t)nr * 3 * gs, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(p->bDelay.p, delay, (size_t)(multi ? p->No : 1) * gs, cudaMemcpyHostToDevice, st));
  if (pipelined) {
    const int n_out = (method == DREAM_DAS_RCA_ROWTX) ? (int)p->Nr : (int)p->Nt;
    const int n_in = (method == DREAM_DAS_RCA_ROWTX) ? (int)p->Nt : (int)p->Nr;
    const bool bf16 = p->precision == DREAM_PREC_BF16_STORE;
    if (bf16 && (r = p->bY16.ensure((size_t)ny * 2))) return r;
    if (p->copy_stream == nullptr) CU(cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking));
    for (auto &ev : p->chunk_ev)
      if (ev == nullptr) CU(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    int check = 0;
    if (method >= DREAM_DAS_RCA_COLTX && (check = check_rca_edges(p->Nt, p->Nr))) return check;
    const std::vector<int> cuts = upload_chunks(n_in);
    unsigned long long *doob = (unsigned long long *)p->bOob.p;
    CU(cudaMemsetAsync(doob, 0, sizeof(unsigned long long), st));
    // the copy stream must not overwrite A-scans a previous call still reads
    CU(cudaEventRecord(p->chunk_ev[15], st));
    CU(cudaStreamWaitEvent(p->copy_stream, p->chunk_ev[15], 0));
    const size_t pitch = (size_t)n_in * p->K * 4;
    for (size_t c = 0; c + 1 < cuts.size(); c++) {
      const int lo = cuts[c], hi = cuts[c + 1];
      const size_t off = (size_t)lo * p->K * 4, width = (size_t)(hi - lo) * p->K * 4;
      CU(cudaMemcpy2DAsync((char *)p->bY.p + off, pitch, (const char *)Y + off, pitch, width, (size_t)n_out,
                           cudaMemcpyHostToDevice, p->copy_stream));
      if (bf16) {
        CU(convert_f32_to_bf16_2d((const float *)p->bY.p + (size_t)lo * p->K, (uint16_t *)p->bY16.p + (size_t)lo * p->K,
                                  n_out, (int64_t)(hi - lo) * p->K, (int64_t)n_in * p->K, p->copy_stream));
        p->launches++;
      }
      CU(cudaEventRecord(p->chunk_ev[c], p->copy_stream));
      CU(cudaStreamWaitEvent(st, p->chunk_ev[c], 0));
      // a register chunk that divides the range keeps every chunk full
      const int jc = ((hi - lo) % 16 == 0) ? 16 : (((hi - lo) % 8 == 0) ? 8 : 0);
      r = launch_fast_plan(p, bf16 ? p->bY16.p : p->bY.p, p->bRo.p, p->bGt.p, p->bGr.p, dt, delay_type, p->bDelay.p,
                           cp, nullptr, (float *)p->bIm.p, doob, st, lo, hi, c > 0 ? 1 : 0, jc);
      if (r) return r;
    }
    void *staged = nullptr;
    if ((r = start_read_back(p, Im, p->bIm.p, (size_t)p->No * is, st, staged))) return r;
    CU(cudaMemcpyAsync(p->h_oob, doob, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    finish_read_back(Im, staged, (size_t)p->No * is);
    uint64_t oob = *p->h_oob;
    if (oob_count) *oob_count = (int64_t)oob;
    return status_from_oob(oob, err_level);
  }
  const void *dYrun = p->bY.p;
  if (p->precision == DREAM_PREC_BF16_STORE && ny > 0) {
    if ((r = p->bY16.ensure((size_t)ny * 2))) return r;
    CU(convert_f32_to_bf16((const float *)p->bY.p, p->bY16.p, ny, st));
    p->launches++;
    dYrun = p->bY16.p;
  }
  unsigned long long *doob = (unsigned long long *)p->bOob.p;
  CU(cudaMemsetAsync(doob, 0, sizeof(unsigned long long), st));
  r = run_device_impl(p, dYrun, p->bRo.p, p->bGt.p, p->bGr.p, dt, delay_type, p->bDelay.p, cp, p->bIm.p,
                      doob, st);
  if (r) return r;
  void *staged = nullptr;
  if ((r = start_read_back(p, Im, p->bIm.p, (size_t)p->No * is, st, staged))) return r;
  CU(cudaMemcpyAsync(p->h_oob, doob, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  finish_read_back(Im, staged, (size_t)p->No * is);
  uint64_t oob = *p->h_oob;
  if (oob_count) *oob_count = (int64_t)oob;
  return status_from_oob(oob, err_level);
  DREAM_API_CATCH
}

// ---------------------------------------------------------------------------
// das_uni
// ---------------------------------------------------------------------------

int dream_das_uni_plan_create(dream_das_plan **plan, int das_type, int64_t a_scan_len, const double *tri,
                              int precision, int device) {
  DREAM_API_TRY
  if (plan == nullptr || tri == nullptr) return fail(DREAM_ERR_ARGUMENT, "NULL argument");
  *plan = nullptr;
  if (precision != DREAM_PREC_F64 && precision != DREAM_PREC_F32)
    return fail(DREAM_ERR_UNSUPPORTED, "das_uni supports F64 and F32");
  const bool f32 = precision == DREAM_PREC_F32;
  int64_t Nt = uni_count(tri[0], tri[1], tri[2], f32);
  int64_t Nr = (das_type == DREAM_DAS_SAFT) ? 0 : uni_count(tri[3], tri[4], tri[5], f32);
  int64_t Nx = uni_count(tri[6], tri[7], tri[8], f32);
  int64_t Ny = uni_count(tri[9], tri[10], tri[11], f32);
  int64_t Nz = uni_count(tri[12], tri[13], tri[14], f32);
  if (Nt < 0 || Nr < 0 || Nx < 0 || Ny < 0 || Nz < 0)
    return fail(DREAM_ERR_ARGUMENT, "invalid (min, pitch, max) triplet");
  if (Nx * Ny * Nz > ((int64_t)1 << 40)) return fail(DREAM_ERR_ARGUMENT, "too many image points");
  if (das_type != DREAM_DAS_SAFT && Nr == 0) return fail(DREAM_ERR_ARGUMENT, "empty receive triplet");
  int r = dream_das_plan_create(plan, das_type, a_scan_len, Nx * Ny * Nz, Nt, Nr, precision, device);
  if (r) return r;
  dream_das_plan *p = *plan;
  p->uni = true;
  for (int i = 0; i < 15; i++) p->tri[i] = tri[i];
  p->Nx = Nx;
  p->Ny = Ny;
  p->Nz = Nz;
  return 0;
  DREAM_API_CATCH
}

static int uni_launch(dream_das_plan *p, const void *dY, const double *tri, double dt, double delay, double cp,
                      void *dIm, unsigned long long *doob, cudaStream_t st) {
  for (int i = 0; i < 15; i++) {
    if (p->das_type == DREAM_DAS_SAFT && i >= 3 && i < 6) continue;
    if (tri[i] != p->tri[i] && !(tri[i] != tri[i] && p->tri[i] != p->tri[i]))
      return fail(DREAM_ERR_ARGUMENT, "triplets differ from the plan's (create a new plan)");
  }
  PlainLaunch L;
  memset(&L, 0, sizeof(L));
  L.method = effective_method(p);
  L.uni = true;
  L.Y = dY;
  L.K = p->K;
  L.No = p->No;
  L.Nt = p->Nt;
  L.Nr = p->Nr;
  L.Nx = p->Nx;
  L.Ny = p->Ny;
  L.Nz = p->Nz;
  L.Im = dIm;
  L.oob = doob;
  for (int i = 0; i < 15; i++) {
    L.tri64[i] = tri[i];
    L.tri32[i] = (float)tri[i];
  }
  if (p->precision == DREAM_PREC_F64) L.c64 = constants_f64(dt, cp, delay);
  else L.c32 = constants_uni_f32((float)dt, (float)cp, (float)delay);
  if (p->No == 0) return 0;
  if (p->K == 0) return zero_length_ascans(p, dIm, doob, st);
  return launch_plain(p, L, st);
}

int dream_das_uni_run_device(dream_das_plan *p, const void *dY, const double *tri, double dt, double delay,
                             double cp, void *dIm, int err_level, int64_t *oob_count, void *stream) {
  DREAM_API_TRY
  if (p == nullptr || !p->uni) return fail(DREAM_ERR_ARGUMENT, "not a uniform-grid plan");
  if (tri == nullptr) return fail(DREAM_ERR_ARGUMENT, "tri is NULL");
  if (p->cancelled.load()) return fail(DREAM_ERR_CANCELLED, "DAS cancelled");
  std::lock_guard<std::mutex> lk(p->mu);
  DeviceGuard g(p->device);
  cudaStream_t st = (cudaStream_t)stream;  // NULL: the default stream
  unsigned long long *doob = (unsigned long long *)p->bOob.p;
  CU(cudaMemsetAsync(doob, 0, sizeof(unsigned long long), st));
  int r = uni_launch(p, dY, tri, dt, delay, cp, dIm, doob, st);
  if (r) return r;
  CU(cudaMemcpyAsync(p->h_oob, doob, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  uint64_t oob = *p->h_oob;
  if (oob_count) *oob_count = (int64_t)oob;
  return status_from_oob(oob, err_level);
  DREAM_API_CATCH
}

int dream_das_uni_run(dream_das_plan *p, const void *Y, const double *tri, double dt, double delay, double cp,
                      void *Im, int err_level, int64_t *oob_count) {
  DREAM_API_TRY
  if (p == nullptr || !p->uni) return fail(DREAM_ERR_ARGUMENT, "not a uniform-grid plan");
  if (tri == nullptr) return fail(DREAM_ERR_ARGUMENT, "tri is NULL");
  if (p->cancelled.load()) return fail(DREAM_ERR_CANCELLED, "DAS cancelled");
  std::lock_guard<std::mutex> lk(p->mu);
  DeviceGuard g(p->device);
  cudaStream_t st = p->stream;
  const size_t es = prec_size(p->precision);
  const int64_t ncol = num_columns(p);
  int r;
  if ((r = p->bY.ensure((size_t)p->K * ncol * es))) return r;
  if ((r = p->bIm.ensure((size_t)p->No * es))) return r;
  if (p->K * ncol > 0) CU(cudaMemcpyAsync(p->bY.p, Y, (size_t)p->K * ncol * es, cudaMemcpyHostToDevice, st));
  unsigned long long *doob = (unsigned long long *)p->bOob.p;
  CU(cudaMemsetAsync(doob, 0, sizeof(unsigned long long), st));
  r = uni_launch(p, p->bY.p, tri, dt, delay, cp, p->bIm.p, doob, st);
  if (r) return r;
  if (p->No > 0) CU(cudaMemcpyAsync(Im, p->bIm.p, (size_t)p->No * es, cudaMemcpyDeviceToHost, st));
  CU(cudaMemcpyAsync(p->h_oob, doob, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  uint64_t oob = *p->h_oob;
  if (oob_count) *oob_count = (int64_t)oob;
  return status_from_oob(oob, err_level);
  DREAM_API_CATCH
}

}  // extern "C"
