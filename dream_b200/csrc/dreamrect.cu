// dreamrect.cu -- spatial impulse response (SIR) of a rectangular transducer
// on the GPU: DREAM's dreamrect without attenuation (src/dreamrect.cc:248-302,
// opencl/dreamrect.cl), the model that produces the responses from which
// A-scans are synthesised.
//
// For observation point n, the aperture [-a/2, a/2] x [-b/2, b/2] is cut into
// dx x dy surface elements whose centres advance by repeated addition
// (ys += dy outer, xs += dx inner). Element e contributes
//   ai = ((v*ds)/(2*pi*r)) / dt * 1000   to sample   it = rint((t - delay)/dt),
// t = (r*1000)/cp, r its distance to the point, and h[it] += ai in element
// order. The centres are computed on the host with the reference's own
// additions; every operation is the correctly rounded IEEE one, unfused.
//
// Layout. One warp per observation point. The samples a point can receive
// lie between the travel times to the nearest and the farthest point of the
// a x b rectangle (+-2 samples), at most the travel-time difference across
// its diagonal; that window of the SIR sits in shared memory (sized by the
// diagonal bound, up to 8 warps per CTA), windows beyond 192 KB per CTA are
// accumulated in the output column itself. The warp
// takes 32 consecutive elements per step: lanes that hit the same sample are
// grouped (__match_any_sync) and the lowest lane of each group adds the
// group's amplitudes in lane order (as many shuffle steps as the largest
// group has members), so every sample receives its terms in element order
// and the SIR equals the reference's bit for bit.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "das_common.cuh"
#include "das_kernels.h"
#include "dream_sir.h"

namespace dream {
namespace {

constexpr double RECT_TWO_PI = 2 * 3.14159265358979323846;  // 2*M_PI as the reference evaluates it
constexpr int RECT_WARPS = 8;                     // observation points per CTA
constexpr int64_t RECT_SMEM_MAX = 192 * 1024;     // shared memory for the CTA's SIR windows

struct RectParams {
  const double *Ro;
  int64_t No;
  const double *xs, *ys;  // element centres (nx, ny)
  int nx, ny;
  double ds, dt, v, cp;
  double half_a, half_b;  // a/2, b/2
  int64_t win;             // samples of a point's SIR window in shared memory (0: none)
  int64_t nt;
  const double *delay;
  int delay_multi;
  double *H;
  unsigned long long *oob;
};

// Sample index of a term at distance r, as the kernel computes it.
__device__ __forceinline__ int64_t rect_sample(double r, double dlay, const RectParams &P) {
  const double t = __ddiv_rn(__dmul_rn(r, 1000.0), P.cp);
  return __double2ll_rn(__ddiv_rn(__dsub_rn(t, dlay), P.dt));  // rint, ties to even
}

__global__ void __launch_bounds__(RECT_WARPS * 32) rect_kernel(const RectParams P) {
  extern __shared__ __align__(16) double rect_dyn[];  // [warps][P.win]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double *win_sm = rect_dyn + (int64_t)warp * P.win;
  const int64_t n = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
  if (n >= P.No) return;  // whole warps only: no block-wide barrier below
  const double xo = P.Ro[n], yo = P.Ro[n + P.No], zo = P.Ro[n + 2 * P.No];
  const double dlay = P.delay[P.delay_multi ? n : 0];
  double *out = P.H + n * P.nt;
  // Window of samples this point can receive: every element centre lies in
  // the a x b rectangle, so r is between the distances to its nearest point
  // and to its farthest corner; +-2 samples cover the rounding of r and t.
  const double ex = fmax(fabs(xo) - P.half_a, 0.0), ey = fmax(fabs(yo) - P.half_b, 0.0);
  const double fx = fabs(xo) + P.half_a, fy = fabs(yo) + P.half_b;
  const double r_lo = sqrt(ex * ex + ey * ey + zo * zo), r_hi = sqrt(fx * fx + fy * fy + zo * zo);
  const int64_t s_a = rect_sample(r_lo, dlay, P), s_b = rect_sample(r_hi, dlay, P);
  const int64_t w0 = max((int64_t)0, min(s_a, s_b) - 2), w1 = min(P.nt, max(s_a, s_b) + 3);
  const bool in_smem = w1 - w0 <= P.win;
  // the SIR: shared-memory window (offset w0) or the output column itself
  double *h = in_smem ? win_sm - w0 : out;
  if (in_smem) {
    for (int64_t i = lane; i < P.win; i += 32) win_sm[i] = 0.0;
  } else {
    for (int64_t i = lane; i < P.nt; i += 32) out[i] = 0.0;
  }
  __syncwarp();
  const double rz2 = __dmul_rn(zo, zo);
  const double vds = __dmul_rn(P.v, P.ds);
  const int64_t E = (int64_t)P.nx * P.ny;
  unsigned int oob = 0;
  // this lane's element e = iy*nx + ix, advanced by 32 per step without a division
  int64_t iy = lane / P.nx;
  int ix = lane - (int)(iy * P.nx);
  for (int64_t e0 = 0; e0 < E; e0 += 32) {
    const int64_t e = e0 + lane;
    bool in = false;
    int64_t it = 0;
    double ai = 0.0;
    if (e < E) {
      const double rx = __dsub_rn(xo, __ldg(P.xs + ix));
      const double ry = __dsub_rn(yo, __ldg(P.ys + iy));
      const double r = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)), rz2));
      ai = __ddiv_rn(vds, __dmul_rn(RECT_TWO_PI, r));
      ai = __ddiv_rn(ai, P.dt);
      ai = __dmul_rn(ai, 1000.0);
      it = rect_sample(r, dlay, P);
      in = it >= 0 && it < P.nt;
      oob += in ? 0u : 1u;
      in = in && it >= w0 && it < w1;  // always true in the window's derivation; guards the shared slot
    }
    // lanes adding into the same sample form a group; the others get unique keys
    const unsigned long long key = in ? (unsigned long long)it : ~0ull - (unsigned long long)lane;
    const unsigned int group = __match_any_sync(0xffffffffu, key);
    const bool leader = in && (__ffs(group) - 1) == lane;
    // each leader walks its group's lanes in ascending order (its own first);
    // the warp takes as many steps as the largest group has members
    const unsigned int steps = __reduce_max_sync(0xffffffffu, leader ? (unsigned)__popc(group) : 0u);
    double acc = leader ? h[it] : 0.0;
    unsigned int rem = leader ? group : 0u;
    for (unsigned int k = 0; k < steps; k++) {
      const int src = rem ? __ffs(rem) - 1 : lane;
      const bool add = rem != 0u;
      rem &= rem - 1u;
      const double aj = __shfl_sync(0xffffffffu, ai, src);
      if (add) acc = __dadd_rn(acc, aj);
    }
    if (leader) h[it] = acc;
    __syncwarp();  // this step's sums are visible to the next step's leaders
    ix += 32;
    while (ix >= P.nx) {  // once for rows of 32 or more elements
      ix -= P.nx;
      iy++;
    }
  }
  if (in_smem) {
    for (int64_t i = lane; i < P.nt; i += 32) out[i] = (i >= w0 && i < w1) ? win_sm[i - w0] : 0.0;
  }
  add_count(P.oob, oob);
}

// Element centres exactly as the reference's loops produce them.
int rect_centres(double a, double b, double dx, double dy, std::vector<double> &xs, std::vector<double> &ys) {
  if (!(dx > 0.0) || !(dy > 0.0)) return set_last_error(DREAM_ERR_ARGUMENT, "dreamrect: dx and dy must be positive");
  const double xsmin = -a / 2.0, xsmax = a / 2.0, ysmin = -b / 2.0, ysmax = b / 2.0;
  xs.clear();
  ys.clear();
  for (double x = xsmin + dx / 2.0; x <= xsmax; x += dx) {
    xs.push_back(x);
    if (xs.size() > (size_t(1) << 24)) return set_last_error(DREAM_ERR_ARGUMENT, "dreamrect: too many x elements");
  }
  for (double y = ysmin + dy / 2.0; y <= ysmax; y += dy) {
    ys.push_back(y);
    if (ys.size() > (size_t(1) << 24)) return set_last_error(DREAM_ERR_ARGUMENT, "dreamrect: too many y elements");
  }
  return 0;
}

struct RectBuffers {
  std::mutex mu;
  double *centres = nullptr, *Ro = nullptr, *delay = nullptr, *H = nullptr;
  size_t cap_c = 0, cap_ro = 0, cap_d = 0, cap_h = 0;
  unsigned long long *oob = nullptr;
  cudaStream_t st = nullptr;
};

int grow(double *&p, size_t &cap, size_t bytes) {
  if (bytes <= cap) return 0;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return set_last_error(DREAM_ERR_ALLOC, "dreamrect: device allocation failed");
  }
  cap = bytes;
  return 0;
}

RectBuffers &rect_buffers(int device) {
  static std::vector<RectBuffers> bufs(64);
  return bufs[device];
}

int status_of(uint64_t oob, int err_level) {
  if (oob == 0) return 0;
  switch (err_level) {
    case DREAM_ERR_LEVEL_IGNORE: return DREAM_STATUS_IGNORE_OUT_OF_BOUNDS;
    case DREAM_ERR_LEVEL_WARN: return DREAM_STATUS_WARN_OUT_OF_BOUNDS;
    case DREAM_ERR_LEVEL_STOP: return DREAM_STATUS_OUT_OF_BOUNDS;
    default: return DREAM_STATUS_NONE;
  }
}

// With the device current and the buffers locked: SIRs of the points in dRo
// into dH (device pointers), status from the out-of-bounds count.
int rect_device(RectBuffers &rb, const double *dRo, int64_t No, double a, double b, double dx, double dy, double dt,
                int64_t nt, int delay_type, const double *ddelay, double v, double cp, double *dH, int err_level,
                int64_t *oob_count, cudaStream_t st) {
  if (No < 0 || nt < 0) return set_last_error(DREAM_ERR_ARGUMENT, "dreamrect: negative size");
  if (delay_type != DREAM_DELAY_SINGLE && delay_type != DREAM_DELAY_MULTIPLE)
    return set_last_error(DREAM_ERR_ARGUMENT, "unknown delay type");
  std::vector<double> xs, ys;
  int r = rect_centres(a, b, dx, dy, xs, ys);
  if (r) return r;
  if (oob_count) *oob_count = 0;
  if (No == 0) return 0;
  if (nt == 0) {  // no sample to land in: every surface element is out of bounds
    const int64_t all = No * (int64_t)xs.size() * (int64_t)ys.size();
    if (oob_count) *oob_count = all;
    return status_of((uint64_t)all, err_level);
  }
  if (dRo == nullptr || ddelay == nullptr || dH == nullptr) return set_last_error(DREAM_ERR_ARGUMENT, "NULL pointer");
  cudaError_t e = cudaSuccess;
  if (rb.oob == nullptr && (e = cudaMalloc(&rb.oob, sizeof(unsigned long long))) != cudaSuccess)
    return set_last_error(DREAM_ERR_ALLOC, cudaGetErrorString(e));
  if ((r = grow(rb.centres, rb.cap_c, std::max<size_t>(1, xs.size() + ys.size()) * 8))) return r;
  const size_t nx = xs.size(), ny = ys.size();
  std::vector<double> both(xs);
  both.insert(both.end(), ys.begin(), ys.end());
  if (!both.empty()) e = cudaMemcpyAsync(rb.centres, both.data(), both.size() * 8, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(rb.oob, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return set_last_error(DREAM_ERR_CUDA, cudaGetErrorString(e));
  RectParams P;
  P.Ro = dRo;
  P.No = No;
  P.xs = rb.centres;
  P.ys = rb.centres + nx;
  P.nx = (int)nx;
  P.ny = (int)ny;
  P.ds = dx * dy;
  P.half_a = a / 2.0;
  P.half_b = b / 2.0;
  P.dt = dt;
  P.v = v;
  P.cp = cp;
  P.nt = nt;
  P.delay = ddelay;
  P.delay_multi = delay_type == DREAM_DELAY_MULTIPLE;
  P.H = dH;
  P.oob = rb.oob;
  if (nx == 0 || ny == 0) {  // no surface element: the SIRs are zero
    e = cudaMemsetAsync(dH, 0, (size_t)No * nt * 8, st);
  } else {
    // No point's window is wider than the travel-time difference across the
    // rectangle's diagonal (+ the +-2 margin and rounding): size the shared
    // windows by that bound, so short responses leave room for many warps.
    const double span = std::sqrt(a * a + b * b) * 1000.0 / std::fabs(cp) / std::fabs(dt);
    int64_t win = std::isfinite(span) ? std::min<int64_t>(nt, (int64_t)span + 8) : nt;
    int warps = RECT_WARPS;
    while (warps > 1 && (int64_t)warps * win * 8 > RECT_SMEM_MAX) warps >>= 1;
    if ((int64_t)warps * win * 8 > RECT_SMEM_MAX) {  // very long windows: accumulate in the output columns
      win = 0;
      warps = RECT_WARPS;
    }
    P.win = win;
    const unsigned grid = (unsigned)((No + warps - 1) / warps);
    const size_t bytes = (size_t)warps * win * sizeof(double);
    e = ensure_smem(rect_kernel, RECT_SMEM_MAX);
    if (e == cudaSuccess) rect_kernel<<<grid, warps * 32, bytes, st>>>(P);
    if (e == cudaSuccess) e = cudaGetLastError();
  }
  unsigned long long h_oob = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_oob, rb.oob, sizeof(h_oob), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return set_last_error(DREAM_ERR_CUDA, std::string("dreamrect: ") + cudaGetErrorString(e));
  if (oob_count) *oob_count = (int64_t)h_oob;
  return status_of(h_oob, err_level);
}

struct DeviceScope {
  int prev = -1;
  bool ok = true;
  explicit DeviceScope(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) ok = cudaSetDevice(dev) == cudaSuccess;
  }
  ~DeviceScope() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

int check_device(int device) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev || device >= 64)
    return set_last_error(DREAM_ERR_ARGUMENT, "invalid CUDA device ordinal");
  return 0;
}

}  // namespace
}  // namespace dream

using namespace dream;

extern "C" {

int dream_rect_run_device(const double *dRo, int64_t No, double a, double b, double dx, double dy, double dt,
                          int64_t nt, int delay_type, const double *ddelay, double v, double cp, double *dH,
                          int err_level, int64_t *oob_count, int device, void *stream) {
  int r = check_device(device);
  if (r) return r;
  RectBuffers &rb = rect_buffers(device);
  std::lock_guard<std::mutex> lk(rb.mu);
  DeviceScope ds(device);
  if (!ds.ok) return set_last_error(DREAM_ERR_CUDA, "cudaSetDevice failed");
  return rect_device(rb, dRo, No, a, b, dx, dy, dt, nt, delay_type, ddelay, v, cp, dH, err_level, oob_count,
                     (cudaStream_t)stream);
}

int dream_rect_run(const double *Ro, int64_t No, double a, double b, double dx, double dy, double dt, int64_t nt,
                   int delay_type, const double *delay, double v, double cp, double *H, int err_level,
                   int64_t *oob_count, int device) {
  int r = check_device(device);
  if (r) return r;
  if (No < 0 || nt < 0) return set_last_error(DREAM_ERR_ARGUMENT, "dreamrect: negative size");
  if (No > 0 && (Ro == nullptr || delay == nullptr || (nt > 0 && H == nullptr)))
    return set_last_error(DREAM_ERR_ARGUMENT, "NULL host pointer");
  RectBuffers &rb = rect_buffers(device);
  std::lock_guard<std::mutex> lk(rb.mu);
  DeviceScope ds(device);
  if (!ds.ok) return set_last_error(DREAM_ERR_CUDA, "cudaSetDevice failed");
  cudaError_t e = cudaSuccess;
  if (rb.st == nullptr && (e = cudaStreamCreateWithFlags(&rb.st, cudaStreamNonBlocking)) != cudaSuccess)
    return set_last_error(DREAM_ERR_CUDA, cudaGetErrorString(e));
  const size_t nd = delay_type == DREAM_DELAY_MULTIPLE ? (size_t)No : 1;
  if ((r = grow(rb.Ro, rb.cap_ro, std::max<size_t>(1, (size_t)No * 3) * 8)) ||
      (r = grow(rb.delay, rb.cap_d, std::max<size_t>(1, nd) * 8)) ||
      (r = grow(rb.H, rb.cap_h, std::max<size_t>(1, (size_t)No * nt) * 8)))
    return r;
  if (No > 0) {
    e = cudaMemcpyAsync(rb.Ro, Ro, (size_t)No * 3 * 8, cudaMemcpyHostToDevice, rb.st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(rb.delay, delay, nd * 8, cudaMemcpyHostToDevice, rb.st);
    if (e != cudaSuccess) return set_last_error(DREAM_ERR_CUDA, cudaGetErrorString(e));
  }
  int st = rect_device(rb, rb.Ro, No, a, b, dx, dy, dt, nt, delay_type, rb.delay, v, cp, rb.H, err_level, oob_count,
                       rb.st);
  if (st < 0) return st;
  if (No > 0 && nt > 0) {
    e = cudaMemcpyAsync(H, rb.H, (size_t)No * nt * 8, cudaMemcpyDeviceToHost, rb.st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(rb.st);
    if (e != cudaSuccess) return set_last_error(DREAM_ERR_CUDA, cudaGetErrorString(e));
  }
  return st;
}

}  // extern "C"
