// dreamrect.cu -- spatial impulse responses (SIR) of a rectangular
// transducer and of arrays of rectangular elements on the GPU: DREAM's
// dreamrect (src/dreamrect.cc:248-302, opencl/dreamrect.cl) and
// dream_arr_rect (src/dream_arr_rect.cc:192-244, src/arr_functions.cc)
// without attenuation, the models that produce the responses from which
// A-scans are synthesised.
//
// Array element m (one for dreamrect, at the origin) sees observation point
// n at Ro[n] - G[m] with the delay (delay - foc_m) - steer_m. Its
// a x b aperture is cut into dx x dy surface elements whose centres advance
// by repeated addition (ys += dy outer, xs += dx inner). Surface element e
// contributes
//   ai = (((w_m*v)*ds)/(2*pi*r)) / dt * 1000   to sample   it = rint((t - delay_m)/dt),
// t = (r*1000)/cp, r its distance to the point, and h[it] += ai in (m, e)
// order. Centres, focusing / steering delays and weights are computed on the
// host with the reference's own operations (libm for sin, cos, exp); every
// device operation is the correctly rounded IEEE one, unfused.
//
// Layout. One warp per observation point. An array element's terms lie
// between the travel times to the nearest and the farthest point of its
// rectangle (+-2 samples for the rounding of r and t); an element whose
// window misses [0, nt) has no in-bounds term and is skipped (its terms are
// counted out of bounds without being evaluated). The union of the live
// elements' windows sits in shared memory (sized on the host by the
// diameter of the array and the spread of its delays, up to 8 warps per
// CTA); longer windows are accumulated in the output column itself. The warp
// takes 32 consecutive terms of the live elements per step: lanes that hit
// the same sample are grouped (__match_any_sync) and the lowest lane of each
// group adds the group's amplitudes in lane order (as many shuffle steps as
// the largest group has members), so every sample receives its terms in the
// reference's order and the SIR equals the reference's bit for bit. Windows
// are only trusted where the rounding bound holds (sample magnitudes below
// 2^36); a term that still lands in [0, nt) outside its point's window is
// counted, and the launch is then repeated with every element live and
// every window [0, nt).
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
constexpr double RECT_WIN_TRUST = 68719476736.0;  // 2^36: sample magnitudes whose +-2 window margin is proven
// A sample-index estimate farther than this from a half-integer rounds like
// the exact chain: with sample magnitudes below RECT_WIN_TRUST the two differ
// by at most 10 * 2^-53 * 2^36 < 2^-13 samples.
constexpr double RECT_Q_SAFE = 0.5 - 1.0 / 1024.0;
constexpr unsigned RECT_MISS = 1u;      // a term fell in [0, nt) outside its point's window
constexpr unsigned RECT_LAST_OOB = 2u;  // a term of the array's last element was out of bounds

// One array element: centre, focusing and steering delays (us) and
// (weight*v)*ds, the numerator of its terms.
struct ArrElem {
  double gx, gy, gz, foc, steer, wvds;
};

struct RectParams {
  const double *Ro;
  int64_t No;
  const double *xs, *ys;  // surface-element centres (nx, ny)
  int nx, ny;
  const ArrElem *el;      // array elements (M)
  int64_t M;
  double dt, cp;
  double c1, inv_dt;      // 1000/cp and 1/dt, for the sample-index estimate
  double ab;              // |a| + |b|
  double half_a, half_b;  // a/2, b/2
  int64_t win;            // samples of a point's SIR window in shared memory (0: none)
  int64_t nt;
  const double *delay;
  int delay_multi;
  int full;               // every element live, windows [0, nt) in the output columns
  double *H;
  unsigned long long *oob;        // out-of-bounds terms
  unsigned int *flags;            // RECT_MISS | RECT_LAST_OOB
};

// The observation point as array element m sees it; `fast`: its sample
// magnitudes are below RECT_WIN_TRUST (windows and index estimates hold).
struct ElemView {
  double xo, yo, zo, rz2, dl, w;
  bool fast;
};

// Point n (reloaded from global memory: kept out of the term loop's registers).
__device__ __forceinline__ void elem_view(const RectParams &P, int64_t m, int64_t n, ElemView &V) {
  const double xo = __ldg(P.Ro + n), yo = __ldg(P.Ro + n + P.No), zo = __ldg(P.Ro + n + 2 * P.No);
  const double dlay = __ldg(P.delay + (P.delay_multi ? n : 0));
  const ArrElem *E = P.el + m;
  V.xo = __dsub_rn(xo, __ldg(&E->gx));
  V.yo = __dsub_rn(yo, __ldg(&E->gy));
  V.zo = __dsub_rn(zo, __ldg(&E->gz));
  V.rz2 = __dmul_rn(V.zo, V.zo);
  V.dl = __dsub_rn(__dsub_rn(dlay, __ldg(&E->foc)), __ldg(&E->steer));
  V.w = __ldg(&E->wvds);
  const double bound = ((fabs(V.xo) + fabs(V.yo) + fabs(V.zo) + P.ab) * fabs(P.c1) + fabs(V.dl)) * fabs(P.inv_dt);
  V.fast = !P.full && bound < RECT_WIN_TRUST;
}

// Sample index of a term at distance r, as the kernel computes it.
__device__ __forceinline__ double rect_q(double r, double dl, const RectParams &P) {
  const double t = __ddiv_rn(__dmul_rn(r, 1000.0), P.cp);
  return __ddiv_rn(__dsub_rn(t, dl), P.dt);
}

// Live test and sample window [lo, hi) of an element's terms: every surface
// element centre lies in the a x b rectangle, so r is between the distances
// to its nearest point and to its farthest corner. Unbounded where the
// margin is not proven (or in the repeated launch).
__device__ __forceinline__ bool elem_window(const RectParams &P, const ElemView &V, int64_t &lo, int64_t &hi) {
  const double ax = fabs(V.xo), ay = fabs(V.yo);
  const double ex = fmax(ax - P.half_a, 0.0), ey = fmax(ay - P.half_b, 0.0);
  const double fx = ax + P.half_a, fy = ay + P.half_b;
  if (!V.fast) {
    lo = 0;
    hi = P.nt;
    return true;
  }
  // sample estimates (within 2^-13 of the exact chain's, see RECT_Q_SAFE)
  const double qa = (sqrt(ex * ex + ey * ey + V.rz2) * P.c1 - V.dl) * P.inv_dt;
  const double qb = (sqrt(fx * fx + fy * fy + V.rz2) * P.c1 - V.dl) * P.inv_dt;
  const int64_t sa = __double2ll_rn(qa), sb = __double2ll_rn(qb);
  lo = min(sa, sb) - 2;
  hi = max(sa, sb) + 3;
  return lo < P.nt && hi > 0;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// One warp step: lane's term (if valid) at surface element (ix, iy) of the
// element V is added to its sample, every sample receiving its terms in lane
// order. Lanes that hit the same sample are grouped (__match_any_sync); the
// lowest lane of each group adds the group's amplitudes in lane order. When
// every group is a run of consecutive lanes (the common case: along a row
// the sample index changes monotonically on either side of the point's
// projection) the leaders read their run from the warp's 32 staged
// amplitudes, four per trip; otherwise they walk their member masks.
// SKIP: steps with no term in the SIR skip the amplitudes and the sums (arrays,
// whose live elements still place most terms outside short windows); without
// it the amplitude divisions overlap the index computation.
template <bool SKIP>
__device__ __forceinline__ void term_step(const RectParams &P, const ElemView &V, bool valid, int ix, int iy,
                                          int lane, int64_t w0, int64_t w1, double *h, double *stage,
                                          unsigned long long &oob, unsigned int &flags, bool last) {
  bool in = false;
  int64_t it = 0;
  double r = 1.0;  // idle lanes: a finite amplitude that is never added
  double ai = 0.0;
  if (valid) {
    const double rx = __dsub_rn(V.xo, __ldg(P.xs + ix));
    const double ry = __dsub_rn(V.yo, __ldg(P.ys + iy));
    r = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)), V.rz2));
    if (!SKIP) {
      ai = __ddiv_rn(V.w, __dmul_rn(RECT_TWO_PI, r));
      ai = __ddiv_rn(ai, P.dt);
      ai = __dmul_rn(ai, 1000.0);
    }
    // rint((t - dl)/dt), ties to even: the estimate where it is certain, else the exact chain
    const double qa = __dmul_rn(__dsub_rn(__dmul_rn(r, P.c1), V.dl), P.inv_dt);
    const double na = rint(qa);
    if (V.fast && fabs(qa - na) < RECT_Q_SAFE)
      it = (int64_t)na;
    else
      it = __double2ll_rn(rect_q(r, V.dl, P));
    in = it >= 0 && it < P.nt;
    oob += in ? 0u : 1u;
    if (!in && last) flags |= RECT_LAST_OOB;
    const bool inside = it >= w0 && it < w1;  // true whenever the window bound holds
    if (in && !inside) flags |= RECT_MISS;
    in = in && inside;
  }
  if (SKIP) {
    if (!__any_sync(0xffffffffu, in)) return;  // no term of this step lands in the SIR
    ai = __ddiv_rn(V.w, __dmul_rn(RECT_TWO_PI, r));
    ai = __ddiv_rn(ai, P.dt);
    ai = __dmul_rn(ai, 1000.0);
  }
  // lanes adding into the same sample form a group; the others get unique keys
  const unsigned long long key = in ? (unsigned long long)it : ~0ull - (unsigned long long)lane;
  const unsigned int group = __match_any_sync(0xffffffffu, key);
  const int len = __popc(group);
  const bool leader = in && (group & ((1u << lane) - 1u)) == 0u;  // lowest lane of its group
  // a run: the group's lanes are lane .. lane + len - 1
  const bool run = (group >> lane) == (len == 32 ? 0xffffffffu : (1u << len) - 1u);
  if (__all_sync(0xffffffffu, !leader || run)) {
    stage[lane] = ai;
    __syncwarp();
    if (leader) {
      double acc = __dadd_rn(h[it], ai);
      const double *q = stage + lane + 1;
      int k = len - 1;
      for (; k >= 4; k -= 4, q += 4) {
        acc = __dadd_rn(acc, q[0]);
        acc = __dadd_rn(acc, q[1]);
        acc = __dadd_rn(acc, q[2]);
        acc = __dadd_rn(acc, q[3]);
      }
      for (; k > 0; k--, q++) acc = __dadd_rn(acc, q[0]);
      h[it] = acc;
    }
  } else {
    // each leader walks its group's lanes in ascending order (its own first);
    // the warp takes as many steps as the largest group has members
    const unsigned int steps = __reduce_max_sync(0xffffffffu, leader ? (unsigned)len : 0u);
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
  }
  __syncwarp();  // this step's sums (and stage reads) complete before the next step
}

// ARR = false: dreamrect (one element at the origin, P.M == 1), ARR = true: arrays.
template <bool ARR>
__global__ void __launch_bounds__(RECT_WARPS * 32) rect_kernel(const RectParams P) {
  extern __shared__ __align__(16) double rect_dyn[];  // [warps][32] staged amplitudes, then [warps][P.win]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double *stage = rect_dyn + warp * 32;
  double *win_sm = rect_dyn + (blockDim.x >> 5) * 32 + (int64_t)warp * P.win;
  const int64_t n = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
  if (n >= P.No) return;  // whole warps only: no block-wide barrier below
  double *out = P.H + n * P.nt;
  ElemView V;
  // union of the live elements' windows
  int64_t lo = INT64_MAX, hi = INT64_MIN;
  bool live0 = false;  // dreamrect: its element is live
  if (!ARR) {
    elem_view(P, 0, n, V);
    live0 = elem_window(P, V, lo, hi);
  } else {
    for (int64_t m = lane; m < P.M; m += 32) {
      int64_t l, h;
      elem_view(P, m, n, V);
      if (elem_window(P, V, l, h)) {
        lo = min(lo, l);
        hi = max(hi, h);
      }
    }
    for (int o = 16; o; o >>= 1) {
      lo = min(lo, (int64_t)__shfl_xor_sync(0xffffffffu, (long long)lo, o));
      hi = max(hi, (int64_t)__shfl_xor_sync(0xffffffffu, (long long)hi, o));
    }
  }
  int64_t w0 = 0, w1 = 0;
  if ((ARR || live0) && lo < hi) {
    w0 = max((int64_t)0, lo);
    w1 = min(P.nt, hi);
  }
  const bool in_smem = !P.full && w1 - w0 <= P.win;
  // the SIR: shared-memory window (offset w0) or the output column itself
  double *h = in_smem ? win_sm - w0 : out;
  if (in_smem) {
    for (int64_t i = lane; i < P.win; i += 32) win_sm[i] = 0.0;
  } else {
    for (int64_t i = lane; i < P.nt; i += 32) out[i] = 0.0;
  }
  __syncwarp();
  const int64_t E = (int64_t)P.nx * P.ny;  // terms per element (> 0)
  unsigned long long oob = 0;
  unsigned int flags = 0;
  if (!ARR) {
    if (!live0) {  // no term in bounds
      if (lane == 0) {
        oob = (unsigned long long)E;
        flags = RECT_LAST_OOB;
      }
    } else {
      // this lane's surface element e = iy*nx + ix, advanced by 32 per step without a division
      int iy = lane / P.nx;
      int ix = lane - iy * P.nx;
      for (int64_t e0 = 0; e0 < E; e0 += 32) {
        term_step<false>(P, V, e0 + lane < E, ix, iy, lane, w0, w1, h, stage, oob, flags, true);
        ix += 32;
        while (ix >= P.nx) {  // once for rows of 32 or more elements
          ix -= P.nx;
          iy++;
        }
      }
    }
  } else {
    for (int64_t c0 = 0; c0 < P.M; c0 += 32) {
      // the next 32 elements: dead ones only add to the out-of-bounds count
      bool live = false;
      if (c0 + lane < P.M) {
        int64_t l, h2;
        elem_view(P, c0 + lane, n, V);
        live = elem_window(P, V, l, h2);
        if (!live) {
          oob += (unsigned long long)E;
          if (c0 + lane == P.M - 1) flags |= RECT_LAST_OOB;
        }
      }
      const unsigned int L = __ballot_sync(0xffffffffu, live);
      if (L == 0u) continue;
      const int64_t total = (int64_t)__popc(L) * E;
      // this lane's term: live element j (its bits still set in `rest`), surface element (ix, iy)
      const int64_t j = lane / E, e = lane - j * E;
      int iy = (int)(e / P.nx);
      int ix = (int)(e - (int64_t)iy * P.nx);
      unsigned int rest = L;
      for (int64_t k = 0; k < j && rest; k++) rest &= rest - 1u;
      bool last = rest && c0 + __ffs(rest) - 1 == P.M - 1;  // this lane's element is the array's last
      if (rest) elem_view(P, c0 + __ffs(rest) - 1, n, V);
      for (int64_t g0 = 0; g0 < total; g0 += 32) {
        term_step<true>(P, V, g0 + lane < total, ix, iy, lane, w0, w1, h, stage, oob, flags, last);
        // advance by 32 terms without a division (once per wrap for rows of 32 or more)
        ix += 32;
        bool next = false;
        while (ix >= P.nx) {
          ix -= P.nx;
          if (++iy == P.ny) {
            iy = 0;
            rest &= rest - 1u;
            next = true;
          }
        }
        if (next && rest) {
          last = c0 + __ffs(rest) - 1 == P.M - 1;
          elem_view(P, c0 + __ffs(rest) - 1, n, V);
        }
      }
    }
  }
  if (in_smem) {
    for (int64_t i = lane; i < P.nt; i += 32) out[i] = (i >= w0 && i < w1) ? win_sm[i - w0] : 0.0;
  }
  oob = warp_sum_u64(oob);
  flags = __reduce_or_sync(0xffffffffu, flags);
  if (lane == 0) {
    if (oob) atomicAdd(P.oob, oob);
    if (flags) atomicOr(P.flags, flags);
  }
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
  double *centres = nullptr, *Ro = nullptr, *delay = nullptr, *H = nullptr, *elems = nullptr;
  size_t cap_c = 0, cap_ro = 0, cap_d = 0, cap_h = 0, cap_e = 0;
  unsigned long long *ctr = nullptr;  // [0] out-of-bounds terms, [1] RECT_* flags (low word)
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

// Array description: element centres G (M x 3, column-major) and the
// focusing, steering and apodisation settings, all on the host.
struct ArrDesc {
  int64_t M = 1;
  bool single = true;         // dreamrect: one element at the origin (G unused)
  const double *G = nullptr;
  int foc_met = DREAM_FOC_OFF, steer_met = DREAM_STEER_OFF, apod_met = DREAM_APOD_OFF;
  const double *focal = nullptr, *apod = nullptr;
  double theta = 0.0, phi = 0.0, apod_par = 0.0;
};

// Per-element centres, delays and term numerators, with the reference's
// operations in its order (max_dim_arr, focusing, beamsteering and
// apodization of src/arr_functions.cc:60-262, called as
// src/dream_arr_rect.cc:206-234 calls them; weight*v*ds of
// src/dreamrect.cc:306). Host code is compiled without contraction, so each
// product and sum is rounded on its own, and sin / cos / exp are the C
// library's, as in the reference's build.
int arr_elements(const ArrDesc &A, double v, double cp, double ds, std::vector<ArrElem> &out) {
  const int64_t M = A.M;
  out.assign((size_t)M, ArrElem{0.0, 0.0, 0.0, 0.0, 0.0, 0.0});
  if (M == 0) return 0;
  if (A.single) {  // dreamrect: one element at the origin, unit weight
    out[0].wvds = 1.0 * v * ds;
    return 0;
  }
  const double *gx = A.G, *gy = A.G + M, *gz = A.G + 2 * M;
  double x_max = std::fabs(gx[0]), y_max = std::fabs(gy[0]);
  for (int64_t i = 1; i < M; i++)
    if (std::fabs(gx[i]) > x_max) x_max = std::fabs(gx[i]);
  for (int64_t i = 1; i < M; i++)
    if (std::fabs(gy[i]) > y_max) y_max = std::fabs(gy[i]);
  const double r_max = std::sqrt(x_max * x_max + y_max * y_max);
  const double pi = 3.14159265358979323846, deg2rad = pi / 180.0;
  for (int64_t n = 0; n < M; n++) {
    ArrElem &el = out[(size_t)n];
    el.gx = gx[n];
    el.gy = gy[n];
    el.gz = gz[n];
    double foc = 0.0;
    if (A.foc_met == DREAM_FOC_UD) {
      foc = A.focal[n];
    } else if (A.foc_met != DREAM_FOC_OFF) {
      const double f = A.focal[0];
      double diff = 0.0;
      switch (A.foc_met) {
        case DREAM_FOC_X: diff = std::sqrt(x_max * x_max + f * f) - std::sqrt(gx[n] * gx[n] + f * f); break;
        case DREAM_FOC_Y: diff = std::sqrt(y_max * y_max + f * f) - std::sqrt(gy[n] * gy[n] + f * f); break;
        case DREAM_FOC_XY:
          diff = std::sqrt(r_max * r_max + f * f) - std::sqrt(gx[n] * gx[n] + gy[n] * gy[n] + f * f);
          break;
        default: {  // DREAM_FOC_X_Y
          const double rx = std::sqrt(gx[n] * gx[n] + f * f), ry = std::sqrt(gy[n] * gy[n] + f * f);
          diff = std::sqrt(r_max * r_max + f * f) - (rx + ry);
        }
      }
      foc = diff * 1.0e3 / cp;
    }
    double steer = 0.0;
    if (A.steer_met == DREAM_STEER_X || A.steer_met == DREAM_STEER_XY) {
      const double sx = std::sin(A.theta * deg2rad);
      steer = (x_max * sx + gx[n] * sx) * 1.0e3 / cp;
    }
    if (A.steer_met == DREAM_STEER_Y || A.steer_met == DREAM_STEER_XY) {
      const double sy = std::sin(A.phi * deg2rad);
      const double st_y = (y_max * sy + gy[n] * sy) * 1.0e3 / cp;
      steer = A.steer_met == DREAM_STEER_XY ? steer + st_y : st_y;
    }
    double w = 1.0;
    if (A.apod_met != DREAM_APOD_OFF) {
      const double r = std::sqrt(gx[n] * gx[n] + gy[n] * gy[n]);
      const double c = 1.0 - r * r / (r_max * r_max);
      switch (A.apod_met) {
        case DREAM_APOD_UD: w = A.apod[n]; break;
        case DREAM_APOD_TRIANGLE: w = 1.0 - std::fabs(r) / r_max; break;
        case DREAM_APOD_GAUSS: w = std::exp(-(A.apod_par * r * r) / (r_max * r_max)); break;
        case DREAM_APOD_RAISED: w = A.apod_par + std::cos(r * pi / r_max); break;
        case DREAM_APOD_HANN: w = 0.5 * (1.0 - std::cos((r + r_max) * pi / r_max)); break;
        case DREAM_APOD_HAMMING: {
          const double a0 = 25.0 / 46.0;
          w = a0 - (1.0 - a0) * std::cos((r + r_max) * pi / r_max);
        } break;
        case DREAM_APOD_SIMPLY: w = c; break;
        default: w = c * c;  // DREAM_APOD_CLAMPED
      }
    }
    el.foc = foc;
    el.steer = steer;
    el.wvds = w * v * ds;
  }
  return 0;
}

int check_desc(const ArrDesc &A) {
  if (A.M < 0) return set_last_error(DREAM_ERR_ARGUMENT, "dream_arr_rect: negative number of elements");
  if (!A.single && A.M > 0 && A.G == nullptr)
    return set_last_error(DREAM_ERR_ARGUMENT, "dream_arr_rect: NULL element grid");
  if (A.foc_met < DREAM_FOC_OFF || A.foc_met > DREAM_FOC_UD)
    return set_last_error(DREAM_ERR_ARGUMENT, "dream_arr_rect: unknown focusing method");
  if (A.steer_met < DREAM_STEER_OFF || A.steer_met > DREAM_STEER_XY)
    return set_last_error(DREAM_ERR_ARGUMENT, "dream_arr_rect: unknown beam steering method");
  if (A.apod_met < DREAM_APOD_OFF || A.apod_met > DREAM_APOD_UD)
    return set_last_error(DREAM_ERR_ARGUMENT, "dream_arr_rect: unknown apodization method");
  if (A.foc_met != DREAM_FOC_OFF && A.focal == nullptr)
    return set_last_error(DREAM_ERR_ARGUMENT, "dream_arr_rect: NULL focal");
  if (A.apod_met == DREAM_APOD_UD && A.apod == nullptr)
    return set_last_error(DREAM_ERR_ARGUMENT, "dream_arr_rect: NULL apodization weights");
  return 0;
}

// Shared-memory window bound of a launch: no point's union window is wider
// than the travel-time difference across the array's extent (the element
// rectangles around their centres) plus the spread of the element delays,
// +-2 samples per side and rounding.
int64_t window_bound(const std::vector<ArrElem> &el, double a, double b, double dt, double cp, int64_t nt) {
  double x0 = INFINITY, x1 = -INFINITY, y0 = INFINITY, y1 = -INFINITY, z0 = INFINITY, z1 = -INFINITY;
  double d0 = INFINITY, d1 = -INFINITY;
  for (const ArrElem &e : el) {
    x0 = std::min(x0, e.gx), x1 = std::max(x1, e.gx);
    y0 = std::min(y0, e.gy), y1 = std::max(y1, e.gy);
    z0 = std::min(z0, e.gz), z1 = std::max(z1, e.gz);
    d0 = std::min(d0, e.foc + e.steer), d1 = std::max(d1, e.foc + e.steer);
  }
  const double ex = x1 - x0 + std::fabs(a), ey = y1 - y0 + std::fabs(b), ez = z1 - z0;
  const double span =
      (std::sqrt(ex * ex + ey * ey + ez * ez) * 1000.0 / std::fabs(cp) + (d1 - d0)) / std::fabs(dt);
  if (!std::isfinite(span) || span > (double)nt) return nt;
  return std::min<int64_t>(nt, (int64_t)(span * (1.0 + 1e-9)) + 16);
}

// With the device current and the buffers locked: SIRs of the points in dRo
// into dH (device pointers), status from the out-of-bounds count.
int rect_device(RectBuffers &rb, const double *dRo, int64_t No, double a, double b, double dx, double dy, double dt,
                int64_t nt, int delay_type, const double *ddelay, double v, double cp, const ArrDesc &A, double *dH,
                int err_level, int64_t *oob_count, cudaStream_t st) {
  const char *fn = A.single ? "dreamrect" : "dream_arr_rect";
  if (No < 0 || nt < 0) return set_last_error(DREAM_ERR_ARGUMENT, std::string(fn) + ": negative size");
  if (delay_type != DREAM_DELAY_SINGLE && delay_type != DREAM_DELAY_MULTIPLE)
    return set_last_error(DREAM_ERR_ARGUMENT, "unknown delay type");
  int r = check_desc(A);
  if (r) return r;
  std::vector<double> xs, ys;
  if ((r = rect_centres(a, b, dx, dy, xs, ys))) return r;
  std::vector<ArrElem> el;
  if ((r = arr_elements(A, v, cp, dx * dy, el))) return r;
  if (oob_count) *oob_count = 0;
  const size_t nx = xs.size(), ny = ys.size();
  const uint64_t terms = (uint64_t)A.M * nx * ny;
  if (No == 0) return 0;
  if (nt == 0) {  // no sample to land in: every term is out of bounds
    const uint64_t all = (uint64_t)No * terms;
    if (oob_count) *oob_count = (int64_t)all;
    return status_of(all, err_level);  // the last element's terms are out of bounds too
  }
  if (dRo == nullptr || ddelay == nullptr || dH == nullptr) return set_last_error(DREAM_ERR_ARGUMENT, "NULL pointer");
  cudaError_t e = cudaSuccess;
  if (rb.ctr == nullptr && (e = cudaMalloc(&rb.ctr, 2 * sizeof(unsigned long long))) != cudaSuccess)
    return set_last_error(DREAM_ERR_ALLOC, cudaGetErrorString(e));
  if (terms == 0) {  // no surface element: the SIRs are zero
    e = cudaMemsetAsync(dH, 0, (size_t)No * nt * 8, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return set_last_error(DREAM_ERR_CUDA, std::string(fn) + ": " + cudaGetErrorString(e));
    return 0;
  }
  if ((r = grow(rb.centres, rb.cap_c, (nx + ny) * 8)) || (r = grow(rb.elems, rb.cap_e, el.size() * sizeof(ArrElem))))
    return r;
  std::vector<double> both(xs);
  both.insert(both.end(), ys.begin(), ys.end());
  e = cudaMemcpyAsync(rb.centres, both.data(), both.size() * 8, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(rb.elems, el.data(), el.size() * sizeof(ArrElem), cudaMemcpyHostToDevice, st);
  RectParams P;
  P.Ro = dRo;
  P.No = No;
  P.xs = rb.centres;
  P.ys = rb.centres + nx;
  P.nx = (int)nx;
  P.ny = (int)ny;
  P.el = reinterpret_cast<const ArrElem *>(rb.elems);
  P.M = A.M;
  P.half_a = a / 2.0;
  P.half_b = b / 2.0;
  P.dt = dt;
  P.cp = cp;
  P.c1 = 1000.0 / cp;
  P.inv_dt = 1.0 / dt;
  P.ab = std::fabs(a) + std::fabs(b);
  P.nt = nt;
  P.delay = ddelay;
  P.delay_multi = delay_type == DREAM_DELAY_MULTIPLE;
  P.H = dH;
  P.oob = rb.ctr;
  P.flags = reinterpret_cast<unsigned int *>(rb.ctr + 1);
  unsigned long long h_ctr[2] = {0, 0};
  const auto kernel = A.single ? rect_kernel<false> : rect_kernel<true>;
  if (e == cudaSuccess) e = ensure_smem(kernel, RECT_SMEM_MAX);
  for (int full = 0; full < 2 && e == cudaSuccess; full++) {
    int64_t win = full ? 0 : window_bound(el, a, b, dt, cp, nt);
    int warps = RECT_WARPS;
    while (warps > 1 && (int64_t)warps * (win + 32) * 8 > RECT_SMEM_MAX) warps >>= 1;
    if ((int64_t)warps * (win + 32) * 8 > RECT_SMEM_MAX) {  // very long windows: accumulate in the output columns
      win = 0;
      warps = RECT_WARPS;
    }
    P.win = win;
    P.full = full;
    const unsigned grid = (unsigned)((No + warps - 1) / warps);
    e = cudaMemsetAsync(rb.ctr, 0, sizeof(h_ctr), st);
    if (e == cudaSuccess) kernel<<<grid, warps * 32, (size_t)warps * (win + 32) * sizeof(double), st>>>(P);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_ctr, rb.ctr, sizeof(h_ctr), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (!(h_ctr[1] & RECT_MISS)) break;  // every term fell in its point's window
  }
  if (e != cudaSuccess) return set_last_error(DREAM_ERR_CUDA, std::string(fn) + ": " + cudaGetErrorString(e));
  if (oob_count) *oob_count = (int64_t)h_ctr[0];
  // the reference keeps, per point, the status of the array's last element
  // (src/dream_arr_rect.cc:209-243); 'stop' ends at the first out-of-bounds term
  return status_of(err_level == DREAM_ERR_LEVEL_STOP ? h_ctr[0] : (h_ctr[1] & RECT_LAST_OOB), err_level);
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

namespace {

int rect_entry_device(const double *dRo, int64_t No, double a, double b, double dx, double dy, double dt,
                      int64_t nt, int delay_type, const double *ddelay, double v, double cp, const ArrDesc &A,
                      double *dH, int err_level, int64_t *oob_count, int device, void *stream) {
  int r = check_device(device);
  if (r) return r;
  RectBuffers &rb = rect_buffers(device);
  std::lock_guard<std::mutex> lk(rb.mu);
  DeviceScope ds(device);
  if (!ds.ok) return set_last_error(DREAM_ERR_CUDA, "cudaSetDevice failed");
  return rect_device(rb, dRo, No, a, b, dx, dy, dt, nt, delay_type, ddelay, v, cp, A, dH, err_level, oob_count,
                     (cudaStream_t)stream);
}

int rect_entry_host(const double *Ro, int64_t No, double a, double b, double dx, double dy, double dt, int64_t nt,
                    int delay_type, const double *delay, double v, double cp, const ArrDesc &A, double *H,
                    int err_level, int64_t *oob_count, int device) {
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
  int st = rect_device(rb, rb.Ro, No, a, b, dx, dy, dt, nt, delay_type, rb.delay, v, cp, A, rb.H, err_level,
                       oob_count, rb.st);
  if (st < 0) return st;
  if (No > 0 && nt > 0) {
    e = cudaMemcpyAsync(H, rb.H, (size_t)No * nt * 8, cudaMemcpyDeviceToHost, rb.st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(rb.st);
    if (e != cudaSuccess) return set_last_error(DREAM_ERR_CUDA, cudaGetErrorString(e));
  }
  return st;
}

ArrDesc arr_desc(int64_t num_elements, const double *G, int foc_met, const double *focal, int steer_met,
                 double theta, double phi, int apod_met, const double *apod, double apod_par) {
  ArrDesc A;
  A.single = false;
  A.M = num_elements;
  A.G = G;
  A.foc_met = foc_met;
  A.focal = focal;
  A.steer_met = steer_met;
  A.theta = theta;
  A.phi = phi;
  A.apod_met = apod_met;
  A.apod = apod;
  A.apod_par = apod_par;
  return A;
}

}  // namespace

int dream_rect_run_device(const double *dRo, int64_t No, double a, double b, double dx, double dy, double dt,
                          int64_t nt, int delay_type, const double *ddelay, double v, double cp, double *dH,
                          int err_level, int64_t *oob_count, int device, void *stream) {
  DREAM_API_TRY
  return rect_entry_device(dRo, No, a, b, dx, dy, dt, nt, delay_type, ddelay, v, cp, ArrDesc(), dH, err_level,
                           oob_count, device, stream);
  DREAM_API_CATCH
}

int dream_rect_run(const double *Ro, int64_t No, double a, double b, double dx, double dy, double dt, int64_t nt,
                   int delay_type, const double *delay, double v, double cp, double *H, int err_level,
                   int64_t *oob_count, int device) {
  DREAM_API_TRY
  return rect_entry_host(Ro, No, a, b, dx, dy, dt, nt, delay_type, delay, v, cp, ArrDesc(), H, err_level, oob_count,
                         device);
  DREAM_API_CATCH
}

int dream_arr_rect_run_device(const double *dRo, int64_t No, double a, double b, double dx, double dy, double dt,
                              int64_t nt, int delay_type, const double *ddelay, double v, double cp,
                              int64_t num_elements, const double *G, int foc_met, const double *focal,
                              int steer_met, double theta, double phi, int apod_met, const double *apod,
                              double apod_par, double *dH, int err_level, int64_t *oob_count, int device,
                              void *stream) {
  DREAM_API_TRY
  if (num_elements > 0 && G == nullptr) return set_last_error(DREAM_ERR_ARGUMENT, "dream_arr_rect: NULL element grid");
  return rect_entry_device(dRo, No, a, b, dx, dy, dt, nt, delay_type, ddelay, v, cp,
                           arr_desc(num_elements, G, foc_met, focal, steer_met, theta, phi, apod_met, apod, apod_par),
                           dH, err_level, oob_count, device, stream);
  DREAM_API_CATCH
}

int dream_arr_rect_run(const double *Ro, int64_t No, double a, double b, double dx, double dy, double dt,
                       int64_t nt, int delay_type, const double *delay, double v, double cp, int64_t num_elements,
                       const double *G, int foc_met, const double *focal, int steer_met, double theta, double phi,
                       int apod_met, const double *apod, double apod_par, double *H, int err_level,
                       int64_t *oob_count, int device) {
  DREAM_API_TRY
  if (num_elements > 0 && G == nullptr) return set_last_error(DREAM_ERR_ARGUMENT, "dream_arr_rect: NULL element grid");
  return rect_entry_host(Ro, No, a, b, dx, dy, dt, nt, delay_type, delay, v, cp,
                         arr_desc(num_elements, G, foc_met, focal, steer_met, theta, phi, apod_met, apod, apod_par),
                         H, err_level, oob_count, device);
  DREAM_API_CATCH
}

}  // extern "C"
