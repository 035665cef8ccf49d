// das_plain.cu -- the plain DAS kernels: FP64 (DAS<double>) and FP32
// (DAS<float>) on arbitrary geometry (`das`) and on uniform grids (`das_uni`).
//
// These kernels are the drop-in replacement of the reference's per-pixel
// loops and keep their arithmetic exactly:
//   SAFT        extra_src/das.cc:306-357, opencl/das_uni_double.cl:9-77
//   TFM         extra_src/das.cc:365-427, opencl/das_uni_double.cl:79-167
//   RCA col-tx  extra_src/das.cc:437-529, opencl/das_uni_double.cl:169-281
//   RCA row-tx  extra_src/das.cc:533-626, opencl/das_uni_double.cl:283-394
// Each thread owns one image point and sums its terms in the reference order
// (outer element loop, inner element loop), so the image is bit-identical to
// the reference CPU code, not merely close to it. With a grid hint the warps
// take 8 x 4 patches of the image grid (PLAIN_PATCH_F x PLAIN_PATCH_S) instead
// of 32 consecutive points, which changes only which thread owns which point.
//
// What differs from the reference is where the work goes. The inner-loop
// element leg (receive leg for TFM/col-tx, column leg for row-tx) depends
// only on (pixel, inner element), so it is computed once per pixel into a
// per-thread shared-memory table instead of once per term; every term then
// costs one add, one multiply, the bounds test, the truncation and one
// gather from Y. Hoisting is exact: the leg is the same rounded value.
#include "das_common.cuh"
#include "das_kernels.h"

namespace dream {

template <class T>
struct PlainParams {
  const T *Y;
  int64_t K;
  const T *Ro;
  int64_t No;
  const T *Gt;
  int Nt;
  const T *Gr;
  int Nr;
  int64_t no0, no1;  // pixel range [no0, no1) of this launch, or patch-row range when n_fast > 0
  int64_t n_fast, n_slow;  // grid hint: warps take patches of (fast, slow) points
  const T *delay;  // das: device delays in us (1 value, or No when delay_multi)
  int delay_multi;
  T delay_ms;      // das_uni: the scalar delay in ms
  T Fs, ocp, Kf;
  T *Im;
  unsigned long long *oob;
  int64_t ny;               // elements in Y (bounds-checked builds)
  unsigned long long *bad;  // gather index violations (bounds-checked builds)
  int64_t *idx;             // index mode: idx[col * No + no] = sample index or -1
  int bigk;  // K >= 2^22 (FP32): use the conversion unit for truncation
  // uniform grids
  T tri[15];
  int64_t Nx, Ny, Nz;
};

// Truncation of p in (-1, K). Long A-scans (FP32, K >= 2^22) need the
// conversion unit; every other case uses the exact add-based form.
template <class T, bool BIGK>
__device__ __forceinline__ int to_index(T p) {
  if (BIGK) return __float2int_rz((float)p);
  return trunc_index(p);
}

// delay / 1000 the way each reference form computes it: DAS<double> in
// double, DAS<float> in double rounded to float (extra_src/das.cc:318).
__device__ __forceinline__ double delay_to_ms(double d) { return d / 1000.0; }
__device__ __forceinline__ float delay_to_ms(float d) {
  return __double2float_rn((double)d / 1000.0);
}

constexpr int UNROLL = 8;  // gathers in flight per thread before their in-order adds

// Sample ycol[off] of Y. The bounds-checked build tests the element index
// against the extent of Y first (a violation is counted and reads 0); the
// normal build is the plain load.
// FP64 addresses the sample from the base of Y with a 64-bit element index,
// FP32 from the column pointer: on a 64x64-element TFM frame (K 3000, 512x512
// points) each form is the faster one for its type (FP64 2.46 vs 2.86 ms,
// FP32 1.19 vs 1.36 ms).
template <class T>
__device__ __forceinline__ T load_y(const PlainParams<T> &P, const T *ycol, int64_t off) {
#ifdef DREAM_DAS_CHECKED
  const int64_t gi = (ycol - P.Y) + off;
  return gather_ok<T>(gi, P.ny, P.bad) ? __ldg(P.Y + gi) : (T)0;
#else
  if constexpr (sizeof(T) == 8) return __ldg(P.Y + ((ycol - P.Y) + off));
  else return __ldg(ycol + off);
#endif
}

// IDX: instead of gathering and summing, write every term's sample index
// (the one the gather would read; -1 for an out-of-bounds term) to P.idx.
// PATCH: warps take 2-D patches of the grid (P.n_fast > 0); a template
// parameter, so the consecutive-point kernel compiles as if it did not exist.
template <class T, int M, bool UNI, bool TAB, bool BIGK, bool IDX = false, bool PATCH = false>
__global__ void __launch_bounds__(256) das_plain_kernel(const PlainParams<T> P) {
  using A = Ar<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *tab = reinterpret_cast<T *>(smem_raw);
  const int tid = threadIdx.x;
  const int bd = blockDim.x;
  int64_t no_raw;
  bool active;
  if constexpr (PATCH) {
    // 2-D patches: warp w of block (x, y) covers PLAIN_PATCH_F points along
    // the grid's fast axis (patch x * warps + w) x PLAIN_PATCH_S along the
    // slow one (patch row no0 + y)
    const int lane = tid & 31;
    const int64_t f = ((int64_t)blockIdx.x * (bd >> 5) + (tid >> 5)) * PLAIN_PATCH_F + lane % PLAIN_PATCH_F;
    const int64_t s = (P.no0 + blockIdx.y) * PLAIN_PATCH_S + lane / PLAIN_PATCH_F;
    active = f < P.n_fast && s < P.n_slow;
    no_raw = s * P.n_fast + f;
  } else {
    no_raw = P.no0 + (int64_t)blockIdx.x * bd + tid;
    active = no_raw < P.no1;
  }
  const int64_t no = active ? no_raw : (PATCH ? 0 : P.no0);  // inactive lanes read a valid point and write nothing

  // ---- image point ----
  T xo, yo, zo;
  if (UNI) {
    // linear index -> (ny fastest, nz, nx)   (opencl/das_uni_double.cl:32-43)
    int64_t yq = no / P.Ny, ny = no - yq * P.Ny;
    int64_t zq = yq / P.Nz, nz = yq - zq * P.Nz;
    int64_t xq = zq / P.Nx, nx = zq - xq * P.Nx;
    xo = A::add(P.tri[6], A::mul((T)nx, P.tri[7]));
    yo = A::add(P.tri[9], A::mul((T)ny, P.tri[10]));
    zo = A::add(P.tri[12], A::mul((T)nz, P.tri[13]));
  } else {
    xo = P.Ro[no];
    yo = P.Ro[no + P.No];
    zo = P.Ro[no + 2 * P.No];
  }
  const T delay_ms = UNI ? P.delay_ms : delay_to_ms(P.delay[P.delay_multi ? no : 0]);

  // ---- element coordinates ----
  // transmit / column elements
  auto elem_t = [&](int n, T &ex, T &ey, T &ez) {
    if (UNI) {
      ex = A::add(P.tri[0], A::mul((T)n, P.tri[1]));
      ey = (T)0;
      ez = (T)0;
    } else {
      ex = P.Gt[n];
      ey = P.Gt[n + P.Nt];
      ez = P.Gt[n + 2 * P.Nt];
    }
  };
  // receive / row elements (uniform RCA rows lie along y)
  auto elem_r = [&](int n, T &ex, T &ey, T &ez) {
    if (UNI) {
      T c = A::add(P.tri[3], A::mul((T)n, P.tri[4]));
      if (M == RCA_COLTX || M == RCA_ROWTX) {
        ex = (T)0; ey = c;
      } else {
        ex = c; ey = (T)0;
      }
      ez = (T)0;
    } else {
      ex = P.Gr[n];
      ey = P.Gr[n + P.Nr];
      ez = P.Gr[n + 2 * P.Nr];
    }
  };

  // ---- RCA stripe clamps (extra_src/das.cc:464-467,475-486,493-503) ----
  T gy_c = (T)0, gx_r = (T)0;
  if (M == RCA_COLTX || M == RCA_ROWTX) {
    T gc_y_min, gc_y_max, gr_x_min, gr_x_max;
    if (UNI) {  // opencl/das_uni_double.cl:213-216
      gc_y_min = P.tri[3]; gc_y_max = P.tri[5];
      gr_x_min = P.tri[0]; gr_x_max = P.tri[2];
    } else {  // literal (num_cols/num_rows mixed) reads of the reference
      gc_y_min = P.Gr[0 + 1 * P.Nt];
      gc_y_max = P.Gr[P.Nt - 1 + 1 * P.Nt];
      gr_x_min = P.Gt[0];
      gr_x_max = P.Gt[P.Nr - 1];
    }
    if (yo >= gc_y_min && yo <= gc_y_max) gy_c = (T)0;
    else if (yo < gc_y_min) gy_c = A::sub(gc_y_min, yo);
    else gy_c = A::sub(gc_y_max, yo);
    if (UNI) {
      if (xo < gr_x_min || xo > gr_x_max) gx_r = (xo < gr_x_min) ? A::sub(gr_x_min, xo) : A::sub(gr_x_max, xo);
    } else {
      if (xo >= gr_x_min && xo <= gr_x_max) gx_r = (T)0;
      else if (xo < gr_x_min) gx_r = A::sub(gr_x_min, xo);
      else gx_r = A::sub(gr_x_max, xo);
    }
  }

  // leg of a column stripe / row stripe / point element
  auto leg_col = [&](int n) {
    T ex, ey, ez;
    elem_t(n, ex, ey, ez);
    return leg_time(A::sub(ex, xo), gy_c, A::sub(ez, zo), P.ocp);
  };
  auto leg_row = [&](int n) {
    T ex, ey, ez;
    elem_r(n, ex, ey, ez);
    return leg_time(gx_r, A::sub(ey, yo), A::sub(ez, zo), P.ocp);
  };
  auto leg_tx = [&](int n) {
    T ex, ey, ez;
    elem_t(n, ex, ey, ez);
    return leg_time(A::sub(ex, xo), A::sub(ey, yo), A::sub(ez, zo), P.ocp);
  };
  auto leg_rx = [&](int n) {
    T ex, ey, ez;
    elem_r(n, ex, ey, ez);
    return leg_time(A::sub(ex, xo), A::sub(ey, yo), A::sub(ez, zo), P.ocp);
  };

  T im = (T)0;
  unsigned int oob = 0;
  const T *ycol = P.Y;

  if (M == SAFT) {
    for (int n = 0; n < P.Nt; n++) {
      T t = A::add(leg_tx(n), delay_ms);
      T tdp = A::mul((T)2, t);  // exact doubling, as 2.0*t_tr
      T p = A::mul(tdp, P.Fs);
      if constexpr (IDX) {
        const bool v = p > (T)-1 && p < P.Kf;
        if (active) P.idx[(int64_t)n * P.No + no] = v ? (int64_t)to_index<T, BIGK>(p) : -1;
        oob += v ? 0 : 1;
      } else if (p > (T)-1 && p < P.Kf) {
        im = A::add(im, load_y(P, ycol, to_index<T, BIGK>(p)));
      } else {
        oob++;
      }
      ycol += P.K;
    }
  } else {
    // outer / inner element roles and which leg carries the delay
    const int n_out = (M == RCA_ROWTX) ? P.Nr : P.Nt;
    const int n_in = (M == RCA_ROWTX) ? P.Nt : P.Nr;
    // das row-tx: delay on the (inner) column leg; das_uni row-tx: on the
    // (outer) row leg (opencl/das_uni_double.cl:358-360).
    const bool delay_outer = (M != RCA_ROWTX) || UNI;
    auto inner_leg = [&](int i) -> T {
      T l;
      if (M == TFM) l = leg_rx(i);
      else if (M == RCA_COLTX) l = leg_row(i);
      else l = leg_col(i);
      return delay_outer ? l : A::add(l, delay_ms);
    };
    if (TAB) {
      for (int i = 0; i < n_in; i++) tab[i * bd + tid] = inner_leg(i);
    }
    for (int o = 0; o < n_out; o++) {
      T lo;
      if (M == TFM) lo = leg_tx(o);
      else if (M == RCA_COLTX) lo = leg_col(o);
      else lo = leg_row(o);
      if (delay_outer) lo = A::add(lo, delay_ms);
      int i = 0;
      // UNROLL terms at a time: all gathers are issued before the adds, which
      // then run in the reference order (the sum is unchanged bit for bit).
      for (; i + UNROLL <= n_in; i += UNROLL) {
        T y[UNROLL];
        bool v[UNROLL];
#pragma unroll
        for (int u = 0; u < UNROLL; u++) {
          T li = TAB ? tab[(i + u) * bd + tid] : inner_leg(i + u);
          T p = A::mul(A::add(lo, li), P.Fs);
          v[u] = p > (T)-1 && p < P.Kf;
          if constexpr (IDX) {
            if (active) P.idx[((int64_t)o * n_in + i + u) * P.No + no] = v[u] ? (int64_t)to_index<T, BIGK>(p) : -1;
            y[u] = (T)0;
          } else {
            y[u] = v[u] ? load_y(P, ycol, (int64_t)u * P.K + to_index<T, BIGK>(p)) : (T)0;
          }
        }
#pragma unroll
        for (int u = 0; u < UNROLL; u++) {
          if (v[u]) im = A::add(im, y[u]);
          else oob++;
        }
        ycol += UNROLL * P.K;
      }
      for (; i < n_in; i++) {
        T li = TAB ? tab[i * bd + tid] : inner_leg(i);
        T p = A::mul(A::add(lo, li), P.Fs);
        if constexpr (IDX) {
          const bool v = p > (T)-1 && p < P.Kf;
          if (active) P.idx[((int64_t)o * n_in + i) * P.No + no] = v ? (int64_t)to_index<T, BIGK>(p) : -1;
          oob += v ? 0 : 1;
        } else if (p > (T)-1 && p < P.Kf) {
          im = A::add(im, load_y(P, ycol, to_index<T, BIGK>(p)));
        } else {
          oob++;
        }
        ycol += P.K;
      }
    }
  }
  if (!IDX && active) P.Im[no] = im;
  add_count(P.oob, active ? oob : 0u);
}

// ---------------------------------------------------------------------------
// launcher
// ---------------------------------------------------------------------------

template <class T, int M, bool UNI, bool TAB, bool IDX = false>
static cudaError_t launch_one(const PlainParams<T> &P, int bd, size_t smem, cudaStream_t st) {
  const bool patch = P.n_fast > 0, bigk = sizeof(T) == 4 && P.bigk;
  auto kern = patch ? (bigk ? das_plain_kernel<T, M, UNI, TAB, true, IDX, true>
                            : das_plain_kernel<T, M, UNI, TAB, false, IDX, true>)
                    : (bigk ? das_plain_kernel<T, M, UNI, TAB, true, IDX, false>
                            : das_plain_kernel<T, M, UNI, TAB, false, IDX, false>);
  cudaError_t e = ensure_smem(kern, smem);
  if (e != cudaSuccess) return e;
  dim3 grid;
  if (patch) {  // [no0, no1) are patch rows; a block holds bd / 32 patches of a row
    const int64_t wpb = bd >> 5;
    grid = dim3((unsigned)(((P.n_fast + PLAIN_PATCH_F - 1) / PLAIN_PATCH_F + wpb - 1) / wpb), (unsigned)(P.no1 - P.no0));
  } else {
    grid = dim3((unsigned)((P.no1 - P.no0 + bd - 1) / bd));
  }
  kern<<<grid, bd, smem, st>>>(P);
  return cudaGetLastError();
}

template <class T, bool UNI, bool IDX = false>
static cudaError_t launch_method(int method, const PlainParams<T> &P, cudaStream_t st) {
  const int n_in = (method == SAFT) ? 0 : (method == RCA_ROWTX ? P.Nt : P.Nr);
  // Largest block whose per-thread inner-leg table fits in 64 KB (three
  // blocks per SM); very long inner loops fall back to recomputing the leg.
  int bd = 256;
  while (bd > 32 && (size_t)n_in * bd * sizeof(T) > 64 * 1024) bd >>= 1;
  bool tab = (size_t)n_in * bd * sizeof(T) <= 200 * 1024;
  if (!tab) bd = 128;
  size_t smem = tab ? (size_t)n_in * bd * sizeof(T) : 0;
  switch (method) {
    case SAFT: return launch_one<T, SAFT, UNI, false, IDX>(P, 256, 0, st);
    case TFM:
      return tab ? launch_one<T, TFM, UNI, true, IDX>(P, bd, smem, st)
                 : launch_one<T, TFM, UNI, false, IDX>(P, bd, 0, st);
    case RCA_COLTX:
      return tab ? launch_one<T, RCA_COLTX, UNI, true, IDX>(P, bd, smem, st)
                 : launch_one<T, RCA_COLTX, UNI, false, IDX>(P, bd, 0, st);
    case RCA_ROWTX:
      return tab ? launch_one<T, RCA_ROWTX, UNI, true, IDX>(P, bd, smem, st)
                 : launch_one<T, RCA_ROWTX, UNI, false, IDX>(P, bd, 0, st);
  }
  return cudaErrorInvalidValue;
}

template <class T>
static PlainParams<T> make_params(const PlainLaunch &L) {
  PlainParams<T> P{};
  P.Y = (const T *)L.Y;
  P.K = L.K;
  P.Ro = (const T *)L.Ro;
  P.No = L.No;
  P.no0 = L.no0;
  P.no1 = L.no1;
  P.n_fast = L.n_fast;
  P.n_slow = L.n_fast > 0 ? L.No / L.n_fast : 0;
  P.Gt = (const T *)L.Gt;
  P.Nt = (int)L.Nt;
  P.Gr = (const T *)L.Gr;
  P.Nr = (int)L.Nr;
  P.delay = (const T *)L.delay_vec;
  P.delay_multi = L.delay_multi ? 1 : 0;
  P.Im = (T *)L.Im;
  P.oob = L.oob;
  P.ny = L.ny;
  P.bad = L.bad;
  P.idx = L.idx;
  P.bigk = L.K >= (int64_t(1) << 22);
  P.Nx = L.Nx;
  P.Ny = L.Ny;
  P.Nz = L.Nz;
  return P;
}

cudaError_t launch_plain_f64(const PlainLaunch &L, cudaStream_t st) {
  PlainParams<double> P = make_params<double>(L);
  P.Fs = L.c64.Fs;
  P.ocp = L.c64.ocp;
  P.delay_ms = L.c64.delay_ms;
  P.Kf = (double)L.K;
  for (int i = 0; i < 15; i++) P.tri[i] = L.tri64[i];
  if (L.idx)
    return L.uni ? launch_method<double, true, true>(L.method, P, st)
                 : launch_method<double, false, true>(L.method, P, st);
  return L.uni ? launch_method<double, true>(L.method, P, st) : launch_method<double, false>(L.method, P, st);
}

cudaError_t launch_plain_f32(const PlainLaunch &L, cudaStream_t st) {
  PlainParams<float> P = make_params<float>(L);
  P.Fs = L.c32.Fs;
  P.ocp = L.c32.ocp;
  P.delay_ms = L.c32.delay_ms;
  P.Kf = (float)L.K;
  for (int i = 0; i < 15; i++) P.tri[i] = L.tri32[i];
  if (L.idx)
    return L.uni ? launch_method<float, true, true>(L.method, P, st)
                 : launch_method<float, false, true>(L.method, P, st);
  return L.uni ? launch_method<float, true>(L.method, P, st) : launch_method<float, false>(L.method, P, st);
}

}  // namespace dream
