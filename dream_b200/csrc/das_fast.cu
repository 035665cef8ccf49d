// das_fast.cu -- DAS with FP32- or BF16-stored A-scans, FP32 compensated
// accumulation and FP64-exact sample indices (precision upgrade of the
// reference's das_double/das_float forms; optional per-column weights for
// the differentiable operator).
//
// Index exactness. A term's sample index is trunc(RN(RN(a + b) * Fs)) with
// a, b the two FP64 leg times of the reference (extra_src/das.cc:392-404 and
// its RCA/SAFT counterparts). Each leg is computed exactly once per (pixel,
// element) in FP64, scaled by Fs in FP64 (A = RN(a*Fs), B = RN(b*Fs)) and
// stored as fixed point with 24 fraction bits relative to a tile-wide integer
// base. For A + B the fixed-point sum differs from the exact product
// RN(RN(a+b)*Fs) by less than 2^-24 + 4 ulp(p), so floor(A + B + delta) with
// delta = 2^-22 equals the exact floor whenever the fractional part of the
// shifted sum is at least 2*delta. Terms inside that 2^-21-wide band (about
// one in a million) take an exact FP64 recomputation. The selected indices
// are therefore identical to the FP64 plain kernel's.
//
// Hot loop. The fixed-point leg carries the A-scan column offset in its high
// word: with A64 = (offset_t + baseA) << 32 | fraction and the same for B, one
// 64-bit add gives the sample's element offset in the high word and the
// fraction in the low word, so a term costs: 64-bit add, one compare, address,
// load, add.
//
// Tiles. A CTA owns a 2-D tile of image points (tile_f along the fastest grid
// axis x tile_s along the next one, when the caller gives the grid's fastest
// extent n_fast; otherwise consecutive points). Warps are 8 x 4 points so the
// 32 gathers of one warp fall on one or two 128-byte lines of the A-scan.
#include <cuda_bf16.h>

#include "das_common.cuh"
#include "das_fast.h"

namespace dream {

namespace {

constexpr int FB = 24;                 // fraction bits of the relative legs
constexpr uint32_t DELTA_UNITS = 4;    // delta = 2^-22 in 2^-24 units
constexpr uint32_t AMB_LO = 8u << 8;   // 2*delta in the 2^-32 units of the low word
constexpr int JC = 16;                 // inner elements per register chunk
constexpr int MAX_EXTENT = 126;        // max integer spread of a leg over a tile

template <class YT>
__device__ __forceinline__ float load_sample(const YT *p);
template <>
__device__ __forceinline__ float load_sample<float>(const float *p) {
  return __ldg(p);
}
template <>
__device__ __forceinline__ float load_sample<__nv_bfloat16>(const __nv_bfloat16 *p) {
  unsigned short u = __ldg(reinterpret_cast<const unsigned short *>(p));
  return __uint_as_float(((unsigned int)u) << 16);
}

// base + off elements as one 32x32->64 multiply-add, which runs on the FMA
// pipe and leaves the integer ALU to the index arithmetic.
template <class YT>
__device__ __forceinline__ const YT *elem_addr(const YT *base, uint32_t off) {
  const YT *r;
  asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(r) : "r"(off), "r"((uint32_t)sizeof(YT)), "l"(base));
  return r;
}

// Neumaier compensated add of x into (s, c).
__device__ __forceinline__ void neumaier(float &s, float &c, float x) {
  float t = s + x;
  float e = (fabsf(s) >= fabsf(x)) ? ((s - t) + x) : ((x - t) + s);
  c += e;
  s = t;
}

struct Pixel {
  double xo, yo, zo, delay_ms, gy_c, gx_r;
};

__device__ __forceinline__ double A_mul_Fs(const FastParams &P, double leg) { return Ar<double>::mul(leg, P.Fs); }

__device__ __forceinline__ void pixel_of(const FastParams &P, int64_t no, Pixel &px) {
  using A = Ar<double>;
  px.xo = P.Ro[no];
  px.yo = P.Ro[no + P.No];
  px.zo = P.Ro[no + 2 * P.No];
  px.delay_ms = P.delay[P.delay_multi ? no : 0] / 1000.0;
  px.gy_c = 0.0;
  px.gx_r = 0.0;
  if (P.method == RCA_COLTX || P.method == RCA_ROWTX) {
    // literal stripe-edge reads of extra_src/das.cc:464-467
    const double gc_y_min = P.Gr[0 + 1 * P.Nt], gc_y_max = P.Gr[P.Nt - 1 + 1 * P.Nt];
    const double gr_x_min = P.Gt[0], gr_x_max = P.Gt[P.Nr - 1];
    if (px.yo >= gc_y_min && px.yo <= gc_y_max) px.gy_c = 0.0;
    else if (px.yo < gc_y_min) px.gy_c = A::sub(gc_y_min, px.yo);
    else px.gy_c = A::sub(gc_y_max, px.yo);
    if (px.xo >= gr_x_min && px.xo <= gr_x_max) px.gx_r = 0.0;
    else if (px.xo < gr_x_min) px.gx_r = A::sub(gr_x_min, px.xo);
    else px.gx_r = A::sub(gr_x_max, px.xo);
  }
}

// Exact FP64 leg of outer element o / inner element i, including the delay on
// the leg that carries it (TFM and col-tx: outer; row-tx: inner, the column).
__device__ __forceinline__ double outer_leg(const FastParams &P, const Pixel &px, int o) {
  using A = Ar<double>;
  double l;
  if (P.method == TFM) {
    l = leg_time(A::sub(P.Gt[o], px.xo), A::sub(P.Gt[o + P.Nt], px.yo), A::sub(P.Gt[o + 2 * P.Nt], px.zo), P.ocp);
  } else if (P.method == RCA_COLTX) {
    l = leg_time(A::sub(P.Gt[o], px.xo), px.gy_c, A::sub(P.Gt[o + 2 * P.Nt], px.zo), P.ocp);
  } else {  // row-tx: outer = rows
    l = leg_time(px.gx_r, A::sub(P.Gr[o + P.Nr], px.yo), A::sub(P.Gr[o + 2 * P.Nr], px.zo), P.ocp);
  }
  return (P.method == RCA_ROWTX) ? l : A::add(l, px.delay_ms);
}

__device__ __forceinline__ double inner_leg(const FastParams &P, const Pixel &px, int i) {
  using A = Ar<double>;
  double l;
  if (P.method == TFM) {
    l = leg_time(A::sub(P.Gr[i], px.xo), A::sub(P.Gr[i + P.Nr], px.yo), A::sub(P.Gr[i + 2 * P.Nr], px.zo), P.ocp);
  } else if (P.method == RCA_COLTX) {
    l = leg_time(px.gx_r, A::sub(P.Gr[i + P.Nr], px.yo), A::sub(P.Gr[i + 2 * P.Nr], px.zo), P.ocp);
  } else {  // row-tx: inner = columns, carrying the delay
    l = A::add(leg_time(A::sub(P.Gt[i], px.xo), px.gy_c, A::sub(P.Gt[i + 2 * P.Nt], px.zo), P.ocp), px.delay_ms);
  }
  return l;
}

// The reference's exact index of term (o, i): returns false when out of bounds.
__device__ __noinline__ bool exact_index(const FastParams &P, const Pixel &px, int o, int i, int &k) {
  using A = Ar<double>;
  double p = A::mul(A::add(outer_leg(P, px, o), inner_leg(P, px, i)), P.Fs);
  if (P.K > 0 && p > -1.0 && p < (double)P.K) {
    k = trunc_index(p);
    return true;
  }
  return false;
}

// Scaled leg -> integer floor and 24-bit fixed point v = floor << 24 + frac,
// the same arithmetic wherever a leg is converted. ok = false for legs of
// 2^26 samples or more: beyond that the FP64 rounding of A + B is no longer
// far enough below delta, and the tile takes the exact path.
__device__ __forceinline__ uint32_t fix24(double L, int &fl, bool &ok) {
  ok = fabs(L) < 67108864.0;  // 2^26
  double f = floor(ok ? L : 0.0);
  fl = (int)f;
  uint32_t frac = (uint32_t)__double2uint_rn((L - f) * 16777216.0);  // in [0, 2^24]
  return ((uint32_t)fl << FB) + frac;
}

struct TileShared {
  int *minA, *maxA, *minB, *maxB;
  uint32_t *ahi;   // [n_out]: high word of the outer legs (column offset + base)
  uint32_t *arel;  // [n_out][nthreads]
  int *flags;      // [0]: extent or range failure
};

// Exact partial sum of terms (o, i0 .. i0+jn-1): every index through the FP64
// recomputation. Taken for the rare chunks holding an ambiguous or
// out-of-range term, so the hot loop below stays free of calls.
template <class YT, bool WEIGHTED>
__device__ __noinline__ float exact_partial(const FastParams &P, const Pixel &px, int o, int i0, int jn, int n_in,
                                            unsigned int &oob) {
  const YT *__restrict__ Y = reinterpret_cast<const YT *>(P.Y);
  float part = 0.0f;
  for (int j = 0; j < jn; j++) {
    int k;
    const int64_t col = (int64_t)o * n_in + i0 + j;
    if (exact_index(P, px, o, i0 + j, k)) {
      float y = load_sample(Y + col * P.K + k);
      part = WEIGHTED ? fmaf(__ldg(P.w + col), y, part) : part + y;
    } else {
      oob++;
    }
  }
  return part;
}

// One outer element against a chunk of JN inner elements (JN = JC for full
// chunks, so the unrolled body carries no per-term predicates). Gathers are
// issued unconditionally: in an in-bounds tile every floor index, ambiguous
// or not, lies inside its A-scan. Ambiguity is tracked as the minimum
// fraction word; a chunk whose minimum falls in the band is recomputed.
template <class YT, bool WEIGHTED, bool CHECKED, bool FULL>
__device__ __forceinline__ float chunk_terms(const FastParams &P, const Pixel &px, const uint64_t (&B64)[JC],
                                             uint64_t A64, int64_t colbase, int o, int i0, int jn, int n_in,
                                             unsigned int &oob) {
  const YT *__restrict__ Y = reinterpret_cast<const YT *>(P.Y);
  const int64_t K = P.K;
  float y[JC];
  uint32_t minlo = 0xffffffffu;
  bool bad = false;
#pragma unroll
  for (int j = 0; j < JC; j++) {
    y[j] = 0.0f;
    if (FULL || j < jn) {
      const uint64_t s = A64 + B64[j];
      const uint32_t lo = (uint32_t)s;
      const uint32_t off = (uint32_t)(s >> 32);
      minlo = min(minlo, lo);
      if (CHECKED) {
        const int64_t col0 = (colbase + i0 + j) * K;
        const int32_t kk = (int32_t)(off - (uint32_t)col0);  // floor index, exact modulo 2^32
        const bool in = kk >= 0 && kk < K;
        bad |= !in;
        if (in) y[j] = load_sample(Y + col0 + kk);
      } else {
        y[j] = load_sample(elem_addr(Y, off));
      }
    }
  }
  float part = 0.0f;
  if (WEIGHTED) {
    const float *w = P.w + colbase + i0;
    if (FULL && ((reinterpret_cast<uintptr_t>(w) & 15) == 0)) {
#pragma unroll
      for (int j = 0; j < JC; j += 4) {
        float4 w4 = __ldg(reinterpret_cast<const float4 *>(w + j));
        part = fmaf(w4.x, y[j], part);
        part = fmaf(w4.y, y[j + 1], part);
        part = fmaf(w4.z, y[j + 2], part);
        part = fmaf(w4.w, y[j + 3], part);
      }
    } else {
#pragma unroll
      for (int j = 0; j < JC; j++)
        if (FULL || j < jn) part = fmaf(__ldg(w + j), y[j], part);
    }
  } else {
#pragma unroll
    for (int j = 0; j < JC; j++) part += y[j];
  }
  if (minlo < AMB_LO || bad) part = exact_partial<YT, WEIGHTED>(P, px, o, i0, jn, n_in, oob);
  return part;
}

template <class YT, bool WEIGHTED, bool CHECKED>
__device__ __forceinline__ void tile_loop(const FastParams &P, const Pixel &px, const TileShared &S, int tid,
                                          int nthr, int n_out, int n_in, float &acc_s, float &acc_c,
                                          unsigned int &oob) {
  const int64_t K = P.K;
  for (int i0 = 0; i0 < n_in; i0 += JC) {
    const int jn = min(JC, n_in - i0);
    uint64_t B64[JC];
#pragma unroll
    for (int j = 0; j < JC; j++) {
      B64[j] = 0;
      if (j < jn) {
        const int i = i0 + j;
        int fl;
        bool ok;
        uint32_t v = fix24(A_mul_Fs(P, inner_leg(P, px, i)), fl, ok);
        uint32_t brel = v - ((uint32_t)S.minB[i] << FB);
        uint32_t hi = (uint32_t)(i * K + S.minB[i]);
        B64[j] = ((uint64_t)brel << 8) + ((uint64_t)hi << 32);
      }
    }
    if (jn == JC) {
      // compensation every two outer elements (32 terms)
      int o = 0;
      for (; o + 2 <= n_out; o += 2) {
        const uint64_t A0 = ((uint64_t)S.arel[o * nthr + tid] << 8) + ((uint64_t)S.ahi[o] << 32);
        const uint64_t A1 = ((uint64_t)S.arel[(o + 1) * nthr + tid] << 8) + ((uint64_t)S.ahi[o + 1] << 32);
        float part = chunk_terms<YT, WEIGHTED, CHECKED, true>(P, px, B64, A0, (int64_t)o * n_in, o, i0, JC,
                                                             n_in, oob);
        part += chunk_terms<YT, WEIGHTED, CHECKED, true>(P, px, B64, A1, (int64_t)(o + 1) * n_in, o + 1, i0,
                                                        JC, n_in, oob);
        neumaier(acc_s, acc_c, part);
      }
      for (; o < n_out; o++) {
        const uint64_t A0 = ((uint64_t)S.arel[o * nthr + tid] << 8) + ((uint64_t)S.ahi[o] << 32);
        neumaier(acc_s, acc_c,
                 chunk_terms<YT, WEIGHTED, CHECKED, true>(P, px, B64, A0, (int64_t)o * n_in, o, i0, JC, n_in, oob));
      }
    } else {
      for (int o = 0; o < n_out; o++) {
        const uint64_t A64 = ((uint64_t)S.arel[o * nthr + tid] << 8) + ((uint64_t)S.ahi[o] << 32);
        neumaier(acc_s, acc_c, chunk_terms<YT, WEIGHTED, CHECKED, false>(P, px, B64, A64, (int64_t)o * n_in, o,
                                                                         i0, jn, n_in, oob));
      }
    }
  }
}

}  // namespace

template <class YT, bool WEIGHTED>
__global__ void __launch_bounds__(256) das_fast_kernel(const FastParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int n_out = (P.method == RCA_ROWTX) ? P.Nr : P.Nt;
  const int n_in = (P.method == RCA_ROWTX) ? P.Nt : P.Nr;

  TileShared S;
  S.minA = reinterpret_cast<int *>(smem_raw);
  S.maxA = S.minA + n_out;
  S.minB = S.maxA + n_out;
  S.maxB = S.minB + n_in;
  S.flags = S.maxB + n_in;
  S.ahi = reinterpret_cast<uint32_t *>(S.flags + 4);
  S.arel = S.ahi + n_out;

  // ---- image point of this thread ----
  const int lf = lane % P.wf, ls = lane / P.wf;
  const int warps_f = P.tile_f / P.wf;
  const int wfi = warp % warps_f, wsi = warp / warps_f;
  const int64_t tfi = blockIdx.x, tsi = (int64_t)blockIdx.y + P.slow_tile0;
  const int64_t f = tfi * P.tile_f + wfi * P.wf + lf;
  const int64_t s = tsi * P.tile_s + wsi * (32 / P.wf) + ls;
  const bool active = f < P.n_fast && s < P.n_slow;
  const int64_t no = active ? s * P.n_fast + f : tsi * P.tile_s * P.n_fast + tfi * P.tile_f;

  Pixel px;
  pixel_of(P, no, px);

  for (int i = tid; i < n_out; i += nthr) {
    S.minA[i] = INT_MAX;
    S.maxA[i] = INT_MIN;
  }
  for (int i = tid; i < n_in; i += nthr) {
    S.minB[i] = INT_MAX;
    S.maxB[i] = INT_MIN;
  }
  if (tid == 0) S.flags[0] = 0;
  __syncthreads();

  // ---- pass 1: scaled legs, tile-wide integer ranges ----
  bool bad = false;
  for (int o = 0; o < n_out; o++) {
    int fl;
    bool ok;
    uint32_t v = fix24(A_mul_Fs(P, outer_leg(P, px, o)), fl, ok);
    bad |= !ok;
    S.arel[o * nthr + tid] = v;
    int mn = __reduce_min_sync(0xffffffffu, fl), mx = __reduce_max_sync(0xffffffffu, fl);
    if (lane == 0) {
      atomicMin(&S.minA[o], mn);
      atomicMax(&S.maxA[o], mx);
    }
  }
  for (int i = 0; i < n_in; i++) {
    int fl;
    bool ok;
    fix24(A_mul_Fs(P, inner_leg(P, px, i)), fl, ok);
    bad |= !ok;
    int mn = __reduce_min_sync(0xffffffffu, fl), mx = __reduce_max_sync(0xffffffffu, fl);
    if (lane == 0) {
      atomicMin(&S.minB[i], mn);
      atomicMax(&S.maxB[i], mx);
    }
  }
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&S.flags[0], 1);
  __syncthreads();

  // ---- tile classification (uniform) ----
  int ext = 0, loA = INT_MAX, hiA = INT_MIN, loB = INT_MAX, hiB = INT_MIN;
  for (int o = 0; o < n_out; o++) {
    ext = max(ext, S.maxA[o] - S.minA[o]);
    loA = min(loA, S.minA[o]);
    hiA = max(hiA, S.maxA[o]);
  }
  for (int i = 0; i < n_in; i++) {
    ext = max(ext, S.maxB[i] - S.minB[i]);
    loB = min(loB, S.minB[i]);
    hiB = max(hiB, S.maxB[i]);
  }
  const bool exact_tile = S.flags[0] != 0 || ext > MAX_EXTENT ||
                          (int64_t)n_out * n_in * P.K + (int64_t)hiA + hiB + 256 >= (int64_t(1) << 32) ||
                          (int64_t)loA + loB < -(int64_t(1) << 30);
  // a non-ambiguous term's floor index lies in [minA + minB, maxA + maxB + 2]
  const bool in_bounds = (int64_t)loA + loB >= 0 && (int64_t)hiA + hiB + 2 < P.K;

  float acc_s = 0.0f, acc_c = 0.0f;
  unsigned int oob = 0;
  const YT *__restrict__ Yp = reinterpret_cast<const YT *>(P.Y);
  if (exact_tile) {
    // every term through the exact FP64 index
    for (int o = 0; o < n_out; o++) {
      float part = 0.0f;
      for (int i = 0; i < n_in; i++) {
        int k;
        const int64_t col = (int64_t)o * n_in + i;
        if (exact_index(P, px, o, i, k)) {
          float y = load_sample(Yp + col * P.K + k);
          part = WEIGHTED ? fmaf(__ldg(P.w + col), y, part) : part + y;
        } else {
          oob++;
        }
      }
      neumaier(acc_s, acc_c, part);
    }
  } else {
    // rebase the outer legs on the tile minimum and add the delta shift
    for (int o = 0; o < n_out; o++)
      S.arel[o * nthr + tid] = S.arel[o * nthr + tid] - ((uint32_t)S.minA[o] << FB) + DELTA_UNITS;
    for (int o = tid; o < n_out; o += nthr) S.ahi[o] = (uint32_t)((int64_t)o * n_in * P.K + S.minA[o]);
    __syncthreads();
    if (in_bounds) tile_loop<YT, WEIGHTED, false>(P, px, S, tid, nthr, n_out, n_in, acc_s, acc_c, oob);
    else tile_loop<YT, WEIGHTED, true>(P, px, S, tid, nthr, n_out, n_in, acc_s, acc_c, oob);
  }
  if (active) P.Im[no] = acc_s + acc_c;
  add_count(P.oob, active ? oob : 0u);
}

// SAFT: one leg per term, t_dp = 2*(leg + delay); the FP64 index is computed
// per term (each term has its own element), samples from FP32/BF16 storage.
template <class YT, bool WEIGHTED>
__global__ void __launch_bounds__(256) das_fast_saft_kernel(const FastParams P) {
  using A = Ar<double>;
  const int64_t no_raw = P.no0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = no_raw < P.no1;
  const int64_t no = active ? no_raw : P.no0;
  Pixel px;
  pixel_of(P, no, px);
  const YT *__restrict__ Y = reinterpret_cast<const YT *>(P.Y);
  float acc_s = 0.0f, acc_c = 0.0f, part = 0.0f;
  unsigned int oob = 0;
  for (int n = 0; n < P.Nt; n++) {
    double l = leg_time(A::sub(P.Gt[n], px.xo), A::sub(P.Gt[n + P.Nt], px.yo), A::sub(P.Gt[n + 2 * P.Nt], px.zo),
                        P.ocp);
    double p = A::mul(A::mul(2.0, A::add(l, px.delay_ms)), P.Fs);
    if (P.K > 0 && p > -1.0 && p < (double)P.K) {
      float y = load_sample(Y + (int64_t)n * P.K + trunc_index(p));
      part = WEIGHTED ? fmaf(__ldg(P.w + n), y, part) : part + y;
    } else {
      oob++;
    }
    if ((n & 15) == 15) {
      neumaier(acc_s, acc_c, part);
      part = 0.0f;
    }
  }
  neumaier(acc_s, acc_c, part);
  if (active) P.Im[no] = acc_s + acc_c;
  add_count(P.oob, active ? oob : 0u);
}

__global__ void f32_to_bf16_kernel(const float *__restrict__ x, __nv_bfloat16 *__restrict__ y, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16_rn(x[i]);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

size_t fast_smem_bytes(const FastParams &P, int nthr) {
  const int n_out = (P.method == RCA_ROWTX) ? P.Nr : P.Nt;
  const int n_in = (P.method == RCA_ROWTX) ? P.Nt : P.Nr;
  return (size_t)(3 * n_out + 2 * n_in + 4) * sizeof(int) + (size_t)n_out * nthr * sizeof(uint32_t);
}

template <class YT, bool W>
static cudaError_t launch_fast_t(const FastParams &P, cudaStream_t st) {
  if (P.method == SAFT) {
    int64_t n = P.no1 - P.no0;
    if (n <= 0) return cudaSuccess;
    das_fast_saft_kernel<YT, W><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(P);
    return cudaGetLastError();
  }
  const int nthr = P.tile_f * P.tile_s;
  const size_t smem = fast_smem_bytes(P, nthr);
  auto kern = das_fast_kernel<YT, W>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int64_t gx = (P.n_fast + P.tile_f - 1) / P.tile_f;
  const int64_t gy = P.slow_tile1 - P.slow_tile0;
  if (gx <= 0 || gy <= 0) return cudaSuccess;
  dim3 grid((unsigned)gx, (unsigned)gy);
  kern<<<grid, nthr, smem, st>>>(P);
  return cudaGetLastError();
}

cudaError_t launch_fast(const FastParams &P, bool bf16, cudaStream_t st) {
  const bool W = P.w != nullptr;
  if (bf16) return W ? launch_fast_t<__nv_bfloat16, true>(P, st) : launch_fast_t<__nv_bfloat16, false>(P, st);
  return W ? launch_fast_t<float, true>(P, st) : launch_fast_t<float, false>(P, st);
}

cudaError_t convert_f32_to_bf16(const float *x, void *y, int64_t n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
  f32_to_bf16_kernel<<<blocks, 256, 0, st>>>(x, reinterpret_cast<__nv_bfloat16 *>(y), n);
  return cudaGetLastError();
}

}  // namespace dream
