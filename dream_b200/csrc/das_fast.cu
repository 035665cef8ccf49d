// das_fast.cu -- DAS with FP32- or BF16-stored A-scans, FP32 compensated
// accumulation and FP64-exact sample indices (precision upgrade of the
// reference's das_double/das_float forms; optional per-column weights for
// the differentiable operator).
//
// Index exactness. A term's sample index is trunc(RN(RN(a + b) * Fs)) with
// a, b the two FP64 leg times of the reference (extra_src/das.cc:392-404 and
// its RCA/SAFT counterparts). Each leg is computed exactly once per (pixel,
// element) in FP64, scaled by Fs in FP64 (A = RN(a*Fs), B = RN(b*Fs)) and
// stored as fixed point relative to a tile-wide integer base, in one of two
// formats chosen per tile:
//   fine: 24 fraction bits, legs spreading over < 127 samples in the tile;
//         rounding <= 2^-25 per leg, delta = 2^-22, band 2*delta = 2^-21;
//   wide: 20 fraction bits (coarse grids, spreads up to 4000 samples);
//         rounding <= 2^-21 per leg, delta = 2^-19, band 2^-18.
// For legs below 2^26 samples RN(a*Fs) + RN(b*Fs) differs from
// RN(RN(a+b)*Fs) by at most 3 ulp(2^27) < 2^-24.4, so in both formats the
// fixed-point sum is within delta of the exact p, and floor(A + B + delta)
// equals the exact floor whenever the fractional part of the shifted sum is
// at least 2*delta. Terms inside the band (about 1 in 2 million with the
// fine format) take an exact FP64 recomputation. The finer format matters
// for speed: a warp with one ambiguous lane runs the serial FP64 path. The
// selected indices are identical to the FP64 plain kernel's.
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

// Relative fixed-point format of a tile: fb fraction bits, shifted by
// lo_shift = 32 - fb to the top of the low word of A64 + B64; delta in 2^-fb
// units; amb_lo = 2*delta in the 2^-32 units of the low word.
struct FixFmt {
  int fb, lo_shift;
  uint32_t delta, amb_lo;
};
constexpr FixFmt FMT_FINE{24, 8, 4, 8u << 8};    // delta 2^-22
constexpr FixFmt FMT_WIDE{20, 12, 2, 4u << 12};  // delta 2^-19
constexpr int FINE_EXTENT = 126;                 // max integer spread of a leg over a tile, fine format
constexpr int WIDE_EXTENT = 4000;                // the same, wide format (< 2^12)

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

// Packed FP32 pairs (add.rn.f32x2 / fma.rn.f32x2, sm_100).
__device__ __forceinline__ uint64_t pack_f32x2(float a, float b) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ uint64_t add_f32x2(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ uint64_t fma_f32x2(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
__device__ __forceinline__ float lo_f32(uint64_t v) { return __uint_as_float((uint32_t)v); }
__device__ __forceinline__ float hi_f32(uint64_t v) { return __uint_as_float((uint32_t)(v >> 32)); }

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

// Elements in Y: K times the A-scan columns (Nt for SAFT, Nt*Nr otherwise).
__device__ __forceinline__ int64_t y_count(const FastParams &P) {
  return P.ny ? P.ny : P.K * (int64_t)P.Nt * (P.method == SAFT ? 1 : P.Nr);
}

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

// Scaled leg -> integer floor and fixed point v = floor << fb + frac (modulo
// 2^32), the same arithmetic wherever a leg is converted. ok = false for legs
// of 2^26 samples or more: beyond that the FP64 rounding of A + B is no
// longer far enough below delta, and the tile takes the exact path.
__device__ __forceinline__ uint32_t fix_leg(double L, int fb, int &fl, bool &ok) {
  ok = fabs(L) < 67108864.0;  // 2^26
  double f = floor(ok ? L : 0.0);
  fl = (int)f;
  uint32_t frac = (uint32_t)__double2uint_rn((L - f) * (double)(1u << fb));  // in [0, 2^fb]
  return ((uint32_t)fl << fb) + frac;
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
      const float y = gather_ok<float>(col * P.K + k, y_count(P), P.bad) ? load_sample(Y + col * P.K + k) : 0.0f;
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
template <class YT, bool WEIGHTED, bool CHECKED, bool FULL, int JC, int NO>
__device__ __forceinline__ float chunk_terms(const FastParams &P, const Pixel &px, const uint64_t (&B64)[JC],
                                             const uint64_t (&A64)[NO], int o0, int i0, int jn, int n_in,
                                             uint32_t amb_lo, unsigned int &oob) {
  // NO outer elements x JC inner elements: all NO*JC gathers are issued before
  // any (rare) call to the exact path, so they are in flight together.
  const YT *__restrict__ Y = reinterpret_cast<const YT *>(P.Y);
  const int64_t K = P.K;
  float y[NO][JC];
  uint32_t minlo[NO];
  unsigned int oob_chunk[NO];
#pragma unroll
  for (int q = 0; q < NO; q++) {
    minlo[q] = 0xffffffffu;
    oob_chunk[q] = 0;
#pragma unroll
    for (int j = 0; j < JC; j++) {
      y[q][j] = 0.0f;
      if (FULL || j < jn) {
        const uint64_t s = A64[q] + B64[j];
        const uint32_t lo = (uint32_t)s;
        const uint32_t off = (uint32_t)(s >> 32);
        minlo[q] = min(minlo[q], lo);
        if (CHECKED) {
          // Outside the ambiguity band the floor index is exact: [0, K) is in
          // bounds, -1 means p in (-1, 0), i.e. sample 0 after truncation, and
          // anything else is out of bounds.
          const int64_t col0 = ((int64_t)(o0 + q) * n_in + i0 + j) * K;
          const int32_t kk = (int32_t)(off - (uint32_t)col0);  // floor index, exact modulo 2^32
          if (kk >= 0 && kk < K) {
            if (gather_ok<float>(col0 + kk, y_count(P), P.bad)) y[q][j] = load_sample(Y + col0 + kk);
          } else if (kk == -1) {
            y[q][j] = load_sample(Y + col0);
          } else {
            oob_chunk[q]++;
          }
        } else {
          if (gather_ok<float>((int64_t)off, y_count(P), P.bad)) y[q][j] = load_sample(elem_addr(Y, off));
        }
      }
    }
  }
  float total = 0.0f;
  float partq[NO];
#pragma unroll
  for (int q = 0; q < NO; q++) {
    float part = 0.0f;
    if (WEIGHTED) {
      const float *w = P.w + (int64_t)(o0 + q) * n_in + i0;
      if (FULL && ((reinterpret_cast<uintptr_t>(w) & 15) == 0)) {
        uint64_t acc2 = 0;  // (+0, +0)
#pragma unroll
        for (int j = 0; j < JC; j += 4) {
          float4 w4 = __ldg(reinterpret_cast<const float4 *>(w + j));
          acc2 = fma_f32x2(pack_f32x2(w4.x, w4.y), pack_f32x2(y[q][j], y[q][j + 1]), acc2);
          acc2 = fma_f32x2(pack_f32x2(w4.z, w4.w), pack_f32x2(y[q][j + 2], y[q][j + 3]), acc2);
        }
        part = lo_f32(acc2) + hi_f32(acc2);
      } else {
#pragma unroll
        for (int j = 0; j < JC; j++)
          if (FULL || j < jn) part = fmaf(__ldg(w + j), y[q][j], part);
      }
    } else {
      // packed FP32x2 adds: half the instructions and half the dependency depth
      uint64_t acc2 = pack_f32x2(y[q][0], y[q][1]);
#pragma unroll
      for (int j = 2; j < JC; j += 2) acc2 = add_f32x2(acc2, pack_f32x2(y[q][j], y[q][j + 1]));
      part = lo_f32(acc2) + hi_f32(acc2);
    }
    partq[q] = part;
  }
#pragma unroll
  for (int q = 0; q < NO; q++) {
    if (minlo[q] < amb_lo) {
      // this outer element's partial is replaced by the exact one (which counts its own OOB)
      partq[q] = exact_partial<YT, WEIGHTED>(P, px, o0 + q, i0, jn, n_in, oob);
    } else {
      oob += oob_chunk[q];
    }
    total += partq[q];
  }
  return total;
}

template <class YT, bool WEIGHTED, bool CHECKED, int JC>
__device__ __forceinline__ void tile_loop(const FastParams &P, const Pixel &px, const TileShared &S, const FixFmt F,
                                          int tid,
                                          int nthr, int n_out, int n_in, int i_lo, int i_hi, float &acc_s,
                                          float &acc_c, unsigned int &oob) {
  const int64_t K = P.K;
  for (int i0 = i_lo; i0 < i_hi; i0 += JC) {
    const int jn = min(JC, i_hi - i0);
    uint64_t B64[JC];
#pragma unroll
    for (int j = 0; j < JC; j++) {
      B64[j] = 0;
      if (j < jn) {
        const int i = i0 + j;
        int fl;
        bool ok;
        uint32_t v = fix_leg(A_mul_Fs(P, inner_leg(P, px, i)), F.fb, fl, ok);
        uint32_t brel = v - ((uint32_t)S.minB[i] << F.fb);
        uint32_t hi = (uint32_t)(i * K + S.minB[i]);
        B64[j] = ((uint64_t)brel << F.lo_shift) + ((uint64_t)hi << 32);
      }
    }
    if (jn == JC) {
      // compensation every two outer elements (32 terms)
      int o = 0;
      for (; o + 2 <= n_out; o += 2) {
        const uint64_t A2[2] = {((uint64_t)S.arel[o * nthr + tid] << F.lo_shift) + ((uint64_t)S.ahi[o] << 32),
                                ((uint64_t)S.arel[(o + 1) * nthr + tid] << F.lo_shift) + ((uint64_t)S.ahi[o + 1] << 32)};
        neumaier(acc_s, acc_c, chunk_terms<YT, WEIGHTED, CHECKED, true, JC, 2>(P, px, B64, A2, o, i0, JC, n_in, F.amb_lo, oob));
      }
      for (; o < n_out; o++) {
        const uint64_t A1[1] = {((uint64_t)S.arel[o * nthr + tid] << F.lo_shift) + ((uint64_t)S.ahi[o] << 32)};
        neumaier(acc_s, acc_c, chunk_terms<YT, WEIGHTED, CHECKED, true, JC, 1>(P, px, B64, A1, o, i0, JC, n_in, F.amb_lo, oob));
      }
    } else {
      for (int o = 0; o < n_out; o++) {
        const uint64_t A1[1] = {((uint64_t)S.arel[o * nthr + tid] << F.lo_shift) + ((uint64_t)S.ahi[o] << 32)};
        neumaier(acc_s, acc_c, chunk_terms<YT, WEIGHTED, CHECKED, false, JC, 1>(P, px, B64, A1, o, i0, jn, n_in, F.amb_lo, oob));
      }
    }
  }
}

}  // namespace

// One tile of image points (tile indices tfi along the fast axis, tsi along
// the slow axis) with the frame described by P; smem_raw holds the tile's
// shared arrays (fast_smem_bytes). Called by the one-frame kernel and by the
// persistent batch kernel.
template <class YT, bool WEIGHTED, int JC>
__device__ __forceinline__ void fast_tile(const FastParams &P, int64_t tfi, int64_t tsi, unsigned char *smem_raw) {
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int n_out = (P.method == RCA_ROWTX) ? P.Nr : P.Nt;
  const int n_in = (P.method == RCA_ROWTX) ? P.Nt : P.Nr;
  // inner elements of this launch: all of them unless the caller sets a range
  const int i_lo = P.in_lo, i_hi = P.in_hi > 0 ? P.in_hi : n_in;

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
    uint32_t v = fix_leg(A_mul_Fs(P, outer_leg(P, px, o)), FMT_FINE.fb, fl, ok);
    bad |= !ok;
    S.arel[o * nthr + tid] = v;
    int mn = __reduce_min_sync(0xffffffffu, fl), mx = __reduce_max_sync(0xffffffffu, fl);
    if (lane == 0) {
      atomicMin(&S.minA[o], mn);
      atomicMax(&S.maxA[o], mx);
    }
  }
  for (int i = i_lo; i < i_hi; i++) {
    int fl;
    bool ok;
    fix_leg(A_mul_Fs(P, inner_leg(P, px, i)), FMT_FINE.fb, fl, ok);
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
  for (int i = i_lo; i < i_hi; i++) {
    ext = max(ext, S.maxB[i] - S.minB[i]);
    loB = min(loB, S.minB[i]);
    hiB = max(hiB, S.maxB[i]);
  }
  const bool exact_tile = S.flags[0] != 0 || ext > WIDE_EXTENT ||
                          (int64_t)n_out * n_in * P.K + (int64_t)hiA + hiB + 8448 >= (int64_t(1) << 32) ||
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
      for (int i = i_lo; i < i_hi; i++) {
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
    // format of this tile; rebase the outer legs on the tile minimum and add
    // the delta shift (the wide format converts the outer legs again)
    const FixFmt F = ext > FINE_EXTENT ? FMT_WIDE : FMT_FINE;
    for (int o = 0; o < n_out; o++) {
      uint32_t v = S.arel[o * nthr + tid];
      if (F.fb != FMT_FINE.fb) {
        int fl;
        bool ok;
        v = fix_leg(A_mul_Fs(P, outer_leg(P, px, o)), F.fb, fl, ok);
      }
      S.arel[o * nthr + tid] = v - ((uint32_t)S.minA[o] << F.fb) + F.delta;
    }
    for (int o = tid; o < n_out; o += nthr) S.ahi[o] = (uint32_t)((int64_t)o * n_in * P.K + S.minA[o]);
    __syncthreads();
    if (in_bounds)
      tile_loop<YT, WEIGHTED, false, JC>(P, px, S, F, tid, nthr, n_out, n_in, i_lo, i_hi, acc_s, acc_c, oob);
    else
      tile_loop<YT, WEIGHTED, true, JC>(P, px, S, F, tid, nthr, n_out, n_in, i_lo, i_hi, acc_s, acc_c, oob);
  }
  if (active) P.Im[no] = P.accumulate ? P.Im[no] + (acc_s + acc_c) : acc_s + acc_c;
  add_count(P.oob, active ? oob : 0u);
}

template <class YT, bool WEIGHTED, int JC>
__global__ void __launch_bounds__(256) das_fast_kernel(const FastParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  fast_tile<YT, WEIGHTED, JC>(P, blockIdx.x, (int64_t)blockIdx.y + P.slow_tile0, smem_raw);
}

// Persistent batch kernel: CTAs take (frame, tile) work items from a queue
// (items sorted by decreasing cost on the host) until it is empty. The frame
// descriptor is staged in shared memory; every frame's tile has blockDim.x
// points. ctr must be zero at launch (the batch run resets it).
template <class YT>
__global__ void __launch_bounds__(128) das_batch_kernel(const FastParams *__restrict__ frames,
                                                        const int4 *__restrict__ items, int n_items,
                                                        int *__restrict__ ctr) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ FastParams sP;
  __shared__ int s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(ctr, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= n_items) break;
    const int4 w = items[it];
    if (threadIdx.x == 0) sP = frames[w.x];
    __syncthreads();
    if (sP.jc == 8) fast_tile<YT, false, 8>(sP, w.y, w.z, smem_raw);
    else fast_tile<YT, false, 16>(sP, w.y, w.z, smem_raw);
    __syncthreads();
  }
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
      const int64_t gi = (int64_t)n * P.K + trunc_index(p);
      float y = gather_ok<float>(gi, y_count(P), P.bad) ? load_sample(Y + gi) : 0.0f;
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
  auto kern = (P.jc == 8) ? das_fast_kernel<YT, W, 8> : das_fast_kernel<YT, W, 16>;
  cudaError_t e = ensure_smem(kern, smem);
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

// Stream operations only (memset + launch), so a batch run can be captured
// in a CUDA graph; the kernel attribute is set once by batch_prepare.
cudaError_t launch_batch(const FastParams *frames, const int4 *items, int n_items, int *ctr, size_t smem, bool bf16,
                         int grid, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(ctr, 0, sizeof(int), st);
  if (e != cudaSuccess || n_items == 0) return e;
  if (bf16) das_batch_kernel<__nv_bfloat16><<<grid, 128, smem, st>>>(frames, items, n_items, ctr);
  else das_batch_kernel<float><<<grid, 128, smem, st>>>(frames, items, n_items, ctr);
  return cudaGetLastError();
}

// Sets the dynamic shared-memory limit; returns resident CTAs per SM (0 on error).
int batch_prepare(size_t smem, bool bf16) {
  int n = 0;
  if (bf16) {
    if (cudaFuncSetAttribute(das_batch_kernel<__nv_bfloat16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
      return 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, das_batch_kernel<__nv_bfloat16>, 128, smem);
  } else {
    if (cudaFuncSetAttribute(das_batch_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, das_batch_kernel<float>, 128, smem);
  }
  return n;
}

__global__ void f32_to_bf16_2d_kernel(const float *__restrict__ x, __nv_bfloat16 *__restrict__ y, int64_t rows,
                                      int64_t row_elems, int64_t pitch) {
  const int64_t n = rows * row_elems;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = q / row_elems, e = q - r * row_elems;
    y[r * pitch + e] = __float2bfloat16_rn(x[r * pitch + e]);
  }
}

cudaError_t convert_f32_to_bf16_2d(const float *x, void *y, int64_t rows, int64_t row_elems, int64_t pitch,
                                   cudaStream_t st) {
  const int64_t n = rows * row_elems;
  if (n <= 0) return cudaSuccess;
  int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
  f32_to_bf16_2d_kernel<<<blocks, 256, 0, st>>>(x, reinterpret_cast<__nv_bfloat16 *>(y), rows, row_elems, pitch);
  return cudaGetLastError();
}

cudaError_t convert_f32_to_bf16(const float *x, void *y, int64_t n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
  f32_to_bf16_kernel<<<blocks, 256, 0, st>>>(x, reinterpret_cast<__nv_bfloat16 *>(y), n);
  return cudaGetLastError();
}


// ===========================================================================
// Geometry-bound operator: leg tables, weighted gather, adjoint scatter and
// weight gradient (the differentiable beamformer and its CG solver).
//
// Leg tables hold, per (element, image point), the scaled FP64 leg as 32.32
// fixed point with the A-scan column offset folded into the high word:
//   TA[o][n] = (o*n_in*K << 32) + round(A(n,o) * 2^32) + delta
//   TB[i][n] = (i*K << 32)      + round(B(n,i) * 2^32)
// so TA + TB has the sample's element offset in its high word and the
// fraction (shifted by delta) in its low word, exactly as in the tile kernel;
// the same ambiguity band sends the rare boundary terms to the FP64 path, so
// all three operators use the FP64 reference indices.
// ===========================================================================

namespace {

constexpr uint32_t TAB_DELTA = 1u << 10;       // 2^-22 in 2^-32 units
constexpr uint32_t TAB_AMB_LO = 2 * TAB_DELTA;  // ambiguity band of the table terms

__global__ void legtab_kernel(const FastParams P, int64_t *__restrict__ TA, int64_t *__restrict__ TB,
                              int *__restrict__ range) {
  const int n_out = (P.method == RCA_ROWTX) ? P.Nr : P.Nt;
  const int n_in = (P.method == RCA_ROWTX) ? P.Nt : P.Nr;
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int e = blockIdx.y;  // element: [0, n_out) outer, [n_out, n_out+n_in) inner
  const bool active = n < P.No;
  Pixel px;
  pixel_of(P, active ? n : 0, px);
  const bool outer = e < n_out;
  const double L = outer ? A_mul_Fs(P, outer_leg(P, px, e)) : A_mul_Fs(P, inner_leg(P, px, e - n_out));
  const bool ok = fabs(L) < 67108864.0;  // 2^26, as the tile kernel
  const double f = floor(ok ? L : 0.0);
  const int fl = (int)f;
  const uint64_t frac = (uint64_t)__double2ull_rn((ok ? (L - f) : 0.0) * 4294967296.0);  // [0, 2^32]
  const int64_t colk = outer ? (int64_t)e * n_in * P.K : (int64_t)(e - n_out) * P.K;
  const int64_t v = ((colk + fl) << 32) + (int64_t)frac + (outer ? TAB_DELTA : 0);
  if (active) {
    if (outer) TA[(int64_t)e * P.No + n] = v;
    else TB[(int64_t)(e - n_out) * P.No + n] = v;
  }
  // range[0..3]: min/max floor of outer legs, min/max of inner; [4]: overflow
  int mn = __reduce_min_sync(0xffffffffu, active ? fl : INT_MAX);
  int mx = __reduce_max_sync(0xffffffffu, active ? fl : INT_MIN);
  bool bad = __any_sync(0xffffffffu, active && !ok);
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&range[outer ? 0 : 2], mn);
    atomicMax(&range[outer ? 1 : 3], mx);
    if (bad) atomicOr(&range[4], 1);
  }
}

__global__ void legtab_classify_kernel(int *__restrict__ range, int64_t K, int64_t ny) {
  // range[5] = 1: every non-ambiguous floor index lies in [0, K);
  // range[6] = 1: element offsets fit 32 bits
  const int64_t lo = (int64_t)range[0] + range[2], hi = (int64_t)range[1] + range[3];
  range[5] = (range[4] == 0 && lo >= 0 && hi + 2 < K) ? 1 : 0;
  range[6] = (range[4] == 0 && ny + hi + 256 < (int64_t(1) << 32) && lo > -(int64_t(1) << 30)) ? 1 : 0;
}

// Weighted gather Im[n] = sum_c w[c] Y[k(n,c), c] from the leg tables.
template <class YT, bool WEIGHTED, bool CHECKED, int JC>
__device__ __forceinline__ void tab_gather_body(const FastParams &P, const Pixel &px, const int64_t *TA,
                                                const int64_t *TB, int64_t n, int n_out, int n_in,
                                                float &acc_s, float &acc_c, unsigned int &oob) {
  for (int i0 = 0; i0 < n_in; i0 += JC) {
    const int jn = min(JC, n_in - i0);
    uint64_t B64[JC];
#pragma unroll
    for (int j = 0; j < JC; j++) B64[j] = (j < jn) ? (uint64_t)__ldg(TB + (int64_t)(i0 + j) * P.No + n) : 0;
    for (int o = 0; o < n_out; o++) {
      const uint64_t A1[1] = {(uint64_t)__ldg(TA + (int64_t)o * P.No + n)};
      float part =
          (jn == JC) ? chunk_terms<YT, WEIGHTED, CHECKED, true, JC, 1>(P, px, B64, A1, o, i0, JC, n_in, TAB_AMB_LO, oob)
                     : chunk_terms<YT, WEIGHTED, CHECKED, false, JC, 1>(P, px, B64, A1, o, i0, jn, n_in, TAB_AMB_LO, oob);
      neumaier(acc_s, acc_c, part);
    }
  }
}

template <class YT, bool WEIGHTED>
__global__ void __launch_bounds__(256) tab_gather_kernel(const FastParams P, const int64_t *__restrict__ TA,
                                                         const int64_t *__restrict__ TB,
                                                         const int *__restrict__ range) {
  const int n_out = (P.method == RCA_ROWTX) ? P.Nr : P.Nt;
  const int n_in = (P.method == RCA_ROWTX) ? P.Nt : P.Nr;
  const int64_t n_raw = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = n_raw < P.No;
  const int64_t n = active ? n_raw : 0;
  Pixel px;
  pixel_of(P, n, px);
  float acc_s = 0.0f, acc_c = 0.0f;
  unsigned int oob = 0;
  const bool exact_all = range[6] == 0;
  if (exact_all) {
    for (int o = 0; o < n_out; o++) {
      for (int i0 = 0; i0 < n_in; i0 += 16)
        neumaier(acc_s, acc_c, exact_partial<YT, WEIGHTED>(P, px, o, i0, min(16, n_in - i0), n_in, oob));
    }
  } else if (range[5]) {
    tab_gather_body<YT, WEIGHTED, false, 16>(P, px, TA, TB, n, n_out, n_in, acc_s, acc_c, oob);
  } else {
    tab_gather_body<YT, WEIGHTED, true, 16>(P, px, TA, TB, n, n_out, n_in, acc_s, acc_c, oob);
  }
  if (active) P.Im[n] = acc_s + acc_c;
  add_count(P.oob, active ? oob : 0u);
}

// The term's sample index for the column-owner kernels: returns -1 when the
// term is out of bounds. Outside the ambiguity band the floor index decides
// (-1 is p in (-1, 0): sample 0); inside it the FP64 index is recomputed, the
// only place that needs the image point's coordinates.
__device__ __noinline__ int tab_index_exact(const FastParams &P, int64_t n, int o, int i) {
  Pixel px;
  pixel_of(P, n, px);
  int k;
  return exact_index(P, px, o, i, k) ? k : -1;
}

__device__ __forceinline__ int floor_index(uint64_t s, uint32_t colk, int64_t K) {
  const int32_t kk = (int32_t)((uint32_t)(s >> 32) - colk);
  return (kk >= 0 && kk < K) ? kk : (kk == -1 ? 0 : -1);
}

// Column-owner terms of one image point whose leg sums include an ambiguous
// one: every term goes through tab_index (floor outside the band, FP64
// inside). Kept out of line so that the common path holds its arrays in
// registers. The weight-gradient partials go to the shared accumulator wacc.
template <bool ADJ, bool WG>
__device__ __noinline__ void colowner_point_exact(const FastParams &P, const int64_t *__restrict__ TA,
                                                  const int64_t *__restrict__ TB, int64_t n, int o, int i0, int jn,
                                                  int n_in, float xn, float gn, float *hist, float *wacc) {
  const uint64_t A64 = (uint64_t)__ldg(TA + (int64_t)o * P.No + n);
  const float *Yf = reinterpret_cast<const float *>(P.Y);
  for (int j = 0; j < jn; j++) {
    const int64_t col = (int64_t)o * n_in + i0 + j;
    const uint64_t s = A64 + (uint64_t)__ldg(TB + (int64_t)(i0 + j) * P.No + n);
    const int k = ((uint32_t)s >= TAB_AMB_LO) ? floor_index(s, (uint32_t)(col * P.K), P.K) : tab_index_exact(P, n, o, i0 + j);
    if (k < 0) continue;
    if (ADJ) atomicAdd(hist + (int64_t)j * P.K + k, (P.w ? __ldg(P.w + col) : 1.0f) * xn);
    if (WG) atomicAdd(wacc + j, gn * __ldg(Yf + col * P.K + k));
  }
}

// Column-owner adjoint and weight gradient. A CTA owns outer element o and
// inner elements [i0, i0 + jn) (jn <= CW), loops over a share of the image
// points, PX points per thread per step, and
//   adjoint: Ya[k(n,c), c] += w[c] * X[n]   (shared-memory histogram per column)
//   wgrad:   dW[c] += G[n] * Y[k(n,c), c]  (per-thread partials, block reduction)
// The leg-table loads of the PX points are all issued before any index is
// formed; an image point with an ambiguous term is handed whole to
// colowner_point_exact.
template <bool ADJ, bool WG, int CW, int PX>
__global__ void __launch_bounds__(256, ADJ ? 4 : 3) tab_colowner_kernel(const FastParams P, const int64_t *__restrict__ TA,
                                                           const int64_t *__restrict__ TB,
                                                           const float *__restrict__ X, const float *__restrict__ G,
                                                           float *__restrict__ Ya, float *__restrict__ dW, int splits) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n_in = (P.method == RCA_ROWTX) ? P.Nt : P.Nr;
  const int jmax = min(CW, n_in);
  float *hist = reinterpret_cast<float *>(smem_raw);      // [jmax][K] (adjoint)
  float *red = hist + (ADJ ? (size_t)jmax * P.K : 0);     // [CW][warps] (wgrad)
  float *wacc = red + (WG ? CW * (blockDim.x >> 5) : 0);  // [CW] (wgrad, exact points)
  const int o = blockIdx.x;
  const int i0 = blockIdx.y * CW;
  const int jn = min(CW, n_in - i0);
  const int split = blockIdx.z;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int64_t K = P.K;
  const float *Yf = reinterpret_cast<const float *>(P.Y);
  if (ADJ) {
    for (int64_t q = tid; q < (int64_t)jn * K; q += nthr) hist[q] = 0.0f;
  }
  if (WG && tid < CW) wacc[tid] = 0.0f;
  __syncthreads();
  float wc[CW];
  uint32_t colk[CW];
  float wsum[CW];
#pragma unroll
  for (int j = 0; j < CW; j++) {
    const int64_t col = (int64_t)o * n_in + i0 + j;
    wc[j] = (ADJ && j < jn) ? (P.w ? __ldg(P.w + col) : 1.0f) : 0.0f;
    colk[j] = (uint32_t)(col * K);
    wsum[j] = 0.0f;
  }
  const int64_t per = (P.No + splits - 1) / splits;
  const int64_t n0 = (int64_t)split * per, n1 = min(P.No, n0 + per);
  const int64_t *ta = TA + (int64_t)o * P.No;
  const int64_t *tb = TB + (int64_t)i0 * P.No;
  for (int64_t nb = n0 + tid; nb < n1; nb += (int64_t)PX * nthr) {
    uint64_t s[PX][CW];
    float xn[PX], gn[PX];
    bool on[PX];
#pragma unroll
    for (int q = 0; q < PX; q++) {
      const int64_t n = nb + (int64_t)q * nthr;
      on[q] = n < n1;
      const int64_t nn = on[q] ? n : n0;
      const uint64_t A64 = (uint64_t)__ldg(ta + nn);
      xn[q] = ADJ ? __ldg(X + nn) : 0.0f;
      gn[q] = WG ? __ldg(G + nn) : 0.0f;
#pragma unroll
      for (int j = 0; j < CW; j++) s[q][j] = (j < jn) ? A64 + (uint64_t)__ldg(tb + (int64_t)j * P.No + nn) : ~0ull;
    }
#pragma unroll
    for (int q = 0; q < PX; q++) {
      if (!on[q]) continue;
      uint32_t minlo = 0xffffffffu;
#pragma unroll
      for (int j = 0; j < CW; j++) minlo = min(minlo, (uint32_t)s[q][j]);
      if (minlo >= TAB_AMB_LO) {
        int k[CW];
#pragma unroll
        for (int j = 0; j < CW; j++) k[j] = (j < jn) ? floor_index(s[q][j], colk[j], K) : -1;
        if (WG) {
          float yv[CW];
#pragma unroll
          for (int j = 0; j < CW; j++) yv[j] = (k[j] >= 0) ? __ldg(Yf + ((int64_t)o * n_in + i0 + j) * K + k[j]) : 0.0f;
#pragma unroll
          for (int j = 0; j < CW; j++) wsum[j] = fmaf(gn[q], yv[j], wsum[j]);
        }
        if (ADJ) {
          const float xq = xn[q];
#pragma unroll
          for (int j = 0; j < CW; j++)
            if (k[j] >= 0) atomicAdd(hist + j * K + k[j], wc[j] * xq);
        }
      } else {
        colowner_point_exact<ADJ, WG>(P, TA, TB, nb + (int64_t)q * nthr, o, i0, jn, n_in, xn[q], gn[q], hist, wacc);
      }
    }
  }
  __syncthreads();
  if (ADJ) {
    for (int j = 0; j < jn; j++) {
      float *dst = Ya + ((int64_t)o * n_in + i0 + j) * K;
      for (int64_t k = tid; k < K; k += nthr) {
        const float v = hist[(int64_t)j * K + k];
        if (splits == 1) dst[k] = v;
        else if (v != 0.0f) atomicAdd(dst + k, v);
      }
    }
  }
  if (WG) {
    const int lane = tid & 31, warp = tid >> 5, nw = nthr >> 5;
#pragma unroll
    for (int j = 0; j < CW; j++) {
      float v = wsum[j];
      for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
      if (lane == 0) red[j * nw + warp] = v;
    }
    __syncthreads();
    if (tid < jn) {
      float v = wacc[tid];
      for (int w = 0; w < nw; w++) v += red[tid * nw + w];
      atomicAdd(dW + (int64_t)o * n_in + i0 + tid, v);
    }
  }
}

}  // namespace

cudaError_t build_leg_tables(const FastParams &P, int64_t *TA, int64_t *TB, int *range, cudaStream_t st) {
  const int n_out = (P.method == RCA_ROWTX) ? P.Nr : P.Nt;
  const int n_in = (P.method == RCA_ROWTX) ? P.Nt : P.Nr;
  const int init[7] = {INT_MAX, INT_MIN, INT_MAX, INT_MIN, 0, 0, 0};
  cudaError_t e = cudaMemcpyAsync(range, init, sizeof(init), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  if (P.No > 0) {
    dim3 grid((unsigned)((P.No + 255) / 256), (unsigned)(n_out + n_in));
    legtab_kernel<<<grid, 256, 0, st>>>(P, TA, TB, range);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  legtab_classify_kernel<<<1, 1, 0, st>>>(range, P.K, (int64_t)n_out * n_in * P.K);
  return cudaGetLastError();
}

cudaError_t launch_tab_gather(const FastParams &P, const int64_t *TA, const int64_t *TB, const int *range,
                              cudaStream_t st) {
  if (P.No <= 0) return cudaSuccess;
  const unsigned g = (unsigned)((P.No + 255) / 256);
  if (P.w) tab_gather_kernel<float, true><<<g, 256, 0, st>>>(P, TA, TB, range);
  else tab_gather_kernel<float, false><<<g, 256, 0, st>>>(P, TA, TB, range);
  return cudaGetLastError();
}

// Columns per CTA of the column-owner kernels: a power of two, at most 16
// for the adjoint (histograms of width x K x 4 bytes within 50 KB, so four
// CTAs fit on an SM) and 4 for the weight gradient, no wider than the next
// power of two >= n_in. Narrow CTAs re-read the outer leg table more often
// but keep more warps resident, which is what these latency-bound loops need
// (CG configuration: scatter 0.19 ms at width 4 vs 0.26 ms at width 8).
int colowner_width(int64_t K, int n_in, bool adj) {
  int cw = adj ? 16 : 4;
  while (adj && cw > 1 && (size_t)cw * K * 4 > 50 * 1024) cw >>= 1;
  while (cw > 1 && cw / 2 >= n_in) cw >>= 1;
  return cw;
}

namespace {

template <bool ADJ, bool WG, int CW>
cudaError_t colowner_launch(const FastParams &P, const int64_t *TA, const int64_t *TB, const float *X, const float *G,
                            float *Ya, float *dW, dim3 grid, size_t smem, int splits, cudaStream_t st) {
  constexpr int PX = 1;  // two points per thread: more loads in flight but 104 registers, slower
  cudaError_t e = ensure_smem(tab_colowner_kernel<ADJ, WG, CW, PX>, smem);
  if (e != cudaSuccess) return e;
  tab_colowner_kernel<ADJ, WG, CW, PX><<<grid, 256, smem, st>>>(P, TA, TB, X, G, Ya, dW, splits);
  return cudaGetLastError();
}

template <bool ADJ, bool WG>
cudaError_t colowner_dispatch(int cw, const FastParams &P, const int64_t *TA, const int64_t *TB, const float *X,
                              const float *G, float *Ya, float *dW, dim3 grid, size_t smem, int splits,
                              cudaStream_t st) {
  switch (cw) {
    case 16: return colowner_launch<ADJ, WG, 16>(P, TA, TB, X, G, Ya, dW, grid, smem, splits, st);
    case 8: return colowner_launch<ADJ, WG, 8>(P, TA, TB, X, G, Ya, dW, grid, smem, splits, st);
    case 4: return colowner_launch<ADJ, WG, 4>(P, TA, TB, X, G, Ya, dW, grid, smem, splits, st);
    case 2: return colowner_launch<ADJ, WG, 2>(P, TA, TB, X, G, Ya, dW, grid, smem, splits, st);
    default: return colowner_launch<ADJ, WG, 1>(P, TA, TB, X, G, Ya, dW, grid, smem, splits, st);
  }
}

}  // namespace

cudaError_t launch_tab_colowner(const FastParams &P, const int64_t *TA, const int64_t *TB, const float *X,
                                const float *G, float *Ya, float *dW, bool adj, bool wg, int sm_count,
                                cudaStream_t st) {
  const int n_out = (P.method == RCA_ROWTX) ? P.Nr : P.Nt;
  const int n_in = (P.method == RCA_ROWTX) ? P.Nt : P.Nr;
  if (n_out == 0 || n_in == 0) return cudaSuccess;
  const int cw = colowner_width(P.K, n_in, adj);
  const int jmax = std::min(cw, n_in);
  if (adj && (size_t)jmax * P.K * 4 > 200 * 1024) return cudaErrorInvalidValue;  // A-scans too long for the histogram
  const int groups = (n_in + cw - 1) / cw;
  const int64_t ctas = (int64_t)n_out * groups;
  int splits = (int)std::max<int64_t>(1, std::min<int64_t>(64, (4 * (int64_t)sm_count + ctas - 1) / ctas));
  if (P.No < 4096) splits = 1;
  const size_t smem = (adj ? (size_t)jmax * P.K * 4 : 0) + (wg ? (size_t)cw * 8 * 4 + cw * 4 : 0);
  dim3 grid((unsigned)n_out, (unsigned)groups, (unsigned)splits);
  if (adj && wg) return colowner_dispatch<true, true>(cw, P, TA, TB, X, G, Ya, dW, grid, smem, splits, st);
  if (adj) return colowner_dispatch<true, false>(cw, P, TA, TB, X, G, Ya, dW, grid, smem, splits, st);
  return colowner_dispatch<false, true>(cw, P, TA, TB, X, G, Ya, dW, grid, smem, splits, st);
}

}  // namespace dream
