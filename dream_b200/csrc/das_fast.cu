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

#include <algorithm>

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

// Layout of the tile's shared arrays (TileShared): per-element bases,
// extents and column words first, then (from a 16-byte boundary) the outer
// legs and the staged inner legs of every thread. The set-up's reduction
// scratch lives at the start of the outer-leg table until the legs are
// written. The total is a multiple of 16, so the scatter's windows that follow
// can be read as int4; for 128 outer and 128 inner elements on a 128-point
// tile it is 76288 bytes, three blocks per SM.
__host__ __device__ __forceinline__ size_t tile_head_bytes(int n_out, int n_in) {
  return ((size_t)(2 * (n_out + n_in) + n_out) * sizeof(int) + 15) & ~(size_t)15;
}
__host__ __device__ __forceinline__ size_t fast_smem_bytes_dev(const FastParams &P, int n_out, int n_in, int nthr) {
  const size_t legs = (size_t)(n_out + (P.jc == 8 ? 8 : 16)) * nthr * sizeof(uint32_t);
  return tile_head_bytes(n_out, n_in) + ((legs + 15) & ~(size_t)15);
}

// A-scan column of term (outer o, inner i): o * n_in + i for a full Y. A Y
// holding only the columns of inner elements [ycol_i0, ycol_i0 + ycol_o) (an
// inner-element shard) has ycol_o columns per outer element.
__device__ __forceinline__ int64_t ycol_outer(const FastParams &P, int n_in, int o) {
  return (int64_t)o * (P.ycol_o > 0 ? P.ycol_o : n_in);
}
__device__ __forceinline__ int64_t ycol_inner(const FastParams &P, int i) { return (int64_t)i - P.ycol_i0; }
__device__ __forceinline__ int64_t ycol(const FastParams &P, int n_in, int o, int i) {
  return ycol_outer(P, n_in, o) + ycol_inner(P, i);
}

// Coordinate differences between image point px and element e (outer or
// inner), as the reference forms them for each method: TFM uses the element's
// position; an RCA column (Gt) its x and z with the clamped y offset of the
// column stripe, an RCA row (Gr) its y and z with the clamped x offset.
__device__ __forceinline__ void leg_diffs(const FastParams &P, const Pixel &px, bool outer, int e, double &dx,
                                          double &dy, double &dz) {
  if (P.method == TFM) {
    const double *G = outer ? P.Gt : P.Gr;
    const int N = outer ? P.Nt : P.Nr;
    dx = __ldg(G + e) - px.xo;
    dy = __ldg(G + e + N) - px.yo;
    dz = __ldg(G + e + 2 * N) - px.zo;
  } else if ((P.method == RCA_COLTX) == outer) {  // a column
    dx = __ldg(P.Gt + e) - px.xo;
    dy = px.gy_c;
    dz = __ldg(P.Gt + e + 2 * P.Nt) - px.zo;
  } else {  // a row
    dx = px.gx_r;
    dy = __ldg(P.Gr + e + P.Nr) - px.yo;
    dz = __ldg(P.Gr + e + 2 * P.Nr) - px.zo;
  }
}

// Fixed-point leg: round(L * 2^fb) modulo 2^32, L = |d| * ocp * Fs + delay * Fs
// the leg in samples, from cfix = ocp * Fs * 2^fb and dfix = delay * Fs * 2^fb.
// This is not the reference's rounding chain: it only has to lie within
// 2^-(fb+1) + 2^-24 of the exact FP64 leg, which holds for |L| and
// |delay * Fs| below 2^23 (a few units of 2^-53 relative, plus the final
// rounding); the tile bound keeps every fast-path leg in that range. Adding
// 1.5 * 2^52 leaves the nearest integer in the low mantissa word.
__device__ __forceinline__ uint32_t leg_fix(double dx, double dy, double dz, double cfix, double dfix) {
  const double ss = fma(dz, dz, fma(dy, dy, dx * dx));
  const double t = fma(__dsqrt_rn(ss), cfix, dfix);
  return (uint32_t)__double2loint(__dadd_rn(t, 6755399441055744.0));
}

constexpr double LEG_LIMIT = 8388608.0;  // 2^23 samples: fixed-point legs and delays stay below it

// Range of |g - c| for c in [c0, c1].
__device__ __forceinline__ void offset_range(double g, double c0, double c1, double &lo, double &hi) {
  lo = g < c0 ? c0 - g : (g > c1 ? g - c1 : 0.0);
  hi = fmax(fabs(g - c0), fabs(g - c1));
}

// Range of |s(c)| for c in [c0, c1], s the reference's stripe offset: 0 on
// [e0, e1], e0 - c below, e1 - c above (extra_src/das.cc:470-480).
__device__ __forceinline__ void stripe_range(double e0, double e1, double c0, double c1, double &lo, double &hi) {
  auto s = [&](double c) { return (c >= e0 && c <= e1) ? 0.0 : (c < e0 ? e0 - c : e1 - c); };
  hi = fmax(fabs(s(c0)), fabs(s(c1)));
  lo = (e0 <= e1) ? fmax(0.0, fmax(e0 - c1, c0 - e1)) : 0.0;
}

// Bounding box of a tile's image points and delays: x, y, z, delay (ms).
struct TileBox {
  double lo[4], hi[4];
};

// Leg range [Lmin, Lmax] in samples of element e over the tile box.
__device__ __forceinline__ void leg_range(const FastParams &P, const TileBox &B, bool outer, int e, double &Lmin,
                                          double &Lmax) {
  double lx, hx, ly, hy, lz, hz;
  if (P.method == TFM) {
    const double *G = outer ? P.Gt : P.Gr;
    const int N = outer ? P.Nt : P.Nr;
    offset_range(G[e], B.lo[0], B.hi[0], lx, hx);
    offset_range(G[e + N], B.lo[1], B.hi[1], ly, hy);
    offset_range(G[e + 2 * N], B.lo[2], B.hi[2], lz, hz);
  } else if ((P.method == RCA_COLTX) == outer) {  // a column; stripe edges as pixel_of reads them
    offset_range(P.Gt[e], B.lo[0], B.hi[0], lx, hx);
    stripe_range(P.Gr[0 + P.Nt], P.Gr[P.Nt - 1 + P.Nt], B.lo[1], B.hi[1], ly, hy);
    offset_range(P.Gt[e + 2 * P.Nt], B.lo[2], B.hi[2], lz, hz);
  } else {  // a row
    stripe_range(P.Gt[0], P.Gt[P.Nr - 1], B.lo[0], B.hi[0], lx, hx);
    offset_range(P.Gr[e + P.Nr], B.lo[1], B.hi[1], ly, hy);
    offset_range(P.Gr[e + 2 * P.Nr], B.lo[2], B.hi[2], lz, hz);
  }
  const bool dl = (P.method == RCA_ROWTX) ? !outer : outer;  // the leg that carries the delay
  Lmin = (sqrt(lx * lx + ly * ly + lz * lz) * P.ocp + (dl ? B.lo[3] : 0.0)) * P.Fs;
  Lmax = (sqrt(hx * hx + hy * hy + hz * hz) * P.ocp + (dl ? B.hi[3] : 0.0)) * P.Fs;
}

struct TileShared {
  double *red;     // [warps][8]: box reduction (set-up only; shares arel's space)
  int *stat;       // [warps][8]: classification reduction (set-up only; shares arel's space)
  int *base;       // [n_out + n_in]: integer base of each leg over the tile (outer first)
  int *ext;        // [n_out + n_in]: bound of (floor(leg) - base)
  uint32_t *ahi;   // [n_out]: high word of the outer legs (column offset + base)
  uint32_t *arel;  // [n_out][nthreads]: outer legs, fixed point relative to base, + delta
  uint32_t *brel;  // [JC][nthreads]: the current chunk's inner legs, relative to base
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
    const int64_t col = ycol(P, n_in, o, i0 + j);
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
// fraction word; a chunk whose minimum falls in the band is recomputed. The
// minimum runs as four interleaved chains, two terms per step (one
// three-input minimum), and the packed sums as a tree, so no long dependency
// chain holds the warp; one branch tests all NO outer elements.
template <class YT, bool WEIGHTED, bool CHECKED, bool FULL, int JC, int NO>
__device__ __forceinline__ float chunk_terms(const FastParams &P, const Pixel &px, const uint64_t (&B64)[JC],
                                             const uint64_t (&A64)[NO], int o0, int i0, int jn, int n_in,
                                             uint32_t amb_lo, unsigned int &oob) {
  // NO outer elements x JC inner elements: all NO*JC gathers are issued before
  // any (rare) call to the exact path, so they are in flight together.
  const YT *__restrict__ Y = reinterpret_cast<const YT *>(P.Y);
  const int64_t K = P.K;
  constexpr int NM = JC < 4 ? JC : 4;  // independent minimum chains per outer element
  float y[NO][JC];
  uint32_t mlo[NO][NM];
  unsigned int oob_chunk[NO];
#pragma unroll
  for (int q = 0; q < NO; q++) {
    oob_chunk[q] = 0;
#pragma unroll
    for (int c = 0; c < NM; c++) mlo[q][c] = 0xffffffffu;
#pragma unroll
    for (int j = 0; j < JC; j++) {
      y[q][j] = 0.0f;
      if (FULL || j < jn) {
        const uint64_t s = A64[q] + B64[j];
        if (FULL && (j & 1)) {  // pairs: one three-input minimum per two terms
          const uint32_t prev = (uint32_t)(A64[q] + B64[j - 1]);
          mlo[q][(j >> 1) % NM] = min(mlo[q][(j >> 1) % NM], min(prev, (uint32_t)s));
        } else if (!FULL) {
          mlo[q][j % NM] = min(mlo[q][j % NM], (uint32_t)s);
        }
        const uint32_t off = (uint32_t)(s >> 32);
        if (CHECKED) {
          // Outside the ambiguity band the floor index is exact: [0, K) is in
          // bounds, -1 means p in (-1, 0), i.e. sample 0 after truncation, and
          // anything else is out of bounds.
          const int64_t col0 = ycol(P, n_in, o0 + q, i0 + j) * K;
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
  uint32_t minlo[NO];
#pragma unroll
  for (int q = 0; q < NO; q++) {
    minlo[q] = mlo[q][0];
#pragma unroll
    for (int c = 1; c < NM; c++) minlo[q] = min(minlo[q], mlo[q][c]);
    float part = 0.0f;
    if (WEIGHTED) {
      const float *w = P.w + ycol(P, n_in, o0 + q, i0);
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
      // packed FP32x2 adds: half the instructions; summed as a tree
      uint64_t v[JC / 2];
#pragma unroll
      for (int j = 0; j < JC / 2; j++) v[j] = pack_f32x2(y[q][2 * j], y[q][2 * j + 1]);
#pragma unroll
      for (int w = JC / 4; w >= 1; w /= 2)
#pragma unroll
        for (int j = 0; j < w; j++) v[j] = add_f32x2(v[j], v[j + w]);
      part = lo_f32(v[0]) + hi_f32(v[0]);
    }
    partq[q] = part;
  }
  uint32_t mm = minlo[0];
#pragma unroll
  for (int q = 1; q < NO; q++) mm = min(mm, minlo[q]);
  if (mm < amb_lo) {
#pragma unroll
    for (int q = 0; q < NO; q++) {
      if (minlo[q] < amb_lo) {
        // this outer element's partial is replaced by the exact one (which counts its own OOB)
        partq[q] = exact_partial<YT, WEIGHTED>(P, px, o0 + q, i0, jn, n_in, oob);
      } else {
        oob += oob_chunk[q];
      }
    }
  } else {
#pragma unroll
    for (int q = 0; q < NO; q++) oob += oob_chunk[q];
  }
#pragma unroll
  for (int q = 0; q < NO; q++) total += partq[q];
  return total;
}

template <class YT, bool WEIGHTED, bool CHECKED, int JC>
__device__ __forceinline__ void tile_loop(const FastParams &P, const Pixel &px, const TileShared &S, const FixFmt F,
                                          double cfix, double dfixB, int tid, int nthr, int n_out, int n_in,
                                          int i_lo, int i_hi, float &acc_s, float &acc_c, unsigned int &oob) {
  const int64_t K = P.K;
  for (int i0 = i_lo; i0 < i_hi; i0 += JC) {
    const int jn = min(JC, i_hi - i0);
    // the chunk's inner legs into this thread's shared slots, four at a time
    // (all of them side by side in registers would crowd the gather loop)
    bool bad = false;
#pragma unroll 4
    for (int j = 0; j < jn; j++) {
      const int i = i0 + j;
      double dx, dy, dz;
      leg_diffs(P, px, false, i, dx, dy, dz);
      const uint32_t r = leg_fix(dx, dy, dz, cfix, dfixB) - ((uint32_t)S.base[n_out + i] << F.fb);
      bad |= r >= ((uint32_t)(S.ext[n_out + i] + 1) << F.fb);
      S.brel[j * nthr + tid] = r;
    }
    uint64_t B64[JC];
#pragma unroll
    for (int j = 0; j < JC; j++) {
      B64[j] = 0;
      if (j < jn) {
        const int i = i0 + j;
        const uint32_t hi = (uint32_t)(ycol_inner(P, i) * K + S.base[n_out + i]);
        B64[j] = ((uint64_t)S.brel[j * nthr + tid] << F.lo_shift) + ((uint64_t)hi << 32);
      }
    }
    if (__any_sync(0xffffffffu, bad)) {
      // an inner leg outside the tile's bound: this chunk through the exact path
      for (int o = 0; o < n_out; o++)
        neumaier(acc_s, acc_c, exact_partial<YT, WEIGHTED>(P, px, o, i0, jn, n_in, oob));
      continue;
    }
    if (jn == JC) {
      // compensation every four outer elements
      int o = 0;
      for (; o + 4 <= n_out; o += 4) {
        const uint64_t A2[2] = {((uint64_t)S.arel[o * nthr + tid] << F.lo_shift) + ((uint64_t)S.ahi[o] << 32),
                                ((uint64_t)S.arel[(o + 1) * nthr + tid] << F.lo_shift) + ((uint64_t)S.ahi[o + 1] << 32)};
        const float p0 = chunk_terms<YT, WEIGHTED, CHECKED, true, JC, 2>(P, px, B64, A2, o, i0, JC, n_in, F.amb_lo, oob);
        const uint64_t A3[2] = {((uint64_t)S.arel[(o + 2) * nthr + tid] << F.lo_shift) + ((uint64_t)S.ahi[o + 2] << 32),
                                ((uint64_t)S.arel[(o + 3) * nthr + tid] << F.lo_shift) + ((uint64_t)S.ahi[o + 3] << 32)};
        const float p1 = chunk_terms<YT, WEIGHTED, CHECKED, true, JC, 2>(P, px, B64, A3, o + 2, i0, JC, n_in, F.amb_lo, oob);
        neumaier(acc_s, acc_c, p0 + p1);
      }
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

// Everything a tile needs before its terms: the image point of each thread,
// the leg bounds and fixed-point format of the tile, and (unless the tile
// takes the exact path) the outer legs in shared memory.
struct TileCtx {
  Pixel px;
  int64_t no;
  bool active, exact_tile, in_bounds;
  bool vec_safe;  // in bounds, and every scatter window row ends inside its A-scan
  int tid, nthr, n_out, n_in, i_lo, i_hi;
  FixFmt F;
  double cfix, dfixB;
  int ext_outer, ext_inner;  // largest (top - base) of the outer and of the inner legs
  TileShared S;
};

__device__ __forceinline__ void tile_setup(const FastParams &P, int64_t tfi, int64_t tsi, unsigned char *smem_raw,
                                           TileCtx &T) {
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarps = nthr >> 5;
  const int n_out = (P.method == RCA_ROWTX) ? P.Nr : P.Nt;
  const int n_in = (P.method == RCA_ROWTX) ? P.Nt : P.Nr;
  // inner elements of this launch: all of them unless the caller sets a range
  const int i_lo = P.in_lo, i_hi = P.in_hi > 0 ? P.in_hi : n_in;

  TileShared S;
  S.base = reinterpret_cast<int *>(smem_raw);
  S.ext = S.base + n_out + n_in;
  S.ahi = reinterpret_cast<uint32_t *>(S.ext + n_out + n_in);
  S.arel = reinterpret_cast<uint32_t *>(smem_raw + tile_head_bytes(n_out, n_in));
  S.brel = S.arel + n_out * nthr;
  // n_out * nthr words hold the nwarps * 8 doubles and ints of the set-up
  S.red = reinterpret_cast<double *>(S.arel);
  S.stat = reinterpret_cast<int *>(S.red + nwarps * 8);

  // ---- image point of this thread (inactive lanes repeat the tile's first point) ----
  const int lf = lane % P.wf, ls = lane / P.wf;
  const int warps_f = P.tile_f / P.wf;
  const int wfi = warp % warps_f, wsi = warp / warps_f;
  const int64_t f = tfi * P.tile_f + wfi * P.wf + lf;
  const int64_t s = tsi * P.tile_s + wsi * (32 / P.wf) + ls;
  const bool active = f < P.n_fast && s < P.n_slow;
  const int64_t no = active ? s * P.n_fast + f : tsi * P.tile_s * P.n_fast + tfi * P.tile_f;

  Pixel px;
  pixel_of(P, no, px);

  // ---- 1. tile box, leg bounds, classification ----
  {
    double mn[4] = {px.xo, px.yo, px.zo, px.delay_ms}, mx[4] = {px.xo, px.yo, px.zo, px.delay_ms};
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
      for (int q = 0; q < 4; q++) {
        mn[q] = fmin(mn[q], __shfl_xor_sync(0xffffffffu, mn[q], off));
        mx[q] = fmax(mx[q], __shfl_xor_sync(0xffffffffu, mx[q], off));
      }
    if (lane == 0)
#pragma unroll
      for (int q = 0; q < 4; q++) {
        S.red[warp * 8 + q] = mn[q];
        S.red[warp * 8 + 4 + q] = mx[q];
      }
  }
  __syncthreads();
  TileBox box;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    box.lo[q] = S.red[q];
    box.hi[q] = S.red[4 + q];
  }
  for (int w = 1; w < nwarps; w++)
#pragma unroll
    for (int q = 0; q < 4; q++) {
      box.lo[q] = fmin(box.lo[q], S.red[w * 8 + q]);
      box.hi[q] = fmax(box.hi[q], S.red[w * 8 + 4 + q]);
    }
  // delays beyond the fixed-point range send the tile to the exact path
  int bad = !(fabs(box.lo[3] * P.Fs) < LEG_LIMIT && fabs(box.hi[3] * P.Fs) < LEG_LIMIT);
  int ext_max = 0, extA = 0, loA = INT_MAX, hiA = INT_MIN, loB = INT_MAX, hiB = INT_MIN;
  for (int e = tid; e < n_out + n_in; e += nthr) {
    const bool outer = e < n_out;
    const int el = outer ? e : e - n_out;
    if (!outer && (el < i_lo || el >= i_hi)) {
      S.base[e] = 0;
      S.ext[e] = 0;
      continue;
    }
    double Lmin, Lmax;
    leg_range(P, box, outer, el, Lmin, Lmax);
    int b = 0, t = 0;
    if (Lmin > -LEG_LIMIT && Lmax < LEG_LIMIT && Lmin <= Lmax) {
      b = ((int)floor(Lmin) - 1) & ~3;  // a multiple of 4: the scatter's windows start 16-byte aligned
      t = (int)floor(Lmax) + 1;
    } else {
      bad = 1;
    }
    S.base[e] = b;
    S.ext[e] = t - b;
    ext_max = max(ext_max, t - b);
    if (outer) extA = max(extA, t - b);
    if (outer) {
      loA = min(loA, b);
      hiA = max(hiA, t);
    } else {
      loB = min(loB, b);
      hiB = max(hiB, t);
    }
  }
  bad = __reduce_or_sync(0xffffffffu, bad);
  ext_max = __reduce_max_sync(0xffffffffu, ext_max);
  loA = __reduce_min_sync(0xffffffffu, loA);
  hiA = __reduce_max_sync(0xffffffffu, hiA);
  loB = __reduce_min_sync(0xffffffffu, loB);
  hiB = __reduce_max_sync(0xffffffffu, hiB);
  extA = __reduce_max_sync(0xffffffffu, extA);
  if (lane == 0) {
    S.stat[warp * 8 + 6] = extA;
    S.stat[warp * 8 + 0] = bad;
    S.stat[warp * 8 + 1] = ext_max;
    S.stat[warp * 8 + 2] = loA;
    S.stat[warp * 8 + 3] = hiA;
    S.stat[warp * 8 + 4] = loB;
    S.stat[warp * 8 + 5] = hiB;
  }
  __syncthreads();
  for (int w = 0; w < nwarps; w++) {
    bad |= S.stat[w * 8 + 0];
    ext_max = max(ext_max, S.stat[w * 8 + 1]);
    loA = min(loA, S.stat[w * 8 + 2]);
    hiA = max(hiA, S.stat[w * 8 + 3]);
    loB = min(loB, S.stat[w * 8 + 4]);
    hiB = max(hiB, S.stat[w * 8 + 5]);
    extA = max(extA, S.stat[w * 8 + 6]);
  }
  __syncthreads();  // the scratch is read: the outer legs below may overwrite it
  const int64_t stride = P.ycol_o > 0 ? P.ycol_o : n_in;
  bool exact_tile = bad || ext_max > WIDE_EXTENT || loA > hiA ||
                    (int64_t)n_out * stride * P.K + (int64_t)hiA + hiB + 8448 >= (int64_t(1) << 32) ||
                    (int64_t)loA + loB < -(int64_t(1) << 30);
  // a non-ambiguous term's floor index lies in [loA + loB, hiA + hiB + 2]
  const bool in_bounds = (int64_t)loA + loB >= 0 && (int64_t)hiA + hiB + 2 < P.K;

  const FixFmt F = ext_max > FINE_EXTENT ? FMT_WIDE : FMT_FINE;
  const double scale = (double)(1u << F.fb);
  const double cfix = P.ocp * P.Fs * scale;
  const double dfix = px.delay_ms * P.Fs * scale;
  if (!exact_tile) {
    // ---- 2. outer legs, relative to their bases, plus the delta shift ----
    int leg_bad = 0;
#pragma unroll 4
    for (int o = 0; o < n_out; o++) {
      double dx, dy, dz;
      leg_diffs(P, px, true, o, dx, dy, dz);
      const uint32_t r = leg_fix(dx, dy, dz, cfix, P.method == RCA_ROWTX ? 0.0 : dfix) - ((uint32_t)S.base[o] << F.fb);
      leg_bad |= r >= ((uint32_t)(S.ext[o] + 1) << F.fb);
      S.arel[o * nthr + tid] = r + F.delta;
    }
    for (int o = tid; o < n_out; o += nthr) S.ahi[o] = (uint32_t)(ycol_outer(P, n_in, o) * P.K + S.base[o]);
    exact_tile = __syncthreads_or(leg_bad) != 0;
  }
  T.px = px;
  T.no = no;
  T.active = active;
  T.exact_tile = exact_tile;
  T.in_bounds = in_bounds;
  // a window row ends by base_o + ext_o + base_i + ext_i + 7 <= hiA + hiB + 7
  T.vec_safe = in_bounds && (int64_t)hiA + hiB + 7 <= P.K;
  T.tid = tid;
  T.nthr = nthr;
  T.n_out = n_out;
  T.n_in = n_in;
  T.i_lo = i_lo;
  T.i_hi = i_hi;
  T.F = F;
  T.cfix = cfix;
  T.dfixB = P.method == RCA_ROWTX ? dfix : 0.0;
  T.ext_outer = extA;
  T.ext_inner = 0;
  for (int e = n_out + i_lo; e < n_out + i_hi; e++) T.ext_inner = max(T.ext_inner, S.ext[e]);
  T.S = S;
}

}  // namespace

// One tile of image points (tile indices tfi along the fast axis, tsi along
// the slow axis) with the frame described by P; smem_raw holds the tile's
// shared arrays (fast_smem_bytes). Called by the one-frame kernel and by the
// persistent batch kernel.
//
// 1. The box bounding the tile's points and delays gives every element's leg
//    range over the tile (leg_range): an integer base and extent per leg,
//    and the tile's fixed-point format.
// 2. Each point's outer legs are converted once (leg_fix) into shared memory,
//    relative to their bases; each inner leg is converted once per point in
//    the main loop. A leg outside its bound (which the box bound rules out up
//    to rounding) sends its tile (outer) or chunk (inner) to the exact path
//    before any gather depends on it.
template <class YT, bool WEIGHTED, int JC>
__device__ __forceinline__ void fast_tile(const FastParams &P, int64_t tfi, int64_t tsi, unsigned char *smem_raw) {
  TileCtx T;
  tile_setup(P, tfi, tsi, smem_raw, T);
  float acc_s = 0.0f, acc_c = 0.0f;
  unsigned int oob = 0;
  const YT *__restrict__ Yp = reinterpret_cast<const YT *>(P.Y);
  const Pixel px = T.px;  // a copy for the calls that take it by reference
  if (T.exact_tile) {
    // every term through the exact FP64 index
    for (int o = 0; o < T.n_out; o++) {
      float part = 0.0f;
      for (int i = T.i_lo; i < T.i_hi; i++) {
        int k;
        const int64_t col = ycol(P, T.n_in, o, i);
        if (exact_index(P, px, o, i, k)) {
          float y = load_sample(Yp + col * P.K + k);
          part = WEIGHTED ? fmaf(__ldg(P.w + col), y, part) : part + y;
        } else {
          oob++;
        }
      }
      neumaier(acc_s, acc_c, part);
    }
  } else if (T.in_bounds) {
    tile_loop<YT, WEIGHTED, false, JC>(P, px, T.S, T.F, T.cfix, T.dfixB, T.tid, T.nthr, T.n_out, T.n_in, T.i_lo,
                                       T.i_hi, acc_s, acc_c, oob);
  } else {
    tile_loop<YT, WEIGHTED, true, JC>(P, px, T.S, T.F, T.cfix, T.dfixB, T.tid, T.nthr, T.n_out, T.n_in, T.i_lo,
                                      T.i_hi, acc_s, acc_c, oob);
  }
  if (T.active) P.Im[T.no] = P.accumulate ? P.Im[T.no] + (acc_s + acc_c) : acc_s + acc_c;
  add_count(P.oob, T.active ? oob : 0u);
}

template <class YT, bool WEIGHTED, int JC>
__global__ void __launch_bounds__(256, 2) das_fast_kernel(const FastParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  fast_tile<YT, WEIGHTED, JC>(P, blockIdx.x, (int64_t)blockIdx.y + P.slow_tile0, smem_raw);
}

// Persistent batch kernel: CTAs take (frame, tile) work items from a queue
// (items sorted by decreasing cost on the host) until it is empty. The frame
// descriptor is staged in shared memory; every frame's tile has blockDim.x
// points. ctr must be zero at launch (the batch run resets it).
template <class YT>
__global__ void __launch_bounds__(128, 3) das_batch_kernel(const FastParams *__restrict__ frames,
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
  return fast_smem_bytes_dev(P, n_out, n_in, nthr);
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
// Adjoint (scatter) on pixel tiles: Ya[k(n,c), c] += w[c] * x[n] for the
// tile's image points n and every A-scan column c, at the forward's indices
// (fixed-point floors outside the ambiguity band, the FP64 chain inside it).
// Each term is added with a global reduction; the 32 lanes of a warp hit one
// column at nearby samples, so a warp's reductions fall on a few sectors.
// Ya must be zeroed (or hold the partial sum to add to) before the launch.
// ===========================================================================

namespace {

// Exact scatter of terms (o, i0 .. i0+jn-1) of one image point.
template <bool WEIGHTED>
__device__ __noinline__ void exact_scatter(const FastParams &P, const Pixel &px, int o, int i0, int jn, int n_in,
                                           float xn, float *Ya) {
  for (int j = 0; j < jn; j++) {
    int k;
    const int64_t col = ycol(P, n_in, o, i0 + j);
    if (exact_index(P, px, o, i0 + j, k)) atomicAdd(Ya + col * P.K + k, WEIGHTED ? __ldg(P.w + col) * xn : xn);
  }
}

template <bool WEIGHTED, bool CHECKED, int JC>
__device__ __forceinline__ void scatter_loop(const FastParams &P, const TileCtx &T, float xn, float *Ya) {
  const int64_t K = P.K;
  const TileShared &S = T.S;
  const FixFmt F = T.F;
  const int tid = T.tid, nthr = T.nthr, n_out = T.n_out, n_in = T.n_in;
  const Pixel px = T.px;  // a copy for the exact path (by reference), so T stays in registers
  for (int i0 = T.i_lo; i0 < T.i_hi; i0 += JC) {
    const int jn = min(JC, T.i_hi - i0);
    bool bad = false;
#pragma unroll 1
    for (int j = 0; j < jn; j++) {
      const int i = i0 + j;
      double dx, dy, dz;
      leg_diffs(P, px, false, i, dx, dy, dz);
      const uint32_t r = leg_fix(dx, dy, dz, T.cfix, T.dfixB) - ((uint32_t)S.base[n_out + i] << F.fb);
      bad |= r >= ((uint32_t)(S.ext[n_out + i] + 1) << F.fb);
      S.brel[j * nthr + tid] = r;
    }
    if (__any_sync(0xffffffffu, bad)) {
      if (T.active)
        for (int o = 0; o < n_out; o++) exact_scatter<WEIGHTED>(P, px, o, i0, jn, n_in, xn, Ya);
      continue;
    }
    uint64_t B64[JC];
#pragma unroll
    for (int j = 0; j < JC; j++) {
      B64[j] = 0;
      if (j < jn) {
        const uint32_t hi = (uint32_t)(ycol_inner(P, i0 + j) * K + S.base[n_out + i0 + j]);
        B64[j] = ((uint64_t)S.brel[j * nthr + tid] << F.lo_shift) + ((uint64_t)hi << 32);
      }
    }
    for (int o = 0; o < n_out; o++) {
      const uint64_t A64 = ((uint64_t)S.arel[o * nthr + tid] << F.lo_shift) + ((uint64_t)S.ahi[o] << 32);
      uint64_t sj[JC];
      uint32_t m = 0xffffffffu;
#pragma unroll
      for (int j = 0; j < JC; j++) {
        sj[j] = A64 + B64[j];
        if (j < jn) m = min(m, (uint32_t)sj[j]);
      }
      if (m < F.amb_lo) {  // an ambiguous term: this outer element's chunk through the exact indices
        if (T.active) exact_scatter<WEIGHTED>(P, px, o, i0, jn, n_in, xn, Ya);
        continue;
      }
      const int64_t colo = ycol_outer(P, n_in, o);
#pragma unroll
      for (int j = 0; j < JC; j++) {
        if (j < jn && T.active) {
          const float v = WEIGHTED ? __ldg(P.w + colo + ycol_inner(P, i0 + j)) * xn : xn;
          const uint32_t off = (uint32_t)(sj[j] >> 32);
          if (CHECKED) {
            const int64_t col0 = (colo + ycol_inner(P, i0 + j)) * K;
            const int32_t kk = (int32_t)(off - (uint32_t)col0);
            if (kk >= 0 && kk < K) atomicAdd(Ya + col0 + kk, v);
            else if (kk == -1) atomicAdd(Ya + col0, v);
          } else {
            atomicAdd(Ya + off, v);
          }
        }
      }
    }
  }
}


// Samples per shared-memory window row (windows wider than this send their
// tile to the direct-reduction path). Two buffers of JC rows alternate, so
// 256-point tiles of 64 outer elements keep two CTAs per SM.
constexpr int SCATTER_WCAP = 192;

__device__ __forceinline__ void red_add_v4(float *p, float4 v) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
               : "memory");
}

// Window scatter of one tile: for outer element o and a chunk of inner
// elements, every term goes into the shared-memory window of its column (the
// tile's sample range [base_o + base_i, ... + WS), 16-byte aligned because the
// bases are multiples of 4); then the windows are added to Ya with 4-wide
// vector reductions (the weight applied once per sample) and cleared; two
// buffers alternate, one block barrier per (o, chunk). A term's slot is the
// high word of A64 + B64 when both hold only the relative legs (the inner leg
// carrying its row). The windows hold fixed-point
// integers, x scaled by 2^(22 - E) with max |x| over the tile below 2^E, so
// the shared-memory additions are native integer atomics, exact and
// independent of their order (a slot receives at most one term per thread
// per batch, at most 256 terms of magnitude up to 2^22, and a batch taken
// back subtracts exactly what it added); each value is rounded once, to within
// 2^-22 of the tile's largest |x|.
template <bool WEIGHTED, bool CHECKED, int JC>
__device__ __forceinline__ void scatter_window_loop(const FastParams &P, const TileCtx &T, float xn_f, float *Ya,
                                                    float *winf, int WS) {
  int *win = reinterpret_cast<int *>(winf);
  const int64_t K = P.K;
  const TileShared &S = T.S;
  const FixFmt F = T.F;
  const int tid = T.tid, nthr = T.nthr, n_out = T.n_out, n_in = T.n_in;
  const bool active = T.active;
  const Pixel px = T.px;
  const bool vec = !CHECKED && ((K & 3) == 0) && ((reinterpret_cast<uintptr_t>(Ya) & 15) == 0);
  // fixed-point scale of the tile: max |x| < 2^E, values scaled by 2^(22 - E)
  float mx = fabsf(xn_f);
  for (int off = 16; off > 0; off >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
  __shared__ float s_mx[8];
  if ((tid & 31) == 0) s_mx[tid >> 5] = mx;
  for (int e = tid; e < 2 * JC * WS; e += nthr) win[e] = 0;
  __syncthreads();
  mx = 0.0f;
  for (int w = 0; w < (nthr >> 5); w++) mx = fmaxf(mx, s_mx[w]);
  if (mx == 0.0f) return;  // nothing to add
  int E;
  frexpf(mx, &E);
  const float qscale = ldexpf(1.0f, 22 - E), iS = ldexpf(1.0f, E - 22);
  const int xn = __float2int_rn(xn_f * qscale);
  // flush: a fixed group of nthr / JC threads per window row (one division
  // per tile, none per cell)
  const int tpr = nthr / JC;
  const int fr = tid / tpr, fq = tid - fr * tpr;
  // Two window buffers alternate per (outer element, chunk): the adds of one
  // batch and the flush of the previous one need only the barrier between a
  // batch's adds and its flush (a buffer is added to again only after the
  // next batch's barrier, which every thread reaches after its flush).
  int it = 0;
  for (int i0 = T.i_lo; i0 < T.i_hi; i0 += JC) {
    const int jn = min(JC, T.i_hi - i0);
    bool bad = false;
#pragma unroll 4
    for (int j = 0; j < jn; j++) {
      const int i = i0 + j;
      double dx, dy, dz;
      leg_diffs(P, px, false, i, dx, dy, dz);
      const uint32_t r = leg_fix(dx, dy, dz, T.cfix, T.dfixB) - ((uint32_t)S.base[n_out + i] << F.fb);
      bad |= r >= ((uint32_t)(S.ext[n_out + i] + 1) << F.fb);
      S.brel[j * nthr + tid] = r;
    }
    if (__syncthreads_or(bad)) {
      // an inner leg outside the tile's bound: this chunk through the exact indices, straight to Ya
      if (active)
        for (int o = 0; o < n_out; o++) exact_scatter<WEIGHTED>(P, px, o, i0, jn, n_in, xn_f, Ya);
      continue;
    }
    // the high word of B64[j] starts at row j of the window: the sum's high
    // word is the term's window cell
    uint64_t B64[JC];
#pragma unroll
    for (int j = 0; j < JC; j++)
      B64[j] = (j < jn) ? ((uint64_t)S.brel[j * nthr + tid] << F.lo_shift) + ((uint64_t)(j * WS) << 32) : 0;
    const bool full = jn == JC;
    // this thread's flush row fr: the inner element's part of its column, base and extent
    const bool my_row = fr < jn;
    const int64_t col_r = my_row ? ycol_inner(P, i0 + fr) : 0;
    const int64_t ostride = P.ycol_o > 0 ? P.ycol_o : n_in;  // columns per outer element
    float *ycl = Ya + col_r * K;  // this row's column for outer element o, stepped per o
    const int base_r = my_row ? S.base[n_out + i0 + fr] : 0, ext_r = my_row ? S.ext[n_out + i0 + fr] : 0;
    for (int o = 0; o < n_out; o++) {
      const uint64_t A64 = (uint64_t)S.arel[o * nthr + tid] << F.lo_shift;
      int *wb = win + (it & 1) * (JC * WS);  // this batch's buffer
      // Adds first, ambiguity test after: in the rare ambiguous batch the same
      // integer values are taken back out of the same cells (exact) and the
      // chunk goes through the exact indices, so no term's sum is kept.
      uint32_t mc[2] = {0xffffffffu, 0xffffffffu};  // two chains, two terms per step
      if (full) {
#pragma unroll
        for (int j = 0; j < JC; j += 2) {
          const uint64_t s0 = A64 + B64[j], s1 = A64 + B64[j + 1];
          atomicAdd(wb + (uint32_t)(s0 >> 32), xn);
          atomicAdd(wb + (uint32_t)(s1 >> 32), xn);
          mc[(j >> 1) & 1] = min(mc[(j >> 1) & 1], min((uint32_t)s0, (uint32_t)s1));
        }
      } else {
#pragma unroll
        for (int j = 0; j < JC; j++)
          if (j < jn) {
            const uint64_t s0 = A64 + B64[j];
            atomicAdd(wb + (uint32_t)(s0 >> 32), xn);
            mc[0] = min(mc[0], (uint32_t)s0);
          }
      }
      // Inactive lanes carry x = 0 and add nothing, so they need no test.
      if (min(mc[0], mc[1]) < F.amb_lo) {
        // an ambiguous term: take this outer element's adds back and use the exact indices
        for (int j = 0; j < jn; j++) atomicSub(wb + (uint32_t)((A64 + B64[j]) >> 32), xn);
        for (int j = 0; j < jn; j++) {
          int k;
          if (exact_index(P, px, o, i0 + j, k)) {
            const int slot = k - (S.base[o] + S.base[n_out + i0 + j]);
            const int wr = (S.ext[o] + S.ext[n_out + i0 + j] + 4 + 3) & ~3;  // the row's flushed width
            if (slot >= 0 && slot < wr) atomicAdd(wb + j * WS + slot, xn);
            else atomicAdd(Ya + ycol(P, n_in, o, i0 + j) * K + k, WEIGHTED ? __ldg(P.w + ycol(P, n_in, o, i0 + j)) * xn_f : xn_f);
          }
        }
      }
      __syncthreads();
      if (my_row) {
        // row fr of the window: sample kb + t of column col; the terms of
        // (o, i) lie in its first ext_o + ext_i + 3 cells
        const int64_t kb = (int64_t)S.base[o] + base_r;  // a multiple of 4
        const int wr = (S.ext[o] + ext_r + 4 + 3) & ~3;
        const float sc = WEIGHTED ? iS * __ldg(P.w + o * ostride + col_r) : iS;  // iS a power of two: one rounding either way
        int *wrow = wb + fr * WS;
        if (vec && T.vec_safe) {  // every vector of the row lies inside the A-scan
          for (int t = fq * 4; t < wr; t += tpr * 4) {
            int4 *wp = reinterpret_cast<int4 *>(wrow + t);
            const int4 vi = *wp;
            if (vi.x | vi.y | vi.z | vi.w) {
              *wp = make_int4(0, 0, 0, 0);
              red_add_v4(ycl + kb + t, make_float4((float)vi.x * sc, (float)vi.y * sc, (float)vi.z * sc, (float)vi.w * sc));
            }
          }
        } else if (vec) {
          for (int t = fq * 4; t < wr; t += tpr * 4) {
            int4 *wp = reinterpret_cast<int4 *>(wrow + t);
            const int4 vi = *wp;
            if (vi.x | vi.y | vi.z | vi.w) {
              *wp = make_int4(0, 0, 0, 0);
              const float4 v = make_float4((float)vi.x * sc, (float)vi.y * sc, (float)vi.z * sc, (float)vi.w * sc);
              const int64_t k0 = kb + t;
              if (k0 >= 0 && k0 + 4 <= K) {
                red_add_v4(ycl + k0, v);
              } else {  // a window edge beyond the A-scan holds only zeros; added one by one to stay inside
                const float vv[4] = {v.x, v.y, v.z, v.w};
                for (int q = 0; q < 4; q++)
                  if (vv[q] != 0.0f && k0 + q >= 0 && k0 + q < K) atomicAdd(ycl + k0 + q, vv[q]);
              }
            }
          }
        } else {
          for (int t = fq; t < wr; t += tpr) {
            const int vi = wrow[t];
            if (vi != 0) {
              wrow[t] = 0;
              int64_t k = kb + t;
              if (k == -1) k = 0;  // p in (-1, 0): sample 0 after truncation toward zero
              if (k >= 0 && k < K) atomicAdd(ycl + k, (float)vi * sc);
            }
          }
        }
      }
      ycl += ostride * K;
      it++;
    }
  }
}

template <bool WEIGHTED, int JC>
__global__ void __launch_bounds__(256, 2) das_scatter_kernel(const FastParams P, const float *__restrict__ X,
                                                             float *__restrict__ Ya) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TileCtx T;
  tile_setup(P, blockIdx.x, (int64_t)blockIdx.y + P.slow_tile0, smem_raw, T);
  const float xn = T.active ? __ldg(X + T.no) : 0.0f;
  const int WS = (T.ext_outer + T.ext_inner + 4 + 3) & ~3;  // window samples per column
  float *win = reinterpret_cast<float *>(smem_raw + fast_smem_bytes_dev(P, T.n_out, T.n_in, T.nthr));
  if (!T.exact_tile && WS <= SCATTER_WCAP) {
    if (T.in_bounds) scatter_window_loop<WEIGHTED, false, JC>(P, T, xn, Ya, win, WS);
    else scatter_window_loop<WEIGHTED, true, JC>(P, T, xn, Ya, win, WS);
  } else if (T.exact_tile) {
    const Pixel px = T.px;  // a copy: the exact path takes it by reference, T stays in registers
    if (T.active)
      for (int o = 0; o < T.n_out; o++)
        for (int i0 = T.i_lo; i0 < T.i_hi; i0 += 16)
          exact_scatter<WEIGHTED>(P, px, o, i0, min(16, T.i_hi - i0), T.n_in, xn, Ya);
  } else if (T.in_bounds) {
    scatter_loop<WEIGHTED, false, JC>(P, T, xn, Ya);
  } else {
    scatter_loop<WEIGHTED, true, JC>(P, T, xn, Ya);
  }
}

}  // namespace

// Tile scatter over the same tiles and slow-tile ranges as launch_fast (P as
// for the forward; P.w optional). Ya is not zeroed here.
cudaError_t launch_scatter(const FastParams &P, const float *X, float *Ya, cudaStream_t st) {
  const int nthr = P.tile_f * P.tile_s;
  // the tile's arrays, then two buffers of one (outer, inner chunk) batch's windows
  const size_t smem = fast_smem_bytes(P, nthr) + 2 * (size_t)(P.jc == 8 ? 8 : 16) * SCATTER_WCAP * sizeof(float);
  auto kern = P.w ? (P.jc == 8 ? das_scatter_kernel<true, 8> : das_scatter_kernel<true, 16>)
                  : (P.jc == 8 ? das_scatter_kernel<false, 8> : das_scatter_kernel<false, 16>);
  cudaError_t e = ensure_smem(kern, smem);
  if (e != cudaSuccess) return e;
  const int64_t gx = (P.n_fast + P.tile_f - 1) / P.tile_f;
  const int64_t gy = P.slow_tile1 - P.slow_tile0;
  if (gx <= 0 || gy <= 0) return cudaSuccess;
  kern<<<dim3((unsigned)gx, (unsigned)gy), nthr, smem, st>>>(P, X, Ya);
  return cudaGetLastError();
}

// Column pass after an unweighted scatter S = DAS^T g: dW[c] = sum_k Y[k, c] *
// S[k, c] (the weight gradient: each term g[n] * Y[k(n,c), c] regrouped by
// sample), and, when w is given, S[:, c] *= w[c] in place (the weighted
// adjoint). One CTA per column; columns are K apart in both arrays.
__global__ void __launch_bounds__(256) column_dot_scale_kernel(const float *__restrict__ Y, float *__restrict__ S,
                                                               const float *__restrict__ w, float *__restrict__ dW,
                                                               int64_t K) {
  const int64_t c = blockIdx.x;
  const float *y = Y ? Y + c * K : nullptr;
  float *sc = S + c * K;
  const float wc = w ? __ldg(w + c) : 1.0f;
  float acc = 0.0f;
  for (int64_t k = threadIdx.x; k < K; k += blockDim.x) {
    const float v = sc[k];
    if (y) acc = fmaf(__ldg(y + k), v, acc);
    if (w) sc[k] = v * wc;
  }
  if (dW == nullptr) return;
  __shared__ float red[8];
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) t += red[q];
    dW[c] = t;
  }
}

cudaError_t launch_column_dot_scale(const float *Y, float *S, const float *w, float *dW, int64_t K, int64_t ncol,
                                    cudaStream_t st) {
  if (ncol <= 0 || (K <= 0 && dW == nullptr)) return cudaSuccess;
  for (int64_t c0 = 0; c0 < ncol; c0 += 2147483647) {
    const int64_t n = std::min<int64_t>(ncol - c0, 2147483647);
    column_dot_scale_kernel<<<(unsigned)n, 256, 0, st>>>(Y ? Y + c0 * K : nullptr, S + c0 * K, w ? w + c0 : nullptr,
                                                         dW ? dW + c0 : nullptr, K);
  }
  return cudaGetLastError();
}

}  // namespace dream
