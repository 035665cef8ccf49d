/*
 * das_oracle.c -- CPU restatement of DREAM's delay-and-sum (DAS) beamformer.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker for the CUDA product path
 * in dream_b200/csrc: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it. Nothing in the product path links or calls it.
 *
 * Parity of this restatement is pinned against the reference itself: the
 * unmodified reference `das`/`das_f` modules (built by oracle/build_ref.sh)
 * are run on the same inputs by tests/golden/gen_golden.py, and the test suite
 * checks these functions reproduce the stored outputs bit for bit.
 *
 * Restated reference functions (reference paths, line numbers at the studied
 * revision):
 *   das (SAFT)        extra_src/das.cc:306-357  (das_saft_serial)
 *   das (TFM)         extra_src/das.cc:365-427  (das_tfm_serial)
 *   das (RCA col tx)  extra_src/das.cc:437-529  (das_rca_serial_coltx)
 *   das (RCA row tx)  extra_src/das.cc:533-626  (das_rca_serial_rowtx)
 *   pixel loop        extra_src/das.cc:103-191  (smp_das, delay selection :131-136)
 *   SAFT forcing      extra_src/das.cc:211-213  (Nr == 0 -> SAFT)
 *   error levels      src/dream_error.cc:40-76  (dream_out_of_bounds_err)
 *   das_uni           opencl/das_uni_double.cl:9-394, opencl/das_uni_float.cl
 *                     (the reference has no CPU das_uni; the OpenCL C source is
 *                     restated with IEEE sqrt in place of native_sqrt)
 *
 * Arithmetic rules reproduced exactly (compile with -ffp-contract=off and no
 * -march flags so no product or sum is fused):
 *   - time -> sample index is truncation toward zero of t_dp * Fs_khz;
 *   - association: SAFT 2*(|g-r|/cp + delay); TFM (t_t + delay) + t_r;
 *     RCA (t_col + delay) + t_row in both modes; das_uni row-tx
 *     t_col + (t_row + delay);
 *   - sum of squares ((dx*dx + dy*dy) + dz*dz);
 *   - in the FP32 `das`, Fs_khz, 1/cp and delay/1000 are evaluated in double
 *     and rounded to float (the literals are double, extra_src/das.cc:316-318);
 *     the FP32 das_uni evaluates them in float (opencl/das_uni_float.cl:47-49).
 *
 * All arrays are column-major: Ro[no + j*No], G[n + j*N], Y[k + col*K].
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

/* Mirrors SIRError (include/dream.h:42-47). */
enum { ORC_NONE = 0, ORC_IGNORE_OOB = 1, ORC_WARN_OOB = 2, ORC_OOB = 3 };
/* Mirrors ErrorLevel (include/dream.h:49-55). */
enum { ORC_LVL_NONE = 0, ORC_LVL_IGNORE = 1, ORC_LVL_WARN = 2, ORC_LVL_STOP = 3, ORC_LVL_PSTOP = 4 };
/* Mirrors DASType (include/dream.h:97-102). */
enum { ORC_SAFT = 0, ORC_TFM = 1, ORC_RCA_COLTX = 2, ORC_RCA_ROWTX = 3 };

/* dream_out_of_bounds_err (src/dream_error.cc:40-76) without the printing. */
static int oob_status(int err_level)
{
  switch (err_level) {
  case ORC_LVL_IGNORE: return ORC_IGNORE_OOB;
  case ORC_LVL_WARN: return ORC_WARN_OOB;
  case ORC_LVL_STOP:
  case ORC_LVL_PSTOP: return ORC_OOB;
  default: return ORC_NONE;
  }
}

/*
 * One generic body per precision. T is the arithmetic type; CONSTS computes
 * (Fs_khz, one_over_cp, delay_ms) the way the restated source does.
 *
 * The loop body of each method stays in the reference order (tx outer, rx
 * inner) so the per-pixel sum is accumulated in the same order.
 *
 * idx_out: optional int64 array of length No*Nt*Nr (SAFT: No*Nt) receiving the
 * selected sample index of every term (INT64_MIN marks an out-of-bounds term),
 * ordered [term][pixel] with term = t*Nr + r.
 */
#define ORACLE_BODY(SQRT)                                                              \
  int64_t no, nt_, nr_;                                                                   \
  int status = ORC_NONE;                                                                  \
  int64_t oob = 0;                                                                        \
  for (no = 0; no < No; no++) {                                                           \
    const T xo = Ro[no], yo = Ro[no + No], zo = Ro[no + 2 * No];                          \
    const T dlay = multi_delay ? delay[no] : delay[0];                                    \
    const T delay_ms = DELAY_MS(dlay);                                                    \
    T im = (T)0.0;                                                                        \
    const T *y_p = Y;                                                                     \
    if (method == ORC_SAFT) {                                                             \
      for (nt_ = 0; nt_ < Nt; nt_++) {                                                    \
        T gx = Gt[nt_] - xo, gy = Gt[nt_ + Nt] - yo, gz = Gt[nt_ + 2 * Nt] - zo;          \
        T t_tr = SQRT(gx * gx + gy * gy + gz * gz) * one_over_cp;                         \
        t_tr += delay_ms;                                                                 \
        T t_dp = (T)(2.0 * t_tr);                                                         \
        TERM(t_dp, nt_)                                                                   \
        y_p += K;                                                                         \
      }                                                                                   \
    } else if (method == ORC_TFM) {                                                       \
      for (nt_ = 0; nt_ < Nt; nt_++) {                                                    \
        T gx_t = Gt[nt_] - xo, gy_t = Gt[nt_ + Nt] - yo, gz_t = Gt[nt_ + 2 * Nt] - zo;    \
        T t_t = SQRT(gx_t * gx_t + gy_t * gy_t + gz_t * gz_t) * one_over_cp;              \
        t_t += delay_ms;                                                                  \
        for (nr_ = 0; nr_ < Nr; nr_++) {                                                  \
          T gx_r = Gr[nr_] - xo, gy_r = Gr[nr_ + Nr] - yo, gz_r = Gr[nr_ + 2 * Nr] - zo;  \
          T t_r = SQRT(gx_r * gx_r + gy_r * gy_r + gz_r * gz_r) * one_over_cp;            \
          T t_dp = t_t + t_r;                                                             \
          TERM(t_dp, nt_ * Nr + nr_)                                                      \
          y_p += K;                                                                       \
        }                                                                                 \
      }                                                                                   \
    } else {                                                                              \
      /* RCA: Gt = columns (Nt of them), Gr = rows (Nr). Stripe edges read   */           \
      /* literally as extra_src/das.cc:464-467 (num_cols/num_rows mixed).    */           \
      const T gc_y_min = Gr[0 + 1 * Nt];                                                  \
      const T gc_y_max = Gr[Nt - 1 + 1 * Nt];                                             \
      const T gr_x_min = Gt[0];                                                           \
      const T gr_x_max = Gt[Nr - 1];                                                      \
      T gy_c, gx_r;                                                                       \
      if (yo >= gc_y_min && yo <= gc_y_max) gy_c = (T)0.0;                                \
      else if (yo < gc_y_min) gy_c = gc_y_min - yo;                                       \
      else gy_c = gc_y_max - yo;                                                          \
      if (xo >= gr_x_min && xo <= gr_x_max) gx_r = (T)0.0;                                \
      else if (xo < gr_x_min) gx_r = gr_x_min - xo;                                       \
      else gx_r = gr_x_max - xo;                                                          \
      if (method == ORC_RCA_COLTX) {                                                      \
        for (nt_ = 0; nt_ < Nt; nt_++) {                                                  \
          T gx_c = Gt[nt_] - xo, gz_c = Gt[nt_ + 2 * Nt] - zo;                            \
          T t_c = SQRT(gx_c * gx_c + gy_c * gy_c + gz_c * gz_c) * one_over_cp;            \
          t_c += delay_ms;                                                                \
          for (nr_ = 0; nr_ < Nr; nr_++) {                                                \
            T gy_r = Gr[nr_ + Nr] - yo, gz_r = Gr[nr_ + 2 * Nr] - zo;                     \
            T t_r = SQRT(gx_r * gx_r + gy_r * gy_r + gz_r * gz_r) * one_over_cp;          \
            T t_dp = t_c + t_r;                                                           \
            TERM(t_dp, nt_ * Nr + nr_)                                                    \
            y_p += K;                                                                     \
          }                                                                               \
        }                                                                                 \
      } else {                                                                            \
        for (nr_ = 0; nr_ < Nr; nr_++) {                                                  \
          T gy_r = Gr[nr_ + Nr] - yo, gz_r = Gr[nr_ + 2 * Nr] - zo;                       \
          T t_r = SQRT(gx_r * gx_r + gy_r * gy_r + gz_r * gz_r) * one_over_cp;            \
          for (nt_ = 0; nt_ < Nt; nt_++) {                                                \
            T gx_c = Gt[nt_] - xo, gz_c = Gt[nt_ + 2 * Nt] - zo;                          \
            T t_c = SQRT(gx_c * gx_c + gy_c * gy_c + gz_c * gz_c) * one_over_cp;          \
            t_c += delay_ms;                                                              \
            T t_dp = t_c + t_r;                                                           \
            TERM(t_dp, nr_ * Nt + nt_)                                                    \
            y_p += K;                                                                     \
          }                                                                               \
        }                                                                                 \
      }                                                                                   \
    }                                                                                     \
    Im[no] = im;                                                                          \
  }                                                                                       \
  if (oob_count) *oob_count = oob;                                                        \
  return status;

/* One term: truncate toward zero, bounds check, gather (extra_src/das.cc:403-419). */
#define TERM(t_dp, term)                                                                  \
  {                                                                                       \
    T p_ = (t_dp) * Fs_khz;                                                               \
    int in_ = (K > 0) && (p_ > (T)-1.0) && (p_ < (T)K);                                   \
    int64_t k_ = in_ ? (int64_t)p_ : INT64_MIN;                                           \
    if (idx_out) idx_out[(int64_t)(term) * No + no] = k_;                                 \
    if (in_) {                                                                            \
      im += y_p[k_];                                                                      \
    } else {                                                                              \
      int s_ = oob_status(err_level);                                                     \
      if (s_ > status) status = s_;                                                       \
      oob++;                                                                              \
    }                                                                                     \
  }

/* For K >= 1 the bounds test (p > -1) && (p < K) equals (trunc(p) >= 0) &&
 * (trunc(p) < K) for integer K (K == 0 has no in-bounds sample), and leaves NaN out of bounds, which is where the reference's
 * integer conversion of NaN (INT64_MIN on x86-64) also lands. */

#define DELAY_MS(d) ((double)(d) / 1000.0)
int dream_oracle_das_f64(int method, const double *Y, int64_t K, const double *Ro, int64_t No,
                         const double *Gt, int64_t Nt, const double *Gr, int64_t Nr, double dt,
                         int multi_delay, const double *delay, double cp, int err_level,
                         double *Im, int64_t *oob_count, int64_t *idx_out)
{
  typedef double T;
  const double Fs_khz = (1.0 / dt) * 1000.0;
  const double one_over_cp = 1.0 / cp;
  if (Nr == 0) method = ORC_SAFT; /* extra_src/das.cc:211-213 */
  ORACLE_BODY(sqrt)
}
#undef DELAY_MS

/* DAS<float>: constants computed in double from the float arguments, then
 * rounded to float (extra_src/das.cc:316-318 with T = float). */
#define DELAY_MS(d) ((float)((double)(d) / 1000.0))
int dream_oracle_das_f32(int method, const float *Y, int64_t K, const float *Ro, int64_t No,
                         const float *Gt, int64_t Nt, const float *Gr, int64_t Nr, float dt,
                         int multi_delay, const float *delay, float cp, int err_level, float *Im,
                         int64_t *oob_count, int64_t *idx_out)
{
  typedef float T;
  const float Fs_khz = (float)((1.0 / (double)dt) * 1000.0);
  const float one_over_cp = (float)(1.0 / (double)cp);
  if (Nr == 0) method = ORC_SAFT;
  ORACLE_BODY(sqrtf)
}
#undef DELAY_MS
#undef TERM
#undef ORACLE_BODY

/* ------------------------------------------------------------------------- */
/* das_uni: uniform element and pixel grids (opencl/das_uni_double.cl).      */
/* ------------------------------------------------------------------------- */

/* Grid count as the kernels compute it: (int)((max - min)/d + 1.0)
 * (opencl/das_uni_double.cl:23-28); the division is in the kernel type and the
 * +1.0 literal is double in both kernels. */
int64_t dream_oracle_uni_count_f64(double mn, double d, double mx)
{
  return (int64_t)(int)((mx - mn) / d + 1.0);
}
int64_t dream_oracle_uni_count_f32(float mn, float d, float mx)
{
  return (int64_t)(int)((double)((mx - mn) / d) + 1.0);
}

/*
 * tri: 5 triplets (min, pitch, max) laid out as
 *   [t_min, t_pitch, t_max, r_min, r_pitch, r_max,
 *    x_min, dx, x_max, y_min, dy, y_max, z_min, dz, z_max].
 * Pixel linear index no -> (ny fastest, then nz, then nx)
 * (opencl/das_uni_double.cl:32-43). Elements lie on the x axis (y = z = 0).
 * RCA stripe edges are the triplet min/max (opencl/das_uni_double.cl:213-216).
 * Row-tx adds the delay to the row leg (opencl/das_uni_double.cl:358-360).
 */
#define UNI_BODY(SQRT, COUNT, FS, OCP, DMS)                                            \
  const T min_t = tri[0], pitch_t = tri[1], max_t = tri[2];                               \
  const T min_r = tri[3], pitch_r = tri[4], max_r = tri[5];                               \
  const T min_x = tri[6], dx = tri[7], max_x = tri[8];                                    \
  const T min_y = tri[9], dy = tri[10], max_y = tri[11];                                  \
  const T min_z = tri[12], dz = tri[13], max_z = tri[14];                                 \
  const int64_t Nt = COUNT(min_t, pitch_t, max_t);                                        \
  const int64_t Nr = (method == ORC_SAFT) ? 0 : COUNT(min_r, pitch_r, max_r);             \
  const int64_t Nx = COUNT(min_x, dx, max_x), Ny = COUNT(min_y, dy, max_y),               \
                Nz = COUNT(min_z, dz, max_z);                                             \
  const int64_t No = Nx * Ny * Nz;                                                        \
  const T Fs_khz = FS, one_over_cp = OCP, delay_ms = DMS;                                 \
  int status = ORC_NONE;                                                                  \
  int64_t oob = 0, no, nt_, nr_;                                                          \
  for (no = 0; no < No; no++) {                                                           \
    int64_t y_quot = no / Ny, ny = no - y_quot * Ny;                                      \
    int64_t z_quot = y_quot / Nz, nz = y_quot - z_quot * Nz;                              \
    int64_t x_quot = z_quot / Nx, nx = z_quot - x_quot * Nx;                              \
    const T xo = min_x + ((T)nx) * dx;                                                    \
    const T yo = min_y + ((T)ny) * dy;                                                    \
    const T zo = min_z + ((T)nz) * dz;                                                    \
    T im = (T)0.0;                                                                        \
    const T *y_p = Y;                                                                     \
    if (method == ORC_SAFT) {                                                             \
      for (nt_ = 0; nt_ < Nt; nt_++) {                                                    \
        T gx = (min_t + ((T)nt_) * pitch_t) - xo;                                         \
        T t_tr = SQRT(gx * gx + yo * yo + zo * zo) * one_over_cp;                         \
        t_tr += delay_ms;                                                                 \
        T t_dp = (T)(2.0 * t_tr);                                                         \
        UTERM(t_dp)                                                                       \
        y_p += K;                                                                         \
      }                                                                                   \
    } else if (method == ORC_TFM) {                                                       \
      for (nt_ = 0; nt_ < Nt; nt_++) {                                                    \
        T gx_t = (min_t + ((T)nt_) * pitch_t) - xo;                                       \
        T t_t = SQRT(gx_t * gx_t + yo * yo + zo * zo) * one_over_cp;                      \
        t_t += delay_ms;                                                                  \
        for (nr_ = 0; nr_ < Nr; nr_++) {                                                  \
          T gx_r = (min_r + ((T)nr_) * pitch_r) - xo;                                     \
          T t_r = SQRT(gx_r * gx_r + yo * yo + zo * zo) * one_over_cp;                    \
          T t_dp = t_t + t_r;                                                             \
          UTERM(t_dp)                                                                     \
          y_p += K;                                                                       \
        }                                                                                 \
      }                                                                                   \
    } else {                                                                              \
      /* Columns use the transmit triplet, rows the receive triplet. */                   \
      const T gt_y_min = min_r, gt_y_max = max_r, gr_x_min = min_t, gr_x_max = max_t;     \
      T gy_c, gx_r = (T)0.0;                                                              \
      if (yo >= gt_y_min && yo <= gt_y_max) gy_c = (T)0.0;                                \
      else if (yo < gt_y_min) gy_c = gt_y_min - yo;                                       \
      else gy_c = gt_y_max - yo;                                                          \
      if (xo < gr_x_min || xo > gr_x_max) {                                               \
        if (xo < gr_x_min) gx_r = gr_x_min - xo;                                          \
        else gx_r = gr_x_max - xo;                                                        \
      }                                                                                   \
      if (method == ORC_RCA_COLTX) {                                                      \
        for (nt_ = 0; nt_ < Nt; nt_++) {                                                  \
          T gx_c = (min_t + ((T)nt_) * pitch_t) - xo;                                     \
          T t_c = SQRT(gx_c * gx_c + gy_c * gy_c + zo * zo) * one_over_cp;                \
          t_c += delay_ms;                                                                \
          for (nr_ = 0; nr_ < Nr; nr_++) {                                                \
            T gy_r = (min_r + ((T)nr_) * pitch_r) - yo;                                   \
            T t_r = SQRT(gx_r * gx_r + gy_r * gy_r + zo * zo) * one_over_cp;              \
            T t_dp = t_c + t_r;                                                           \
            UTERM(t_dp)                                                                   \
            y_p += K;                                                                     \
          }                                                                               \
        }                                                                                 \
      } else {                                                                            \
        for (nr_ = 0; nr_ < Nr; nr_++) {                                                  \
          T gy_r = (min_r + ((T)nr_) * pitch_r) - yo;                                     \
          T t_r = SQRT(gx_r * gx_r + gy_r * gy_r + zo * zo) * one_over_cp;                \
          t_r += delay_ms;                                                                \
          for (nt_ = 0; nt_ < Nt; nt_++) {                                                \
            T gx_c = (min_t + ((T)nt_) * pitch_t) - xo;                                   \
            T t_c = SQRT(gx_c * gx_c + gy_c * gy_c + zo * zo) * one_over_cp;              \
            T t_dp = t_c + t_r;                                                           \
            UTERM(t_dp)                                                                   \
            y_p += K;                                                                     \
          }                                                                               \
        }                                                                                 \
      }                                                                                   \
    }                                                                                     \
    Im[no] = im;                                                                          \
  }                                                                                       \
  if (oob_count) *oob_count = oob;                                                        \
  return status;

/* The OpenCL kernels skip out-of-bounds terms silently; the restatement also
 * reports them with the requested error level so the CUDA das_uni can be
 * checked on the same status semantics as das. */
#define UTERM(t_dp)                                                                       \
  {                                                                                       \
    T p_ = (t_dp) * Fs_khz;                                                               \
    if ((K > 0) && (p_ > (T)-1.0) && (p_ < (T)K)) {                                       \
      im += y_p[(int64_t)p_];                                                             \
    } else {                                                                              \
      int s_ = oob_status(err_level);                                                     \
      if (s_ > status) status = s_;                                                       \
      oob++;                                                                              \
    }                                                                                     \
  }

int dream_oracle_das_uni_f64(int method, const double *Y, int64_t K, const double *tri, double dt,
                             double delay, double cp, int err_level, double *Im,
                             int64_t *oob_count)
{
  typedef double T;
  UNI_BODY(sqrt, dream_oracle_uni_count_f64, (1.0 / dt) * 1000.0, 1.0 / cp,
           delay / 1000.0)
}

/* opencl/das_uni_float.cl:47-49: float division for the constants. */
int dream_oracle_das_uni_f32(int method, const float *Y, int64_t K, const float *tri, float dt,
                             float delay, float cp, int err_level, float *Im, int64_t *oob_count)
{
  typedef float T;
  UNI_BODY(sqrtf, dream_oracle_uni_count_f32, (1.0f / dt) * 1000.0f, 1.0f / cp,
           delay / 1000.0f)
}
#undef UTERM
#undef UNI_BODY

/* ------------------------------------------------------------------------- */
/* Weighted DAS and its adjoint on the FP64 index set.                        */
/* ------------------------------------------------------------------------- */
/*
 * The differentiable operator is Im[o] = sum_c w[c] * Y[k(o,c), c] over the
 * terms c = t*Nr + r (rows*Nt + cols for RCA row-tx), with k(o,c) the FP64
 * reference index (an out-of-bounds term contributes nothing). Its adjoint
 * scatters an image x back: Ya[k(o,c), c] += w[c] * x[o]. The weight gradient
 * is dw[c] = sum_o g[o] * Y[k(o,c), c]. These follow from the FP64 index set
 * the restated das produces (idx_out above), so they are written against an
 * explicit index table.
 */
void dream_oracle_das_weighted_f64(const int64_t *idx, int64_t No, int64_t C, int64_t K,
                                   const double *Y, const double *w, double *Im)
{
  int64_t o, c;
  for (o = 0; o < No; o++) {
    double s = 0.0;
    for (c = 0; c < C; c++) {
      int64_t k = idx[c * No + o];
      if (k != INT64_MIN) s += w[c] * Y[k + c * K];
    }
    Im[o] = s;
  }
}

void dream_oracle_das_adjoint_f64(const int64_t *idx, int64_t No, int64_t C, int64_t K,
                                  const double *x, const double *w, double *Ya)
{
  int64_t o, c;
  memset(Ya, 0, sizeof(double) * (size_t)(K * C));
  for (c = 0; c < C; c++) {
    for (o = 0; o < No; o++) {
      int64_t k = idx[c * No + o];
      if (k != INT64_MIN) Ya[k + c * K] += w[c] * x[o];
    }
  }
}

void dream_oracle_das_wgrad_f64(const int64_t *idx, int64_t No, int64_t C, int64_t K,
                                const double *g, const double *Y, double *dw)
{
  int64_t o, c;
  for (c = 0; c < C; c++) {
    double s = 0.0;
    for (o = 0; o < No; o++) {
      int64_t k = idx[c * No + o];
      if (k != INT64_MIN) s += g[o] * Y[k + c * K];
    }
    dw[c] = s;
  }
}
