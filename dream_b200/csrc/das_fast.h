// das_fast.h -- launch descriptor of the FP32/BF16-storage DAS kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dream {

struct FastParams {
  int method;  // 0 SAFT, 1 TFM, 2 RCA col-tx, 3 RCA row-tx
  const void *Y;  // float or bf16, K x (Nt*Nr) column-major
  int64_t K;
  const double *Ro;
  int64_t No;
  const double *Gt;
  int Nt;
  const double *Gr;
  int Nr;
  const double *delay;  // us; 1 value or No values
  int delay_multi;
  double Fs, ocp;  // (1/dt)*1000 and 1/cp in FP64, as DAS<double>
  const float *w;  // per A-scan column weights, or nullptr
  float *Im;
  unsigned long long *oob;
  // image tiling: point n = s*n_fast + f
  int64_t n_fast, n_slow;
  int tile_f, tile_s, wf;  // tile extents; warp lanes along the fast axis
  int jc;                  // inner elements per register chunk: 8 or 16
  int64_t slow_tile0, slow_tile1;  // slow-tile range of this launch
  int64_t no0, no1;                // point range (SAFT launches)
  // inner-element range [in_lo, in_hi) of this launch (in_hi == 0: all inner
  // elements) and whether to add into Im instead of writing it
  int in_lo, in_hi;
  int accumulate;
  // A-scan columns present in Y: column (o, i) is o * ycol_o + i - ycol_i0
  // (ycol_o == 0: o * n_in + i, the full layout)
  int64_t ycol_o;
  int ycol_i0;
  int64_t ny;               // elements in Y (bounds-checked builds; 0: K * columns)
  unsigned long long *bad;  // gather index violations (bounds-checked builds)
};

size_t fast_smem_bytes(const FastParams &P, int nthr);
cudaError_t launch_fast(const FastParams &P, bool bf16, cudaStream_t st);
cudaError_t convert_f32_to_bf16(const float *x, void *y, int64_t n, cudaStream_t st);
// rows x row_elems block of a row-pitched array (same offsets in x and y)
cudaError_t convert_f32_to_bf16_2d(const float *x, void *y, int64_t rows, int64_t row_elems, int64_t pitch,
                                   cudaStream_t st);

// Geometry-bound operator (leg tables; FP32 samples).
// range: 7 ints of device scratch written by build_leg_tables.
cudaError_t build_leg_tables(const FastParams &P, int64_t *TA, int64_t *TB, int *range, cudaStream_t st);
cudaError_t launch_tab_gather(const FastParams &P, const int64_t *TA, const int64_t *TB, const int *range,
                              cudaStream_t st);
// Adjoint scatter (Ya must be zero when splits > 1; the launcher zeroes nothing)
// and/or weight gradient (dW accumulated atomically: zero it first).
cudaError_t launch_tab_colowner(const FastParams &P, const int64_t *TA, const int64_t *TB, const float *X,
                                const float *G, float *Ya, float *dW, bool adj, bool wg, int sm_count,
                                cudaStream_t st);
int colowner_width(int64_t K, int n_in, bool adj);

// Persistent batch launch over (frame, tile_f index, tile_s index) items
// (int4: frame, tfi, tsi, unused); resets the queue counter *ctr first.
cudaError_t launch_batch(const FastParams *frames, const int4 *items, int n_items, int *ctr, size_t smem, bool bf16,
                         int grid, cudaStream_t st);
int batch_prepare(size_t smem, bool bf16);

}  // namespace dream

struct dream_das_frame;

namespace dream {
// Validates one batch frame and fills its launch descriptor (oob left NULL);
// returns 0 or a DREAM_ERR_* status with the message recorded. Used by
// dream_das_batch_create and dream_das_batch_run_noalloc alike.
int batch_frame_params(const ::dream_das_frame &d, FastParams &F);
}  // namespace dream
