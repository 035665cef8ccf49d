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
// Adjoint on the forward's tiles: Ya[k(n,c), c] += w[c] * X[n] (FP32 A-scans;
// P.w may be NULL). Adds into Ya, which the caller zeroes first.
cudaError_t launch_scatter(const FastParams &P, const float *X, float *Ya, cudaStream_t st);
// Per column c of K x ncol arrays: dW[c] = sum_k Y[k,c] * S[k,c] (when Y and dW
// are given), then S[:, c] *= w[c] (when w is given).
cudaError_t launch_column_dot_scale(const float *Y, float *S, const float *w, float *dW, int64_t K, int64_t ncol,
                                    cudaStream_t st);
cudaError_t convert_f32_to_bf16(const float *x, void *y, int64_t n, cudaStream_t st);
// rows x row_elems block of a row-pitched array (same offsets in x and y)
cudaError_t convert_f32_to_bf16_2d(const float *x, void *y, int64_t rows, int64_t row_elems, int64_t pitch,
                                   cudaStream_t st);

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
