/*
 * dream_conv.h -- C ABI of the GPU column-wise convolution (conv_p /
 * fftconv_p), the step before beamforming in DREAM's examples and tests:
 * spatial impulse responses convolved with a pulse give the A-scans.
 *
 * Replaces, for device='cuda':
 *   fftconv_p(A, B)          python/src/py_fftconv_p.cc:40-41,
 *                            python/include/py_fftconv_p.hpp:40-89
 *   conv_p(A, B[, Y[, mode]]) extra_src/oct_conv_p.cc:160-330 (Octave),
 *                            extra_src/mex_conv_p.cc (MATLAB)
 *   per column                extra_src/conv.cc:34-78 (conv), extra_src/fftconv_p.cc
 *
 * Y[:, n] = A[:, n] * B[:, n] (B a matrix with A_N columns) or A[:, n] * B
 * (B a vector, either orientation), Y with A_M + B_M - 1 rows; all FP64 and
 * column-major. Each output sums its products in the reference conv()'s
 * order without fused multiply-add, so for finite inputs the result equals
 * conv() bit for bit and FFTW's fftconv_p to rounding. Status codes are
 * those of dream_das.h (0 success, negative errors; dream_das_last_error()).
 */
#ifndef DREAM_CONV_H
#define DREAM_CONV_H

#include <stdint.h>

#include "dream_das.h"

#ifdef __cplusplus
extern "C" {
#endif

/* In-place modes of conv_p (ConvMode, include/dream.h:91-95). */
#define DREAM_CONV_EQU 0 /* '='  : Y = A * B   */
#define DREAM_CONV_SUM 1 /* '+=' : Y += A * B  */
#define DREAM_CONV_NEG 2 /* '-=' : Y -= A * B  */

/* Device buffers on `stream` (NULL: the default stream); asynchronous. dY
 * holds (A_M + B_M - 1) x A_N values (read first by '+=' and '-='). */
int dream_conv_p_run_device(const double *dA, int64_t A_M, int64_t A_N, const double *dB, int64_t B_M,
                            int64_t B_N, double *dY, int mode, void *stream);

/* Host buffers on CUDA device `device`; blocking. Device memory is kept per
 * device between calls and grown as needed. */
int dream_conv_p_run(const double *A, int64_t A_M, int64_t A_N, const double *B, int64_t B_M, int64_t B_N,
                     double *Y, int mode, int device);

/* Full-matrix-capture A-scan synthesis in two launches (no reference entry:
 * it batches the reference's per-transmit loop of fftconv_p calls,
 * python/tests/test_das_tfm.py:110-115 and test_das_rca.py:117-124):
 * column t*L_r + r of dY ((2M-1 + P_M-1) x L_t*L_r) is
 * (dHr[:, r] (*) dHt[:, t]) (*) dP, with dHt M x L_t (transmit SIRs), dHr
 * M x L_r (receive SIRs; dHt again for TFM), dP the P_M-sample pulse and dDP
 * (2M-1) x L_t*L_r scratch for the double-path responses. Bit-identical to
 * the two fftconv_p calls per transmit. Device buffers; asynchronous on
 * `stream`. */
int dream_conv_p_fmc_device(const double *dHt, int64_t M, int64_t L_t, const double *dHr, int64_t L_r,
                            const double *dP, int64_t P_M, double *dDP, double *dY, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* DREAM_CONV_H */
