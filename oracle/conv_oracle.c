/*
 * conv_oracle.c -- CPU restatement of DREAM's column-wise convolution
 * (conv_p / fftconv_p), the step that turns spatial impulse responses into
 * the A-scans the beamformer reads.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for dream_b200/csrc/conv_p.cu; only
 * tests/ and bench.py's CPU-baseline leg load it.
 *
 * Pinned against the reference's own conv() (extra_src/conv.cc, compiled
 * unmodified by oracle/build_ref.sh into oracle/_ref/libref_cpu.so; stored
 * outputs in tests/golden/ref_cpu_golden.npz). This file restates the direct
 * form line for line:
 *   conv()          extra_src/conv.cc:34-78  (zr[i+j] += xr[i]*yr[j], i outer,
 *                   j inner; '=' clears first, '+=' adds, '-=' subtracts)
 *   column loop     extra_src/oct_conv_p.cc:88-96 (column n of A with column n
 *                   of B, or with the vector B for every column)
 *   argument rules  extra_src/oct_conv_p.cc:225-236, python/include/py_fftconv_p.hpp:70-77
 * fftconv_p (extra_src/fftconv_p.cc, fftconv.cc) computes the same full linear
 * convolution through FFTW, which differs from the direct form by rounding
 * only (FFTW is not installed here); the tests also compare the direct form
 * with numpy.convolve as an independent implementation.
 *
 * Compile with -ffp-contract=off: each product and each sum rounds as written.
 */
#include <stdint.h>

/* mode: 0 '=' (ConvMode::equ), 1 '+=' (ConvMode::sum), 2 '-=' (ConvMode::neg),
 * the ordinals of include/dream.h:91-95. A is A_M x A_N, B is B_M x B_N with
 * B_N == 1 (a vector for every column) or B_N == A_N; Y is
 * (A_M + B_M - 1) x A_N, all column-major. */
void dream_oracle_conv_p(const double *A, int64_t A_M, int64_t A_N, const double *B, int64_t B_M,
                         int64_t B_N, double *Y, int mode)
{
  const int64_t ny = A_M + B_M - 1;
  for (int64_t n = 0; n < A_N; n++) {
    const double *xr = A + n * A_M;
    const double *yr = B + (B_N > 1 ? n * B_M : 0);
    double *zr = Y + n * ny;
    if (mode == 0)
      for (int64_t i = 0; i < ny; i++) zr[i] = 0.0;
    for (int64_t i = 0; i < A_M; i++)
      for (int64_t j = 0; j < B_M; j++) {
        if (mode == 2) zr[i + j] -= xr[i] * yr[j];
        else zr[i + j] += xr[i] * yr[j];
      }
  }
}
