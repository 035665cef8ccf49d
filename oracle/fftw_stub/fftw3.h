/* fftw3.h -- declarations of the few FFTW 3 entry points that DREAM's
 * include/fft.h names, so that the reference's SIR sources (src/dreamrect.cc,
 * src/dream_arr_rect.cc, src/attenuation.cc) compile unmodified here, where
 * FFTW is not installed.
 *
 * TEST INFRASTRUCTURE ONLY (oracle/build_ref.sh). The definitions in
 * oracle/fftw_stub.c allocate with malloc and plan nothing; executing a
 * transform aborts the process. The reference runs a transform only for
 * attenuation (alpha > 0, src/attenuation.cc); with alpha = 0 it constructs
 * its FFT object (plans) but never executes one, which is the only case the
 * oracle uses these builds for.
 */
#ifndef DREAM_ORACLE_FFTW3_STUB_H
#define DREAM_ORACLE_FFTW3_STUB_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct dream_fftw_stub_plan *fftw_plan;

/* planner flags (values irrelevant to the stub) */
#define FFTW_MEASURE (0U)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

void *fftw_malloc(size_t n);
void fftw_free(void *p);
fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned flags);
void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out);
int fftw_import_wisdom_from_string(const char *s);
void fftw_forget_wisdom(void);
char *fftw_export_wisdom_to_string(void);

#ifdef __cplusplus
}
#endif

#endif
