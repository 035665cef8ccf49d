/* fftw_stub.c -- stand-ins for the FFTW 3 entry points declared in
 * oracle/fftw_stub/fftw3.h. TEST INFRASTRUCTURE ONLY: linked into the
 * reference SIR builds of oracle/build_ref.sh so that the reference's own CPU
 * dreamrect and dream_arr_rect run without attenuation (alpha = 0). Planning
 * succeeds and does nothing; any transform aborts, so a build that reached
 * the attenuation path would stop instead of returning wrong numbers. */
#include <stdio.h>
#include <stdlib.h>

#include "fftw_stub/fftw3.h"

struct dream_fftw_stub_plan {
  int n;
};
static struct dream_fftw_stub_plan g_plan;

void *fftw_malloc(size_t n) { return malloc(n ? n : 1); }
void fftw_free(void *p) { free(p); }

fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags) {
  (void)in, (void)out, (void)flags;
  g_plan.n = n;
  return &g_plan;
}
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned flags) {
  (void)in, (void)out, (void)flags;
  g_plan.n = n;
  return &g_plan;
}

static void no_transform(const char *what) {
  fprintf(stderr, "fftw stub: %s called (attenuation path); this oracle build has no FFTW\n", what);
  abort();
}
void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out) {
  (void)p, (void)in, (void)out;
  no_transform("fftw_execute_dft_r2c");
}
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out) {
  (void)p, (void)in, (void)out;
  no_transform("fftw_execute_dft_c2r");
}

int fftw_import_wisdom_from_string(const char *s) {
  (void)s;
  return 0;
}
void fftw_forget_wisdom(void) {}
char *fftw_export_wisdom_to_string(void) { return NULL; }
