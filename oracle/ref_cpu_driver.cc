// ref_cpu_driver.cc -- C entry points into the reference's own CPU code,
// compiled unmodified by oracle/build_ref.sh:
//   dream_ref_conv       conv()                    extra_src/conv.cc:33-78
//   dream_ref_dreamrect  Rect::dreamrect           src/dreamrect.cc
//   dream_ref_arr_rect   ArrRect::dream_arr_rect   src/dream_arr_rect.cc:312-420
// with alpha = 0 (no attenuation: the FFTW stand-ins of oracle/fftw_stub.c
// are planned but never executed). The configuration is the reference's
// Python module's (DREAM_PYTHON, HAVE_FFTW), so dream_idx_type is the signed
// pybind11 ssize_t. TEST INFRASTRUCTURE ONLY: pins the C restatements in
// oracle/ (conv_oracle.c, rect_oracle.c) and the GPU kernels through them.
// The SIR entries return the reference's SIRError as an int; the reference
// reports no out-of-bounds count.
#include <stdint.h>

#include "conv.h"
#include "dream_arr_rect.h"
#include "dreamrect.h"
#include "ref_enums.h"

extern "C" void dream_ref_conv(double *x, int64_t nx, double *y, int64_t ny, double *z, int mode) {
  conv(x, (dream_idx_type)nx, y, (dream_idx_type)ny, z,
       mode == 1 ? ConvMode::sum : (mode == 2 ? ConvMode::neg : ConvMode::equ));
}

extern "C" int dream_ref_dreamrect(double *Ro, int64_t No, double a, double b, double dx, double dy, double dt,
                                   int64_t nt, int delay_multi, double *delay, double v, double cp, int err_level,
                                   double *h) {
  Rect r;
  SIRError e = r.dreamrect(0.0, Ro, (dream_idx_type)No, a, b, dx, dy, dt, (dream_idx_type)nt,
                           delay_multi ? DelayType::multiple : DelayType::single, delay, v, cp, h,
                           ref_codes::err_of(err_level));
  return (int)e;
}

extern "C" int dream_ref_arr_rect(double *Ro, int64_t No, double a, double b, double dx, double dy, double dt,
                                  int64_t nt, int delay_multi, double *delay, double v, double cp, int64_t M,
                                  double *G, int foc_met, double *focal, int steer_met, double theta, double phi,
                                  int apod_met, double *apod, double apod_par, int err_level, double *h) {
  ArrRect ar;
  SIRError e = ar.dream_arr_rect(0.0, Ro, (dream_idx_type)No, a, b, dx, dy, dt, (dream_idx_type)nt,
                                 delay_multi ? DelayType::multiple : DelayType::single, delay, v, cp,
                                 (dream_idx_type)M, G, ref_codes::foc_of(foc_met), focal,
                                 ref_codes::steer_of(steer_met), theta, phi, apod, apod_met != 0,
                                 apod_met != 0 ? ref_codes::apod_of(apod_met) : ApodMet::gauss, apod_par, h,
                                 ref_codes::err_of(err_level));
  return (int)e;
}
