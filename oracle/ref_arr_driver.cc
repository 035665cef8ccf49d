// ref_arr_driver.cc -- calls the reference's own array helpers
// (src/arr_functions.cc: max_dim_arr, focusing, beamsteering, apodization),
// compiled unmodified by oracle/build_ref.sh, the way
// ArrRect::dream_arr_rect_serial (src/dream_arr_rect.cc:206-224) calls them.
// TEST INFRASTRUCTURE ONLY: pins dream_oracle_arr_elements (rect_oracle.c)
// and, through it, the element delays and weights of
// dream_b200/csrc/dreamrect.cu. Integer method codes as in
// include/dream_sir.h (DREAM_FOC_*, DREAM_STEER_*, DREAM_APOD_*).
#include <stdint.h>

#include "arr_functions.h"
#include "ref_enums.h"

using ref_codes::apod_of;
using ref_codes::foc_of;
using ref_codes::steer_of;

extern "C" void dream_ref_arr_elements(double *G, int64_t M, int foc_met, double *focal, int steer_met,
                                       double theta, double phi, int apod_met, double *apod, double apod_par,
                                       double cp, double *foc, double *steer, double *weight) {
  double *gx = G, *gy = G + M, *gz = G + 2 * M;
  double x_max, y_max, r_max;
  max_dim_arr(&x_max, &y_max, &r_max, gx, gy, gz, (dream_idx_type)M);
  for (int64_t n = 0; n < M; n++) {
    double fd = 0.0;
    if (foc_of(foc_met) != FocusMet::ud)
      focusing(foc_of(foc_met), focal[0], gx[n], gy[n], x_max, y_max, r_max, cp, &fd);
    else
      fd = focal[n];
    double sd = 0.0;
    beamsteering(steer_of(steer_met), theta, phi, gx[n], gy[n], x_max, y_max, r_max, cp, &sd);
    double w = 1.0;
    if (apod_met != 0) apodization(apod_of(apod_met), (dream_idx_type)n, apod, &w, gx[n], gy[n], r_max, apod_par);
    foc[n] = fd;
    steer[n] = sd;
    weight[n] = w;
  }
}
