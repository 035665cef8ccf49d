/*
 * rect_oracle.c -- CPU restatement of DREAM's spatial impulse response of a
 * rectangular transducer (dreamrect) and of an array of rectangular elements
 * (dream_arr_rect), both without attenuation.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for dream_b200/csrc/dreamrect.cu;
 * only tests/ and bench.py's CPU-baseline leg load it.
 *
 * Restated (reference paths):
 *   dreamrect_serial   src/dreamrect.cc:248-302 (weight 1, no attenuation)
 *   point loop         src/dreamrect.cc:92-170  (smp_dream_rect: delay[0] or delay[n])
 *   error levels       src/dream_error.cc:40-76 ('stop' ends the point at its first
 *                      out-of-bounds sample, as dreamrect_serial returns there)
 *   dream_arr_rect     src/dream_arr_rect.cc:192-244 (element loop; per point the
 *                      status of the last element is kept), src/arr_functions.cc:60-262
 *                      (max_dim_arr, focusing, beamsteering, apodization)
 * Pinned against the reference itself: its OpenCL kernel opencl/dreamrect.cl,
 * which computes the same per-point sums, is compiled unmodified as C by
 * oracle/build_ref.sh; tests/golden/gen_rect_golden.py stores its outputs and
 * tests/test_oracle_golden.py checks this file reproduces them bit for bit.
 * For arrays, the per-element delays and weights are pinned against the
 * reference's own src/arr_functions.cc (compiled unmodified by
 * oracle/build_ref.sh with oracle/ref_arr_driver.cc); the summation over
 * elements is a restatement, pinned only through its one-element case (the
 * reference's CPU dream_arr_rect needs FFTW and is not built here).
 *
 * Arithmetic exactly as written (-ffp-contract=off): surface-element centres
 * by repeated addition (ys += dy, xs += dx), r = sqrt((rx*rx + ry*ry) + rz*rz),
 * ai = ((v*ds)/(2*pi*r)) / dt * 1000, t = (r*1000)/cp,
 * it = rint((t - delay)/dt) (round half to even), h[it] += ai in element order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* H is nt x No column-major (cleared here). err_level: 0 none, 1 ignore,
 * 2 warn, 3 stop (ErrorLevel ordinals). Returns the SIRError status
 * (0 none, 1 ignore_out_of_bounds, 2 warn_out_of_bounds, 3 out_of_bounds);
 * *oob receives the out-of-bounds surface elements. */
int dream_oracle_rect(const double *Ro, int64_t No, double a, double b, double dx, double dy, double dt,
                      int64_t nt, int delay_multi, const double *delay, double v, double cp, int err_level,
                      double *H, int64_t *oob)
{
  int status = 0;
  int64_t count = 0;
  for (int64_t i = 0; i < nt * No; i++) H[i] = 0.0;
  for (int64_t n = 0; n < No; n++) {
    const double xo = Ro[n], yo = Ro[n + No], zo = Ro[n + 2 * No];
    const double dlay = delay_multi ? delay[n] : delay[0];
    double *h = H + n * nt;
    const double xsmin = -a / 2.0, xsmax = a / 2.0, ysmin = -b / 2.0, ysmax = b / 2.0;
    const double ds = dx * dy;
    const double rz = zo;
    double ys = ysmin + dy / 2.0;
    int stop_point = 0;
    while (ys <= ysmax && !stop_point) {
      const double ry = yo - ys;
      double xs = xsmin + dx / 2.0;
      while (xs <= xsmax) {
        const double rx = xo - xs;
        const double r = sqrt(rx * rx + ry * ry + rz * rz);
        double ai = v * ds / (2 * M_PI * r);
        ai /= dt;
        ai *= 1000.0;
        const double t = r * 1000.0 / cp;
        const int64_t it = (int64_t)rint((t - dlay) / dt);
        if (it < nt && it >= 0) {
          h[it] += ai;
        } else {
          count++;
          if (err_level == 3) {
            status = 3;
            stop_point = 1;
            break;
          }
          if (err_level == 2 && status < 2) status = 2;
          if (err_level == 1 && status < 1) status = 1;
        }
        xs += dx;
      }
      ys += dy;
    }
  }
  if (oob) *oob = count;
  return status;
}

/* Per-element delays (us) and weight of an array, src/arr_functions.cc as
 * src/dream_arr_rect.cc:206-224 calls it. G is M x 3 column-major. foc_met:
 * 0 off, 1 x, 2 y, 3 xy, 4 x+y, 5 ud; steer_met: 0 off, 1 x, 2 y, 3 xy;
 * apod_met: 0 off, 1 triangle, 2 gauss, 3 raised, 4 hann, 5 hamming,
 * 6 simply, 7 clamped, 8 ud. */
void dream_oracle_arr_elements(const double *G, int64_t M, int foc_met, const double *focal, int steer_met,
                               double theta, double phi, int apod_met, const double *apod, double apod_par,
                               double cp, double *foc, double *steer, double *weight)
{
  const double *gx = G, *gy = G + M;
  double x_max, y_max, r_max;
  if (M <= 0) return;
  /* max_dim_arr, src/arr_functions.cc:60-84 */
  x_max = fabs(gx[0]);
  for (int64_t i = 1; i < M; i++)
    if (fabs(gx[i]) > x_max) x_max = fabs(gx[i]);
  y_max = fabs(gy[0]);
  for (int64_t i = 1; i < M; i++)
    if (fabs(gy[i]) > y_max) y_max = fabs(gy[i]);
  r_max = sqrt(x_max * x_max + y_max * y_max);
  for (int64_t n = 0; n < M; n++) {
    double fd = 0.0, sd = 0.0, w = 1.0;
    const double f = focal ? focal[0] : 0.0;
    /* focusing, src/arr_functions.cc:94-148 */
    if (foc_met == 1) {
      double rmax = sqrt(x_max * x_max + f * f);
      double diff = rmax - sqrt(gx[n] * gx[n] + f * f);
      fd = diff * 1.0e3 / cp;
    } else if (foc_met == 2) {
      double rmax = sqrt(y_max * y_max + f * f);
      double diff = rmax - sqrt(gy[n] * gy[n] + f * f);
      fd = diff * 1.0e3 / cp;
    } else if (foc_met == 3) {
      double rmax = sqrt(r_max * r_max + f * f);
      double diff = rmax - sqrt(gx[n] * gx[n] + gy[n] * gy[n] + f * f);
      fd = diff * 1.0e3 / cp;
    } else if (foc_met == 4) {
      double rmax = sqrt(r_max * r_max + f * f);
      double diff = rmax - (sqrt(gx[n] * gx[n] + f * f) + sqrt(gy[n] * gy[n] + f * f));
      fd = diff * 1.0e3 / cp;
    } else if (foc_met == 5) {
      fd = focal[n];
    }
    /* beamsteering, src/arr_functions.cc:156-205 */
    {
      const double deg2rad = M_PI / 180.0;
      double sx_delay = 0.0, sy_delay = 0.0;
      if (steer_met == 1 || steer_met == 3) {
        double sinx = sin(theta * deg2rad);
        double diff = x_max * sinx + gx[n] * sinx;
        sx_delay = diff * 1.0e3 / cp;
      }
      if (steer_met == 2 || steer_met == 3) {
        double siny = sin(phi * deg2rad);
        double diff = y_max * siny + gy[n] * siny;
        sy_delay = diff * 1.0e3 / cp;
      }
      sd = steer_met == 1 ? sx_delay : steer_met == 2 ? sy_delay : steer_met == 3 ? sx_delay + sy_delay : 0.0;
    }
    /* apodization, src/arr_functions.cc:215-262 */
    if (apod_met != 0) {
      double r = sqrt(gx[n] * gx[n] + gy[n] * gy[n]);
      switch (apod_met) {
      case 1: w = 1.0 - fabs(r) / r_max; break;
      case 2: w = exp(-(apod_par * r * r) / (r_max * r_max)); break;
      case 3: w = apod_par + cos(r * M_PI / r_max); break;
      case 4: w = 0.5 * (1.0 - cos((r + r_max) * M_PI / r_max)); break;
      case 5: w = 25.0 / 46.0 - (1.0 - 25.0 / 46.0) * cos((r + r_max) * M_PI / r_max); break;
      case 6: w = 1.0 - r * r / (r_max * r_max); break;
      case 7: w = (1.0 - r * r / (r_max * r_max)) * (1.0 - r * r / (r_max * r_max)); break;
      case 8: w = apod[n]; break;
      }
    }
    foc[n] = fd;
    steer[n] = sd;
    weight[n] = w;
  }
}

/* dream_arr_rect without attenuation: H (nt x No, column-major, cleared
 * here) accumulates every element's dreamrect_serial in element order.
 * Returns the status as the reference reports it (per point the last
 * element's; 'stop' at the first out-of-bounds term); *oob receives the
 * out-of-bounds terms of all elements (up to the stop). */
int dream_oracle_arr_rect(const double *Ro, int64_t No, double a, double b, double dx, double dy, double dt,
                          int64_t nt, int delay_multi, const double *delay, double v, double cp, int64_t M,
                          const double *G, int foc_met, const double *focal, int steer_met, double theta,
                          double phi, int apod_met, const double *apod, double apod_par, int err_level,
                          double *H, int64_t *oob)
{
  int status = 0;
  int64_t count = 0;
  const double *gx = G, *gy = G + M, *gz = G + 2 * M;
  double *fd = malloc(sizeof(double) * 3 * (size_t)(M > 0 ? M : 1)), *sd = fd + M, *w = sd + M;
  if (fd == NULL) return -1;
  dream_oracle_arr_elements(G, M, foc_met, focal, steer_met, theta, phi, apod_met, apod, apod_par, cp, fd, sd, w);
  for (int64_t i = 0; i < nt * No; i++) H[i] = 0.0;
  for (int64_t n = 0; n < No; n++) {
    const double dlay = delay_multi ? delay[n] : delay[0];
    double *h = H + n * nt;
    int point_status = 0;
    for (int64_t m = 0; m < M; m++) {
      /* dreamrect_serial (src/dreamrect.cc:274-335) at Ro - G[m], weight w[m] */
      const double xo = Ro[n] - gx[m], yo = Ro[n + No] - gy[m], zo = Ro[n + 2 * No] - gz[m];
      const double el_delay = dlay - fd[m] - sd[m];
      const double xsmin = -a / 2.0, xsmax = a / 2.0, ysmin = -b / 2.0, ysmax = b / 2.0;
      const double ds = dx * dy;
      double ys = ysmin + dy / 2.0;
      int el_status = 0, stop = 0;
      while (ys <= ysmax && !stop) {
        const double ry = yo - ys;
        double xs = xsmin + dx / 2.0;
        while (xs <= xsmax) {
          const double rx = xo - xs;
          const double r = sqrt(rx * rx + ry * ry + zo * zo);
          double ai = w[m] * v * ds / (2 * M_PI * r);
          ai /= dt;
          ai *= 1000.0;
          const double t = r * 1000.0 / cp;
          const int64_t it = (int64_t)rint((t - el_delay) / dt);
          if (it < nt && it >= 0) {
            h[it] += ai;
          } else {
            count++;
            if (err_level == 3) {
              el_status = 3;
              stop = 1;
              break;
            }
            if (err_level == 1 || err_level == 2) el_status = err_level;
          }
          xs += dx;
        }
        ys += dy;
      }
      point_status = el_status;
      if (stop) break;
    }
    if (point_status) status = point_status;
  }
  free(fd);
  if (oob) *oob = count;
  return status;
}
