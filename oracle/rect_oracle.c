/*
 * rect_oracle.c -- CPU restatement of DREAM's spatial impulse response of a
 * rectangular transducer (dreamrect, no attenuation).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for dream_b200/csrc/dreamrect.cu;
 * only tests/ and bench.py's CPU-baseline leg load it.
 *
 * Restated (reference paths):
 *   dreamrect_serial   src/dreamrect.cc:248-302 (weight 1, no attenuation)
 *   point loop         src/dreamrect.cc:92-170  (smp_dream_rect: delay[0] or delay[n])
 *   error levels       src/dream_error.cc:40-76 ('stop' ends the point at its first
 *                      out-of-bounds sample, as dreamrect_serial returns there)
 * Pinned against the reference itself: its OpenCL kernel opencl/dreamrect.cl,
 * which computes the same per-point sums, is compiled unmodified as C by
 * oracle/build_ref.sh; tests/golden/gen_rect_golden.py stores its outputs and
 * tests/test_oracle_golden.py checks this file reproduces them bit for bit.
 *
 * Arithmetic exactly as written (-ffp-contract=off): surface-element centres
 * by repeated addition (ys += dy, xs += dx), r = sqrt((rx*rx + ry*ry) + rz*rz),
 * ai = ((v*ds)/(2*pi*r)) / dt * 1000, t = (r*1000)/cp,
 * it = rint((t - delay)/dt) (round half to even), h[it] += ai in element order.
 */
#include <math.h>
#include <stdint.h>

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
