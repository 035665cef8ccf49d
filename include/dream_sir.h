/*
 * dream_sir.h -- C ABI of the GPU spatial impulse response (SIR) of a
 * rectangular transducer, the model that produces the responses DREAM
 * convolves into A-scans before beamforming them.
 *
 * Replaces, for device='cuda':
 *   dreamrect(Ro, geom_par, s_par, delay, m_par, err_level)
 *       python/src/py_dreamrect.cc:47-139 (binding), src/dreamrect.cc:174-302
 *       (Rect::dreamrect, dreamrect_serial), opencl/dreamrect.cl (OpenCL kernel)
 *   dream_arr_rect(Ro, geom_par, G, s_par, delay, m_par, foc_met, focal,
 *                  steer_met, steer_par, apod_met, apod, win_par, err_level)
 *       python/src/py_dream_arr_rect.cc:46-227 (binding),
 *       src/dream_arr_rect.cc:192-244 (ArrRect::dream_arr_rect_serial),
 *       src/arr_functions.cc:60-262 (max_dim_arr, focusing, beamsteering,
 *       apodization)
 * without attenuation (m_par alpha = 0; the reference's attenuation path is
 * an FFT-based filter per surface element and has no counterpart here).
 *
 * H is nt x No, column-major: H[k + n*nt] is sample k of the SIR at
 * observation point n (Ro No x 3, column-major, mm). a x b is the element
 * size (mm), dx x dy its discretisation (mm), dt the sampling period (us),
 * delay (us) one value or one per point, v the normal velocity, cp the sound
 * speed (m/s). Every sample receives its surface elements' terms in the
 * reference's order with the reference's rounding, so H equals the
 * reference's bit for bit. Status codes as in dream_das.h: 0..3 mirror
 * SIRError for the out-of-bounds samples under err_level ('stop' reports 3,
 * whose SIRs the reference discards), negative values are errors
 * (dream_das_last_error()). Both entries block until the result is ready.
 */
#ifndef DREAM_SIR_H
#define DREAM_SIR_H

#include <stdint.h>

#include "dream_das.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Device buffers (dRo, ddelay, dH) on CUDA device `device`, work on `stream`
 * (NULL: the default stream). */
int dream_rect_run_device(const double *dRo, int64_t No, double a, double b, double dx, double dy, double dt,
                          int64_t nt, int delay_type, const double *ddelay, double v, double cp, double *dH,
                          int err_level, int64_t *oob_count, int device, void *stream);

/* Host buffers; device memory is kept per device between calls. */
int dream_rect_run(const double *Ro, int64_t No, double a, double b, double dx, double dy, double dt, int64_t nt,
                   int delay_type, const double *delay, double v, double cp, double *H, int err_level,
                   int64_t *oob_count, int device);

/* Focusing, beam-steering and apodisation methods of an array (the
 * reference's FocusMet / SteerMet / ApodMet, include/dream.h, with the
 * strings of include/arg_parser_python.h:316-540 in brackets). */
enum {
  DREAM_FOC_OFF = 0, /* "off" */
  DREAM_FOC_X = 1,   /* "x" */
  DREAM_FOC_Y = 2,   /* "y" */
  DREAM_FOC_XY = 3,  /* "xy" or "on" */
  DREAM_FOC_X_Y = 4, /* "x+y" */
  DREAM_FOC_UD = 5   /* "ud": focal[n] is element n's delay (us) */
};
enum { DREAM_STEER_OFF = 0, DREAM_STEER_X = 1, DREAM_STEER_Y = 2, DREAM_STEER_XY = 3 };
enum {
  DREAM_APOD_OFF = 0,
  DREAM_APOD_TRIANGLE = 1,
  DREAM_APOD_GAUSS = 2,
  DREAM_APOD_RAISED = 3, /* "raised" (raised cosine) */
  DREAM_APOD_HANN = 4,
  DREAM_APOD_HAMMING = 5,
  DREAM_APOD_SIMPLY = 6, /* "simply" (simply supported) */
  DREAM_APOD_CLAMPED = 7,
  DREAM_APOD_UD = 8      /* "ud": apod[n] is element n's weight */
};

/* SIRs of an array of num_elements a x b rectangular elements centred at
 * G (num_elements x 3, column-major, mm), summed per observation point in
 * element order: element n sees the point at Ro - G[n], the delay
 * (delay - foc_n) - steer_n and the weight w_n of its focusing, steering
 * (theta, phi in degrees) and apodisation (apod_par the shape parameter of
 * "gauss" and "raised"). focal holds one focal depth (mm), or num_elements
 * delays for DREAM_FOC_UD; apod num_elements weights for DREAM_APOD_UD (may
 * be NULL otherwise). G, focal and apod are HOST arrays in both entries;
 * dRo, ddelay and dH are device buffers in the _device entry. The result
 * equals the reference's bit for bit; oob_count counts out-of-bounds
 * surface-element terms over all elements. The status follows the
 * reference, which keeps per point the status of the array's last element
 * (src/dream_arr_rect.cc:209-243): DREAM_STATUS_OUT_OF_BOUNDS under 'stop'
 * when any term is out of bounds, the 'ignore' / 'warn' codes only when
 * terms of the last element are. dreamrect is the one-element
 * array at the origin with focusing, steering and apodisation off. */
int dream_arr_rect_run_device(const double *dRo, int64_t No, double a, double b, double dx, double dy, double dt,
                              int64_t nt, int delay_type, const double *ddelay, double v, double cp,
                              int64_t num_elements, const double *G, int foc_met, const double *focal,
                              int steer_met, double theta, double phi, int apod_met, const double *apod,
                              double apod_par, double *dH, int err_level, int64_t *oob_count, int device,
                              void *stream);

int dream_arr_rect_run(const double *Ro, int64_t No, double a, double b, double dx, double dy, double dt,
                       int64_t nt, int delay_type, const double *delay, double v, double cp, int64_t num_elements,
                       const double *G, int foc_met, const double *focal, int steer_met, double theta, double phi,
                       int apod_met, const double *apod, double apod_par, double *H, int err_level,
                       int64_t *oob_count, int device);

#ifdef __cplusplus
}
#endif

#endif /* DREAM_SIR_H */
