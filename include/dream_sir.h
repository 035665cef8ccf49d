/*
 * dream_sir.h -- C ABI of the GPU spatial impulse response (SIR) of a
 * rectangular transducer, the model that produces the responses DREAM
 * convolves into A-scans before beamforming them.
 *
 * Replaces, for device='cuda':
 *   dreamrect(Ro, geom_par, s_par, delay, m_par, err_level)
 *       python/src/py_dreamrect.cc:47-139 (binding), src/dreamrect.cc:174-302
 *       (Rect::dreamrect, dreamrect_serial), opencl/dreamrect.cl (OpenCL kernel)
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

#ifdef __cplusplus
}
#endif

#endif /* DREAM_SIR_H */
