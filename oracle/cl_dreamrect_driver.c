/*
 * Host driver of the reference's opencl/dreamrect.cl compiled as C (see
 * cl_shim.h): runs the kernel body once per observation point, as the
 * OpenCL NDRange of opencl/cl_dreamrect.cc does. TEST INFRASTRUCTURE ONLY:
 * the build is the unmodified reference kernel, used to pin
 * dream_oracle_rect (rect_oracle.c) and to generate tests/golden/rect_golden.npz.
 */
__thread int dream_ref_gid;

void dreamrect(const double *Ro, int No, double a, double b, double dx, double dy, double dt, int nt,
               double delay, double v, double cp, double *H);

void dream_ref_dreamrect(const double *Ro, int No, double a, double b, double dx, double dy, double dt, int nt,
                         double delay, double v, double cp, double *H)
{
  for (dream_ref_gid = 0; dream_ref_gid < No; dream_ref_gid++)
    dreamrect(Ro, No, a, b, dx, dy, dt, nt, delay, v, cp, H);
}
