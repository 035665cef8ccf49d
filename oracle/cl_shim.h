/*
 * cl_shim.h -- lets an OpenCL C kernel of the reference (opencl/dreamrect.cl)
 * compile unmodified as C99 on the host for the oracle's reference build
 * (oracle/build_ref.sh): the address-space qualifiers disappear and the
 * work-item index becomes a thread-local variable that the driver loop sets
 * (so host threads may run the kernel on separate point sets at once). TEST
 * INFRASTRUCTURE ONLY.
 */
#include <math.h>
#define __kernel
#define __global
extern __thread int dream_ref_gid;
#define get_global_id(dim) dream_ref_gid
