/*
 * dream_das.h -- C ABI of the B200 (sm_100a) delay-and-sum beamformer.
 *
 * This is the drop-in boundary for DREAM's DAS path. Every entry point takes
 * plain pointers and sizes; array layouts are DREAM's (column-major):
 *   Y   [K x C]   A-scans, sample k of A-scan column c at Y[k + c*K]
 *               (C = Nt for SAFT, Nt*Nr for TFM and RCA col-tx, Nr*Nt for
 *                RCA row-tx, exactly the reference's column order)
 *   Ro  [No x 3]  observation points, Ro[n + j*No]
 *   Gt  [Nt x 3]  transmit elements (RCA: the columns), Gt[n + j*Nt]
 *   Gr  [Nr x 3]  receive elements (RCA: the rows)
 *   delay         1 value or No values [us]; dt [us]; cp [m/s]; positions [mm]
 *   Im  [No]      output image
 *
 * Reference interfaces replaced (paths inside the DREAM source tree):
 *   dream_das_plan_create        DAS<T>::DAS (include/das.h:56-63,
 *                                extra_src/das.cc:36-53; OpenCL ctor
 *                                opencl/cl_das.cc:30-52)
 *   dream_das_setup_has_changed  DAS<T>::das_setup_has_changed (include/das.h:77-94)
 *   dream_das_run                DAS<T>::das (include/das.h:67-72,
 *                                extra_src/das.cc:199-298) and
 *                                DAS<T>::cl_das (opencl/cl_das.cc:61-159)
 *   dream_das_uni_plan_create    DAS_UNI<T>::DAS_UNI (include/das_uni.h:55-64,
 *                                opencl/cl_das_uni.cc:32-60)
 *   dream_das_uni_run            DAS_UNI<T>::cl_das_uni (opencl/cl_das_uni.cc:70-187)
 *   dream_das_cancel             DAS<T>::abort (extra_src/das.cc:61-65)
 *   status values                SIRError (include/dream.h:42-47)
 *   err_level values             ErrorLevel (include/dream.h:49-55)
 *   das_type values              DASType (include/dream.h:97-102)
 *   delay_type values            DelayType (include/dream.h:57-60)
 *
 * Thread safety: no globals are shared between plans; use one plan per host
 * thread (or per stream). A plan serialises its own calls.
 */
#ifndef DREAM_DAS_H
#define DREAM_DAS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes: >= 0 mirror SIRError, < 0 are errors of this library ---- */
#define DREAM_STATUS_NONE 0
#define DREAM_STATUS_IGNORE_OUT_OF_BOUNDS 1
#define DREAM_STATUS_WARN_OUT_OF_BOUNDS 2
#define DREAM_STATUS_OUT_OF_BOUNDS 3
#define DREAM_ERR_ARGUMENT (-1)    /* invalid argument or shape */
#define DREAM_ERR_CUDA (-2)        /* CUDA runtime error (message via dream_das_last_error) */
#define DREAM_ERR_ALLOC (-3)       /* device allocation failed */
#define DREAM_ERR_UNSUPPORTED (-4) /* combination not implemented */
#define DREAM_ERR_CANCELLED (-5)   /* dream_das_cancel was called */

/* ---- enums (values equal the reference's enum class ordinals) ---- */
#define DREAM_DAS_SAFT 0
#define DREAM_DAS_TFM 1
#define DREAM_DAS_RCA_COLTX 2
#define DREAM_DAS_RCA_ROWTX 3

#define DREAM_ERR_LEVEL_NONE 0
#define DREAM_ERR_LEVEL_IGNORE 1
#define DREAM_ERR_LEVEL_WARN 2
#define DREAM_ERR_LEVEL_STOP 3
#define DREAM_ERR_LEVEL_PARALLEL_STOP 4

#define DREAM_DELAY_SINGLE 0
#define DREAM_DELAY_MULTIPLE 1

/*
 * Precision of a plan.
 *   F64   DAS<double>: everything in FP64; sample indices and images are
 *         bit-identical to the reference CPU `das`.
 *   F32   DAS<float>: everything in FP32 with the reference's constants;
 *         indices and images bit-identical to the reference `das_f`.
 *   F32_STORE  geometry in FP64 and FP64-exact sample indices (the indices
 *         of F64), A-scans stored in FP32, FP32 compensated accumulation,
 *         FP32 image.
 *   BF16_STORE as F32_STORE with the A-scans stored in BF16 (the plan
 *         converts FP32 input on the device; device-pointer calls may pass
 *         BF16 directly, see dream_das_run_device).
 */
#define DREAM_PREC_F64 0
#define DREAM_PREC_F32 1
#define DREAM_PREC_F32_STORE 2
#define DREAM_PREC_BF16_STORE 3

typedef struct dream_das_plan dream_das_plan;

/* Library version string. */
const char *dream_das_version(void);

/* Message of the last error raised on this host thread ("" if none). */
const char *dream_das_last_error(void);

/*
 * Creates a plan (the persistent object the reference bindings cache).
 * num_r_elements == 0 selects SAFT whatever das_type says
 * (extra_src/das.cc:211-213). device is the CUDA ordinal.
 */
int dream_das_plan_create(dream_das_plan **plan, int das_type, int64_t a_scan_len, int64_t No,
                          int64_t num_t_elements, int64_t num_r_elements, int precision,
                          int device);

/* 1 if a plan cannot be reused for this setup, 0 if it can. */
int dream_das_setup_has_changed(const dream_das_plan *plan, int das_type, int64_t a_scan_len,
                                int64_t No, int64_t num_t_elements, int64_t num_r_elements,
                                int precision, int device);

void dream_das_plan_destroy(dream_das_plan *plan);

/*
 * Runs DAS on HOST buffers (copies in, computes, copies out; blocking).
 * Element types: F64 -> double for all arrays; F32 -> float for all arrays;
 * F32_STORE / BF16_STORE -> Y float, Ro/Gt/Gr/delay double, Im float.
 * dt, cp are passed as double; F32 plans round them to float first, as a
 * float-typed caller of DAS<float> would have them.
 * Returns a status (see above); oob_count (may be NULL) receives the number
 * of out-of-bounds terms.
 */
int dream_das_run(dream_das_plan *plan, const void *Y, const void *Ro, const void *Gt,
                  const void *Gr, double dt, int delay_type, const void *delay, double cp,
                  void *Im, int err_level, int64_t *oob_count);

/*
 * As dream_das_run on DEVICE buffers, enqueued on `stream` (a cudaStream_t;
 * NULL is the default stream). Waits for the stream to report the status.
 * BF16_STORE plans take Y as BF16 (uint16 bit patterns) here.
 */
int dream_das_run_device(dream_das_plan *plan, const void *dY, const void *dRo, const void *dGt,
                         const void *dGr, double dt, int delay_type, const void *ddelay, double cp,
                         void *dIm, int err_level, int64_t *oob_count, void *stream);

/*
 * Fully asynchronous device variant: never synchronises and adds the number
 * of out-of-bounds terms to the caller's device counter d_oob (uint64, may be
 * NULL). Safe to capture in a CUDA graph. Returns only argument errors.
 */
int dream_das_run_device_async(dream_das_plan *plan, const void *dY, const void *dRo,
                               const void *dGt, const void *dGr, double dt, int delay_type,
                               const void *ddelay, double cp, void *dIm,
                               unsigned long long *d_oob, void *stream);

/*
 * Uniform-grid plan (DAS_UNI). tri holds 15 values:
 *   [min_t, pitch_t, max_t, min_r, pitch_r, max_r,
 *    min_x, dx, max_x, min_y, dy, max_y, min_z, dz, max_z]
 * (the receive triplet is ignored for SAFT). Only F64 and F32 are offered.
 * Counts are (int)((max - min)/pitch + 1.0) in the plan precision
 * (include/das_uni.h:70-78); pixel n maps to (ny fastest, then nz, then nx).
 */
int dream_das_uni_plan_create(dream_das_plan **plan, int das_type, int64_t a_scan_len,
                              const double *tri, int precision, int device);

/* Number of image points of a plan (uniform plans: Nx*Ny*Nz). */
int64_t dream_das_plan_num_points(const dream_das_plan *plan);

/* Number of A-scan columns Y must hold (Nt for SAFT, Nt*Nr otherwise). */
int64_t dream_das_plan_num_ascans(const dream_das_plan *plan);

/* Runs das_uni on host buffers: Y (T), Im (T) with T of the plan precision. */
int dream_das_uni_run(dream_das_plan *plan, const void *Y, const double *tri, double dt,
                      double delay, double cp, void *Im, int err_level, int64_t *oob_count);

/* Device-buffer variant of dream_das_uni_run. */
int dream_das_uni_run_device(dream_das_plan *plan, const void *dY, const double *tri, double dt,
                             double delay, double cp, void *dIm, int err_level,
                             int64_t *oob_count, void *stream);

/*
 * The sample index of every term: d_idx[c * No + n] = k(n, c) in [0, K), the
 * sample of A-scan column c that das() adds for image point n, or -1 when the
 * term is out of bounds (DAS<T>::das's per-term truncation and bounds test,
 * extra_src/das.cc:306-626). This is the sparse DAS matrix: row n has the
 * entry 1 (or the column's weight) at column c * K + k(n, c), and summing a
 * row in column order gives das()'s image bit for bit (the reference builds
 * the matrix densely in examples/model_based_example.m:381-456). F32 plans
 * give das_f's indices; F64, F32_STORE and BF16_STORE plans das's FP64 ones.
 * Ro, Gt, Gr and the delay are in the plan's geometry precision (FP32 for F32
 * plans, FP64 otherwise). d_idx holds terms x No int64 values; oob_count
 * (optional; synchronises the stream) receives the out-of-bounds terms.
 */
int dream_das_indices_device(dream_das_plan *plan, const void *dRo, const void *dGt, const void *dGr, double dt,
                             int delay_type, const void *ddelay, double cp, int64_t *d_idx,
                             int64_t *oob_count, void *stream);

/* Number of kernels this plan has launched since it was created. */
int64_t dream_das_plan_launch_count(const dream_das_plan *plan);

/*
 * 1 when this library is the bounds-checked build (nvcc -DDREAM_DAS_CHECKED,
 * libdream_das_checked.so), 0 otherwise. In that build every A-scan gather of
 * the das / das_uni kernels tests its element index against the extent of Y
 * and skips (and counts) a load outside it; the reference's counterpart is
 * running the CPU code under a memory checker.
 */
int dream_das_checked_build(void);

/*
 * Gather indices outside Y that the bounds-checked build caught for this plan
 * since it was created (synchronises the device). Always 0 in the normal
 * build; negative status on error.
 */
int64_t dream_das_plan_bound_violations(dream_das_plan *plan);

/*
 * Image-grid hint for the F32_STORE / BF16_STORE kernels: image point n is
 * (n mod n_fast, n / n_fast) on a regular 2-D (or flattened 3-D) grid whose
 * fastest axis has n_fast points, e.g. Nz for Ro = meshgrid(x, z) flattened
 * column-major. Points adjacent on both axes are then processed by the same
 * CTA. 0 removes the hint (consecutive points are grouped). Any value gives
 * the same image; only speed depends on it. No must be a multiple of n_fast.
 */
int dream_das_set_grid_hint(dream_das_plan *plan, int64_t n_fast);

/*
 * Tile of image points per CTA for the F32_STORE / BF16_STORE kernels:
 * tile_f points along the fast grid axis x tile_s along the slow axis
 * (tile_f*tile_s threads, 32..256, a multiple of 32; with a grid hint tile_f
 * is a multiple of 8 and tile_s of 4, without one tile_s must be 1).
 * (0, 0) restores the automatic choice. Used by the autotuner. Automatic,
 * on a hinted grid: 16 x 8 points for the gathers (8 x 32 for frames of fewer
 * points than two waves of 128-point tiles, 8 x 128 per SM), 8 x 32 for the
 * operator's adjoint on TFM frames; 256 consecutive points without a hint; fewer points
 * when many outer elements would overflow the tile's shared memory.
 */
int dream_das_set_tile(dream_das_plan *plan, int tile_f, int tile_s);
int dream_das_get_tile(const dream_das_plan *plan, int *tile_f, int *tile_s);

/* Inner elements per register chunk of the F32_STORE / BF16_STORE kernels:
 * 8 or 16 (0 = automatic, 16). Used by the autotuner. */
int dream_das_set_chunk(dream_das_plan *plan, int jc);

/*
 * Inner-element shard of an F32_STORE / BF16_STORE plan (TFM and RCA; no
 * counterpart in the reference). After dream_das_set_inner_shard(plan, lo, hi)
 * the A-scans passed to the device entry points hold only the columns of
 * inner elements [lo, hi) (TFM: receivers; RCA col-tx: rows; RCA row-tx:
 * columns), column (o, i) at o * (hi - lo) + (i - lo), and the image is the
 * partial sum over those terms; Gt and Gr stay the full element arrays (the
 * RCA stripe edges are read from them). Ranks that each hold one shard of an
 * RCA frame add their partial images (one all-reduce) to get the frame.
 * lo = hi = 0 restores the full layout. The host entry dream_das_run refuses a
 * sharded plan.
 */
int dream_das_set_inner_shard(dream_das_plan *plan, int64_t lo, int64_t hi);

/*
 * L2 blocking of the F32_STORE / BF16_STORE kernels (TFM, RCA; no counterpart
 * in the reference, whose CPU loops have no such cache to fit). A-scans larger
 * than the budget are beamformed in passes over ranges of inner elements (a
 * multiple of 16 each) whose A-scans take at most `bytes`, each pass adding
 * into the image: the pass's samples stay in L2 while every image point
 * gathers from them. 0 = automatic (passes of at most 96 MB when the A-scans
 * exceed 160 MB), < 0 = never split. The image changes only by FP32 rounding.
 */
int dream_das_set_l2_block(dream_das_plan *plan, int64_t bytes);

/*
 * Weighted DAS, the forward operator of the differentiable beamformer:
 *   Im[n] = sum over A-scan columns c of w[c] * Y[k(n, c), c]
 * with k the FP64-exact sample index of the plain method. F32_STORE and
 * BF16_STORE plans only; dW holds one float per A-scan column (Nt for SAFT,
 * Nt*Nr otherwise, in Y's column order). Asynchronous like
 * dream_das_run_device_async.
 */
int dream_das_weighted_run_device(dream_das_plan *plan, const void *dY, const void *dRo,
                                  const void *dGt, const void *dGr, double dt, int delay_type,
                                  const void *ddelay, double cp, const float *dW, float *dIm,
                                  unsigned long long *d_oob, void *stream);

/*
 * Geometry-bound operator of the differentiable beamformer (F32_STORE plans;
 * FP32 A-scans, images and weights). No reference counterpart: DREAM has no
 * adjoint; its explicit DAS matrix example (examples/model_based_example.m:
 * 381-456) is what this replaces.
 *
 * dream_das_bind_geometry keeps the device pointers dRo, dGt, dGr, ddelay
 * (which must stay valid while bound) and the constants; nothing is
 * precomputed: every operator forms its legs per image tile, as the FP32/BF16
 * storage kernels do. With the A-scan column index c and the FP64 reference
 * sample index k(n, c):
 *   forward  Im[n]    = sum_c w[c] * Y[k(n,c), c]          (w NULL: all ones)
 *   adjoint  Ya[k, c] = w[c] * sum_{n: k(n,c)=k} X[n]       (Ya overwritten)
 *   wgrad    dW[c]    = sum_n G[n] * Y[k(n,c), c]           (dW overwritten)
 *   backward adjoint(G, w) into dYg and wgrad(G, Y) into dWg
 * wgrad is computed as sum_k Y[k,c] * (adjoint of G, unweighted)[k,c] through
 * a plan-owned scratch of K x columns floats; backward uses dYg for it. All
 * are asynchronous on `stream`; forward adds out-of-bounds terms to d_oob
 * when it is not NULL. The image tiling follows dream_das_set_grid_hint /
 * dream_das_set_tile / dream_das_set_chunk.
 */
int dream_das_bind_geometry(dream_das_plan *plan, const void *dRo, const void *dGt, const void *dGr,
                            double dt, int delay_type, const void *ddelay, double cp, void *stream);
int dream_das_op_forward(dream_das_plan *plan, const float *dY, const float *dW, float *dIm,
                         unsigned long long *d_oob, void *stream);
int dream_das_op_adjoint(dream_das_plan *plan, const float *dX, const float *dW, float *dYa,
                         void *stream);
int dream_das_op_wgrad(dream_das_plan *plan, const float *dG, const float *dY, float *dWgrad,
                       void *stream);
int dream_das_op_backward(dream_das_plan *plan, const float *dG, const float *dY, const float *dW,
                          float *dYgrad, float *dWgrad, void *stream);

/*
 * Batched DAS: many frames of uneven element counts, A-scan lengths and
 * image sizes in ONE persistent launch. No reference counterpart (the
 * reference beamforms one frame per call); each frame has the meaning of
 * one dream_das_run_device call on an F32_STORE / BF16_STORE plan.
 * Pointers are device pointers that must stay valid while the batch exists;
 * their contents may change between runs (a run reads them when it executes,
 * so a captured CUDA graph of dream_das_batch_run can be replayed on new
 * data). TFM and RCA methods; tile_f * tile_s must be 128 when given.
 */
typedef struct dream_das_frame {
  int das_type;
  int64_t a_scan_len;
  int64_t No;
  int64_t num_t_elements;
  int64_t num_r_elements;
  const void *Y;       /* K x C, FP32 (F32_STORE) or BF16 bits (BF16_STORE) */
  const double *Ro;    /* No x 3 */
  const double *Gt;    /* Nt x 3 */
  const double *Gr;    /* Nr x 3 */
  const double *delay; /* 1 or No values [us] */
  int delay_type;
  double dt, cp;
  float *Im;           /* No */
  int64_t n_fast;      /* grid hint, 0 = none */
  int tile_f, tile_s;  /* 0, 0 = automatic */
  int jc;              /* inner chunk 8 or 16, 0 = automatic */
} dream_das_frame;

typedef struct dream_das_batch dream_das_batch;

int dream_das_batch_create(dream_das_batch **batch, const dream_das_frame *frames, int n_frames,
                           int precision, int device);
/* One persistent launch over all frames (queue reset + kernel, both stream
 * operations: capturable). d_oob (may be NULL) accumulates out-of-bounds terms. */
int dream_das_batch_run(dream_das_batch *batch, unsigned long long *d_oob, void *stream);
/* Number of (frame, tile) work items and the persistent grid size. */
int64_t dream_das_batch_items(const dream_das_batch *batch);
int dream_das_batch_grid(const dream_das_batch *batch);
void dream_das_batch_destroy(dream_das_batch *batch);

/*
 * Allocation-free batch run. No counterpart in the reference (DREAM always
 * allocates its buffers). For callers that cannot call cudaMalloc -- device
 * memory owned by another framework's pool or a budget fixed at start-up,
 * real-time pipelines that forbid allocation after initialisation -- this
 * runs the same persistent batch kernel as dream_das_batch_run without
 * creating a batch object and without allocating: the work queue counter,
 * frame table and tile list go to a 4 MiB device array inside this library
 * (every GPU that loads the library holds it until exit). Batches needing
 * more scratch are rejected with DREAM_ERR_ARGUMENT and a message.
 * The first call on a device looks the array up (cudaGetSymbolAddress). Each
 * call stages its frame table and tile list in a host array that the next call
 * rewrites and copies them to the device on the stream, so a stream that is
 * being captured into a CUDA graph is refused (DREAM_ERR_UNSUPPORTED); use
 * dream_das_batch_run for captured batches. Calls share the array: calls that
 * overlap on the GPU (other streams or threads) race; calls on one stream are
 * ordered. Frames (validated exactly as by dream_das_batch_create) and d_oob
 * as for dream_das_batch_create/_run.
 */
int dream_das_batch_run_noalloc(const dream_das_frame *frames, int n_frames, int precision,
                                int device, unsigned long long *d_oob, void *stream);

/* Requests cancellation: running and later calls return DREAM_ERR_CANCELLED
 * between launches until dream_das_set_running is called. */
void dream_das_cancel(dream_das_plan *plan);
void dream_das_set_running(dream_das_plan *plan);

#ifdef __cplusplus
}
#endif

#endif /* DREAM_DAS_H */
