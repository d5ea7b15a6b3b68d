/* plastimatch_b200 -- B200-native B-spline registration cost function.
 *
 * C ABI of libplastimatch_b200.so.  Plain C types only: the caller passes
 * volume geometry, image and coefficient pointers (host or device memory;
 * the library finds out which) and gets the score and gradient back in the
 * reference's layout and normalisation.
 *
 * The entry points replace the reference's CUDA plugin interface for the
 * B-spline cost function (Plastimatch src/register/cuda/bspline_cuda.h:
 * 124-300), which the reference loads with dlopen/dlsym
 * (src/sys/cuda_delayload.h:23-56) and calls from its flavour dispatchers
 * (src/register/bspline_mse.cxx:1937-1962, src/register/bspline_mi.cxx:
 * 3103-3141).  Differences from that interface, by design:
 *   - every call returns a status code (B200BSP_OK / B200BSP_E_*) and never
 *     exits the process (the reference plugin calls exit()),
 *   - device state lives in an opaque context created once per registration
 *     stage instead of the Dev_Pointers_Bspline struct.
 *
 * Threading: one context per host thread (the reference is single-threaded
 * per registration as well).  Contexts are independent; several may share
 * a device.
 */
#ifndef PLASTIMATCH_B200_H
#define PLASTIMATCH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define B200BSP_OK              0
#define B200BSP_E_BADARG       -1   /* invalid argument or geometry */
#define B200BSP_E_OOM          -2   /* device or pinned allocation failed */
#define B200BSP_E_CUDA         -3   /* CUDA runtime error (see last_error) */
#define B200BSP_E_TIMEOUT      -4   /* a bounded device-side wait gave up */
#define B200BSP_E_STATE        -5   /* call out of order (e.g. no images) */
#define B200BSP_E_UNSUPPORTED  -6   /* valid request this build cannot do */
#define B200BSP_E_IO           -7   /* file missing, unreadable or malformed */

/* Kernel forms. */
#define B200BSP_FORM_TC    0   /* tcgen05 tensor-core field + adjoint (default) */
#define B200BSP_FORM_FP32  1   /* plain FP32 SIMT, one thread per voxel */

/* MSE gradient semantics. */
#define B200BSP_MSE_GRAD_NEAREST    0  /* dc/dv = diff * moving_grad[nearest voxel]
                                          (reference flavours c/g/h/i/k/l) */
#define B200BSP_MSE_GRAD_TRILINEAR  1  /* dc/dv = diff * d(trilinear)/dx
                                          (reference flavours o/p/q/r) */

/* Geometry of one volume, as Plastimatch's Volume holds it
 * (src/base/volume.h:37-57): dim in voxels (x fastest), origin and spacing
 * in mm, direction cosines row-major. */
typedef struct {
    int64_t dim[3];
    float origin[3];
    float spacing[3];
    float dcos[9];
} b200bsp_volume;

/* The B-spline control grid over the fixed image: the ROI and knot spacing
 * of Bspline_xform::initialize (src/base/bspline_xform.cxx:491-507).  The
 * grid's image origin/spacing/dcos are the fixed volume's. */
typedef struct {
    int64_t roi_offset[3];
    int64_t roi_dim[3];
    int64_t vox_per_rgn[3];
} b200bsp_grid;

/* Options fixed for the life of a context. */
typedef struct {
    int form;           /* B200BSP_FORM_* */
    int mse_grad;       /* B200BSP_MSE_GRAD_* */
    int mi_bins;        /* fixed and moving histogram bins (reference default 32) */
    int device;         /* CUDA device ordinal */
    int mi_window;      /* B200BSP_MI_* (0: the reference's PVI-8) */
    int wait_limit;     /* polls before a device-side wait of the tensor-core
                           MSE kernel gives up with B200BSP_E_TIMEOUT
                           (0: the default, 1 << 22) */
    int mi_hist;        /* B200BSP_MI_HIST_* (0: equal spacing) */
    int tc_kernel;      /* B200BSP_TC_KERNEL_* (0: chosen per context) */
} b200bsp_opts;

/* The tensor-core form's MSE kernel.  AUTO starts on the tile kernel (the
 * voxels of one tile on the TMEM lanes); b200bsp_autotune may move it to
 * the x-lane kernel (voxel x on the lanes, 3 <= vox_per_rgn[1] <= 10) and
 * back, and image ROIs (b200bsp_set_roi) move it to the x-lane kernel,
 * which is the one that tests them.  XLANE and TILE pin one (XLANE on a
 * grid it cannot take is B200BSP_E_UNSUPPORTED; with TILE pinned, image
 * ROIs are B200BSP_E_UNSUPPORTED in the tensor-core form). */
#define B200BSP_TC_KERNEL_AUTO   0
#define B200BSP_TC_KERNEL_XLANE  1
#define B200BSP_TC_KERNEL_TILE   2

/* Mattes MI histogram windows: PVI-8 partial-volume binning (the
 * reference's, bspline_mi.cxx) or cubic B-spline Parzen windows on the
 * moving intensity and a box window on the fixed one (Mattes et al., IEEE
 * TMI 22(1) 2003; no reference counterpart).  Parzen needs mi_bins >= 5;
 * each image's value range maps onto bins 2 .. mi_bins - 2. */
#define B200BSP_MI_PVI8    0
#define B200BSP_MI_PARZEN  1

/* PVI-8 histogram bins (Bspline_parms::mi_hist_type,
 * src/register/histogram.h:14-17): equal spacing over each image's value
 * range (bspline_initialize_mi_hist_eqsp, joint_histogram.cxx:115-139) or
 * V-optimal bins (bspline_initialize_mi_hist_vopt, :195-324; the image is
 * read back to the host once in b200bsp_set_images for its dynamic
 * programme).  V-optimal needs mi_bins <= 1000; the reference falls back
 * to equal spacing above that (B200BSP_E_BADARG here). */
#define B200BSP_MI_HIST_EQSP  0
#define B200BSP_MI_HIST_VOPT  1

/* Regularisation weights of Regularization_parms
 * (src/register/regularization_parms.h:16-43). */
typedef struct {
    float curvature_penalty;
    float diffusion_penalty;
    float lame_coefficient_1;
    float lame_coefficient_2;
    float total_displacement_penalty;
    float third_order_penalty;
    float linear_elastic_multiplier;   /* reference default 1 */
    float curvature_mixed_weight;      /* reference default 1 */
} b200bsp_reg_parms;

typedef struct b200bsp_ctx b200bsp_ctx;

/* Fill opts with defaults: TC form, nearest-voxel MSE gradient, 32 bins,
 * device 0. */
void b200bsp_default_opts (b200bsp_opts* opts);

/* Library version string. */
const char* b200bsp_version (void);

/* Create a context for one fixed/moving pair and B-spline grid.  Replaces
 * bspline_cuda_state_create + CUDA_bspline_mse_init_j / CUDA_bspline_mi_init_a
 * (src/register/bspline_state.cxx:165-212, bspline_cuda.h:124-140).
 * Computes rdims/cdims and the basis tables as Bspline_xform::allocate does
 * (src/base/bspline_xform.cxx:361-488).  Allocates all device memory the
 * score and regulariser evaluations need; later scoring calls allocate
 * nothing (b200bsp_interpolate_vf / b200bsp_warp with host outputs allocate
 * one staging buffer on first use, see there). */
int b200bsp_create (const b200bsp_volume* fixed, const b200bsp_volume* moving,
    const b200bsp_grid* grid, const b200bsp_opts* opts, b200bsp_ctx** out);

/* Release the context (bspline_cuda_state_destroy,
 * src/register/bspline_state.cxx:214-271).  NULL is accepted. */
int b200bsp_destroy (b200bsp_ctx* ctx);

/* rdims, cdims and num_coeff of the grid (Bspline_header fields). */
int b200bsp_grid_info (const b200bsp_ctx* ctx, int64_t rdims[3],
    int64_t cdims[3], int64_t* num_coeff);

/* Upload the images.  fixed_img/moving_img: float32, dim[0]*dim[1]*dim[2]
 * voxels, x fastest.  moving_grad: float32 xyz interleaved (the output of
 * volume_gradient, src/base/volume_grad.cxx:137-145) or NULL, in which case
 * it is computed on the device with the reference's formula.  For MI the
 * histogram ranges are set here (EQSP, src/register/joint_histogram.cxx:
 * 115-139).  Pointers may be host or device memory. */
int b200bsp_set_images (b200bsp_ctx* ctx, const float* fixed_img,
    const float* moving_img, const float* moving_grad);

/* Use this CUDA stream (cudaStream_t) for all work of the context.  NULL
 * selects the context's own stream. */
int b200bsp_set_stream (b200bsp_ctx* ctx, void* stream);

/* MSE score and gradient: the work of bspline_score_mse for one metric
 * (src/register/bspline_mse.cxx:1865-1964) followed by
 * bspline_score_normalize (:43-72).  Writes curr_smetric (score/N),
 * curr_smetric_grad (2*dC/dp/N, num_coeff floats, xyz interleaved per knot)
 * and curr_num_vox.  With no overlapping voxel, score = FLT_MAX and the
 * gradient is zero, as in the reference.  coeff/score/grad/num_vox may be
 * host or device pointers; with all of them in device memory the call is
 * stream-ordered and returns without waiting. */
int b200bsp_score_mse (b200bsp_ctx* ctx, const float* coeff, float* score,
    float* grad, int64_t* num_vox);

/* As b200bsp_score_mse with double-precision outputs (the device
 * accumulates the score and gradient in double; this skips the final
 * rounding to float). */
int b200bsp_score_mse_f64 (b200bsp_ctx* ctx, const float* coeff,
    double* score, double* grad, int64_t* num_vox);

/* Mattes mutual information with PVI-8 histograms, flavour g semantics
 * (src/register/bspline_mi.cxx:1505-1750): score = -MI, gradient dS/dp,
 * plus the histograms of pass 1 when f_hist/m_hist/j_hist are non-NULL
 * (host pointers; bins, bins, bins*bins doubles). */
int b200bsp_score_mi (b200bsp_ctx* ctx, const float* coeff, float* score,
    float* grad, int64_t* num_vox, double* f_hist, double* m_hist,
    double* j_hist);

/* Analytic regulariser (Bspline_regularize::compute_score with
 * implementation 'b'/'c', src/register/bspline_regularize.cxx:95-126;
 * src/register/bspline_regularize_analytic.cxx:637-1059).  Writes rmetric
 * and ADDS the regulariser gradient into grad (as the reference adds into
 * total_grad). */
int b200bsp_regularize (b200bsp_ctx* ctx, const float* coeff,
    const b200bsp_reg_parms* parms, float* rmetric, float* grad);

/* As b200bsp_regularize with the score returned in double (the device sums
 * it in double; the reference stores it in a float).  No reference
 * counterpart: for gradient checks by finite differences, where the float
 * rounding of the score would swamp a 1e-3 mm step. */
int b200bsp_regularize_f64 (b200bsp_ctx* ctx, const float* coeff,
    const b200bsp_reg_parms* parms, double* rmetric, float* grad);

/* The whole cost function bspline_score() (src/register/bspline.cxx:
 * 558-632) for one similarity metric: metric_type 0 = MSE, 1 = MI;
 * total_score = lambda * smetric (+ rmetric when reg != NULL, + stiffness *
 * lmetric when landmarks are set), total_grad likewise, in that order.
 * With every output in device memory and no landmarks the call is
 * stream-ordered on the context's stream and returns without waiting (for
 * MSE the regulariser's passes overlap the metric kernel); otherwise it
 * returns with the results in place. */
int b200bsp_score (b200bsp_ctx* ctx, const float* coeff, int metric_type,
    float lambda, const b200bsp_reg_parms* reg, float* total_score,
    float* total_grad, float* smetric, int64_t* num_vox);

/* Landmark pairs for the cost function: Bspline_landmarks::set_landmarks
 * and ::initialize (src/register/bspline_landmarks.cxx:145-215), with the
 * stiffness of Bspline_landmarks::landmark_stiffness.  fixed_xyz and
 * moving_xyz are host arrays of points in mm (xyz per point); the first
 * min(n_fixed, n_moving) pairs are used, and a count of 0 removes the
 * landmarks.  Each fixed landmark must lie inside the fixed image
 * (B200BSP_E_BADARG; the reference exits) and its tile, taken from the
 * absolute voxel index as the reference takes it, inside the grid
 * (B200BSP_E_UNSUPPORTED). */
int b200bsp_set_landmarks (b200bsp_ctx* ctx, const float* fixed_xyz,
    int64_t n_fixed, const float* moving_xyz, int64_t n_moving,
    float stiffness);

/* Bounded device-side waits of the tensor-core MSE kernels (no reference
 * counterpart; the reference exits on failures): `polls` mbarrier polls
 * before a wait gives up and the call returns B200BSP_E_TIMEOUT (0: the
 * default, 1 << 22, or opts.wait_limit).  withhold_mma != 0 is a testing
 * aid of the x-lane kernel (B200BSP_E_UNSUPPORTED on a context that is not
 * on it, e.g. opts.tc_kernel = B200BSP_TC_KERNEL_XLANE): its tensor-core
 * warp then issues no MMA, so the compute warps' first wait runs out after
 * `polls` polls -- the failure path, on a GPU, without a fault.  On expiry every warp leaves its loop, the issued
 * MMAs are drained and TMEM is released; the context stays usable. */
int b200bsp_set_wait_limit (b200bsp_ctx* ctx, int polls, int withhold_mma);

/* Testing aid: the nth device allocation made by the next b200bsp_create
 * calls of this thread fails as if the device were full (0 disables).  The
 * create returns B200BSP_E_OOM and releases everything it allocated. */
void b200bsp_debug_fail_alloc (int nth);

/* Testing aid: nonzero makes this thread's b200bsp_optimize_lbfgs calls
 * drive every iteration from the host (one synchronisation per trial)
 * instead of running them as one graph launch, so the two can be
 * compared. */
void b200bsp_debug_host_lbfgs (int on);

/* Image ROIs of the cost function: Bspline_state::fixed_roi and
 * ::moving_roi (src/register/bspline_state.h:44-45), uchar mask volumes
 * (x fastest, nonzero = inside) with their own geometry.  A fixed voxel
 * counts only where the fixed ROI holds at its position, and a moving
 * position only where the moving ROI holds there (inside_roi and
 * bspline_find_correspondence_dcos_roi, src/util/bspline_correspond.cxx:
 * 52-145) -- the reference's ROI flavours (MSE i, bspline_mse.cxx:82-288;
 * MI h, bspline_mi.cxx:1232-1504).  Either pair (geometry, mask) may be
 * NULL for none; masks are host or device memory.  Replaces the previous
 * ROIs; all four NULL removes them.  Allocates device memory for the masks
 * (kept until the next call or b200bsp_destroy).  MI with ROIs runs on the
 * FP32 tile passes in either form. */
int b200bsp_set_roi (b200bsp_ctx* ctx, const b200bsp_volume* fixed_roi,
    const uint8_t* fixed_mask, const b200bsp_volume* moving_roi,
    const uint8_t* moving_mask);

/* The landmark term alone, bspline_landmarks_score_a
 * (src/register/bspline_landmarks.cxx:25-134): lmetric = the mean squared
 * distance between the moving landmarks and the fixed landmarks carried by
 * the field; ADDS its gradient (stiffness / n times the residual, spread
 * over the landmark's 64 knots) into grad, as the reference adds into
 * total_grad (grad may be NULL).  Float arithmetic in the reference's
 * order: results equal the reference's bit for bit. */
int b200bsp_landmarks_score (b200bsp_ctx* ctx, const float* coeff,
    float* lmetric, float* grad);

/* Mattes MI split into its two passes, for one volume split into slabs
 * across GPUs (no reference counterpart): each slab's context has the whole
 * images and the slab as its ROI.  b200bsp_mi_hist runs pass 1 over the
 * ROI and returns the histograms as exact integers -- hist[0..B) fixed,
 * [B..2B) moving, [2B..2B+B*B) joint (PVI-8 weights in 2^-24 units; the
 * Parzen form fills the joint part only), hist[2B+B*B] the voxel count -- so
 * the slabs' histograms add up exactly to the whole ROI's.
 * b200bsp_mi_grad takes such summed histograms, returns the score they give
 * and this ROI's part of the gradient in double (the slabs' parts add up to
 * the whole gradient).  Neither call checks that the ROI is the whole image:
 * the caller's slabs must tile it. */
int b200bsp_mi_hist (b200bsp_ctx* ctx, const float* coeff, int64_t* hist);
int b200bsp_mi_grad (b200bsp_ctx* ctx, const float* coeff,
    const int64_t* hist, float* score, double* grad, int64_t* num_vox);

/* Autotuner (no reference counterpart): times `evals` MSE evaluations at
 * `coeff` for each way the tensor-core kernel may split a row of tiles
 * into batches (the fewest batches of at most 26 tiles, and up to two
 * more) and keeps the fastest for the context's later calls; *tiles
 * receives its tiles per batch (1 for the FP32 form, which has nothing to
 * tune).  Results stay within the parity bars whatever the split, and are
 * deterministic for a given split. */
int b200bsp_autotune (b200bsp_ctx* ctx, const float* coeff, int evals,
    int* tiles);

/* The MSE kernel the context's next evaluation runs: *kernel receives
 * B200BSP_TC_KERNEL_XLANE or _TILE (AUTO never; 0 for the FP32 form),
 * *tiles its tiles per batch and *batches the batches it launches. */
int b200bsp_mse_kernel (const b200bsp_ctx* ctx, int* kernel, int* tiles,
    int* batches);

/* Dense displacement field over the ROI (bspline_interpolate_vf,
 * src/base/bspline_interpolate.cxx:112-142): vf is dim[0]*dim[1]*dim[2]*3
 * floats of the fixed image, xyz interleaved; voxels outside the ROI are
 * zero.  coeff and vf may be host or device memory; with a host vf the
 * first call allocates a device staging buffer of 12 bytes per fixed voxel,
 * kept until b200bsp_destroy. */
int b200bsp_interpolate_vf (b200bsp_ctx* ctx, const float* coeff, float* vf);

/* Warp the moving image onto the fixed grid with trilinear interpolation
 * and `default_value` outside (bspline_warp with linear interpolation,
 * src/base/bspline_warp.cxx:28-227; no vector-field output).  The reference
 * takes each voxel's tile from its absolute index, so the warp is defined
 * when the grid's ROI is the whole fixed image: B200BSP_E_UNSUPPORTED
 * otherwise.  Host or device pointers; a host `warped` uses the staging
 * buffer of b200bsp_interpolate_vf. */
int b200bsp_warp (b200bsp_ctx* ctx, const float* coeff, float default_value,
    float* warped);

/* Moving-image gradient alone (volume_calc_grad,
 * src/base/volume_grad.cxx:9-76) for an arbitrary volume. */
int b200bsp_volume_grad (const b200bsp_volume* vol, const float* img,
    float* grad_out, int device);

/* Turn per-evaluation device timing (CUDA events on the context's stream)
 * on or off; off by default. */
int b200bsp_enable_timing (b200bsp_ctx* ctx, int on);

/* Device time of the last evaluation in milliseconds (all its kernels and
 * copies, from the first launch to the last), and the number of kernel
 * launches it made.  Needs timing enabled. */
int b200bsp_last_timing (const b200bsp_ctx* ctx, float* ms, int* launches);

/* Device time of the last evaluation's main tile kernel alone (ms). */
int b200bsp_last_main_ms (const b200bsp_ctx* ctx, float* ms);

/* Resample types of registration_resample_volume
 * (src/register/registration_resample.cxx:12-59). */
#define B200BSP_RESAMPLE_VOXEL         0  /* rate = voxels per output voxel */
#define B200BSP_RESAMPLE_VOXEL_LEGACY  1  /* same, legacy_subsampling grid */
#define B200BSP_RESAMPLE_MM            2  /* rate = output spacing (mm) */
#define B200BSP_RESAMPLE_PERCENT       3  /* rate = fraction of the voxels */

/* The output grid of one pyramid level: volume_subsample_vox,
 * volume_subsample_vox_legacy, volume_resample_spacing or
 * volume_resample_percent (src/base/volume_resample.cxx:297-413) by type.
 * out keeps in's direction cosines.  *is_copy (may be NULL) is 1 when the
 * reference clones the input instead (voxel types, rate 1 on every axis).
 * Host only. */
int b200bsp_resample_geometry (const b200bsp_volume* in, int type,
    const float rate[3], b200bsp_volume* out, int* is_copy);

/* Trilinear resampling of a float image onto the grid `out`
 * (volume_resample_float_li, src/base/volume_resample.cxx:70-136):
 * positions step by out's spacing from out's origin, direction cosines are
 * not used (as in the reference), voxels whose rounded input index lies
 * outside the input are 0.  Bit-identical to the reference.  Images may be
 * host or device memory; allocates temporary device buffers and waits for
 * the result. */
int b200bsp_resample (const b200bsp_volume* in, const float* in_img,
    const b200bsp_volume* out, float* out_img, int device);

/* Save the grid over `fixed` with its coefficients in the reference's
 * B-spline coefficient file format (Bspline_xform::save,
 * src/base/bspline_xform.cxx:101-148); Plastimatch reads the file back with
 * bspline_xform_load.  Host memory. */
int b200bsp_xform_save (const char* path, const b200bsp_volume* fixed,
    const b200bsp_grid* grid, const float* coeff);

/* Read a B-spline coefficient file (bspline_xform_load,
 * src/base/bspline_xform.cxx:150-279): the fixed image geometry, the grid
 * and num_coeff always; the coefficients (xyz interleaved per knot) when
 * coeff is non-NULL and coeff_cap >= num_coeff.  Host memory. */
int b200bsp_xform_load (const char* path, b200bsp_volume* fixed,
    b200bsp_grid* grid, float* coeff, int64_t coeff_cap, int64_t* num_coeff);

/* Write a float image (channels 1) or an interleaved vector field
 * (channels 3) as MetaImage, byte for byte as write_mha
 * (src/base/mha_io.cxx:25-103).  Host memory. */
int b200bsp_mha_write (const char* path, const b200bsp_volume* geom,
    int channels, const float* data);

/* Read a MetaImage as read_mha does (src/base/mha_io.cxx:105-241): float,
 * short or unsigned char samples, either byte order, converted to float;
 * `channels` is 3 for a vector field.  With data NULL only the header is
 * read; otherwise cap (floats) must hold dim[0]*dim[1]*dim[2]*channels.
 * Host memory. */
int b200bsp_mha_read (const char* path, b200bsp_volume* geom, int* channels,
    float* data, int64_t cap);

/* Limited-memory BFGS: the optimiser of Plastimatch's "liblbfgs"
 * implementation (src/register/bspline_optimize_liblbfgs.cxx:20-117 with
 * liblbfgs' default parameters), restated from the published methods:
 * two-loop recursion over m correction pairs and the More-Thuente line
 * search.  Vectors stay in device memory (double). */
typedef struct {
    int m;                /* correction pairs kept (6) */
    double epsilon;       /* stop when ||g|| / max(1, ||x||) <= epsilon (1e-5) */
    int max_its;          /* stop after iteration k > max_its (Bspline_parms, 10) */
    int max_feval;        /* ... or after more evaluations than this (10) */
    int max_linesearch;   /* trials per line search (40) */
    double min_step, max_step;   /* 1e-20, 1e20 */
    double ftol;          /* sufficient decrease (1e-4) */
    double gtol;          /* curvature, strong Wolfe (0.9) */
    double xtol;          /* relative interval width (1e-16) */
} b200bsp_lbfgs_parms;

/* status values */
#define B200BSP_LBFGS_CONVERGED          0   /* gradient test met */
#define B200BSP_LBFGS_STOPPED            1   /* max_its / max_feval reached */
#define B200BSP_LBFGS_ALREADY_MINIMIZED  2   /* gradient test met at x0 */
/* negative: the line search failed (rounding, step limits, trial count);
 * x is the last accepted point */

typedef struct {
    int status;
    int iterations;       /* line searches completed */
    int fevals;           /* function evaluations */
    double score;         /* objective at the returned x */
} b200bsp_lbfgs_result;

/* Fill parms with the defaults above. */
void b200bsp_lbfgs_default_parms (b200bsp_lbfgs_parms* parms);

/* Optimise the coefficients of the context's registration: the objective is
 * bspline_score() -- lambda * metric (0 MSE, 1 MI) plus the analytic
 * regulariser when reg is non-NULL -- evaluated on the device.  coeff (host
 * or device) holds x0 on entry; on return it holds what Plastimatch's
 * transform holds after its optimiser: the last evaluated coefficients
 * (a stop inside a line search leaves the last trial point there), and
 * res->score the last evaluated total score.  The first run on a context
 * allocates the optimiser's device vectors ((2m + 5) doubles and 2 floats
 * per coefficient); the context keeps them for later runs with the same m
 * and frees them with itself. */
int b200bsp_optimize_lbfgs (b200bsp_ctx* ctx, int metric_type, float lambda,
    const b200bsp_reg_parms* reg, const b200bsp_lbfgs_parms* parms,
    float* coeff, b200bsp_lbfgs_result* res);

/* The same optimiser on a caller's function: fn receives host copies of x
 * (n doubles) and writes the gradient to g, returning f.  x (host) holds x0
 * on entry and the last accepted point on return (res->score its value). */
typedef double (*b200bsp_eval_fn) (void* user, const double* x, double* g,
    int64_t n);
int b200bsp_lbfgs_minimize (int64_t n, double* x, b200bsp_eval_fn fn,
    void* user, const b200bsp_lbfgs_parms* parms, b200bsp_lbfgs_result* res,
    int device);

/* Largest tile count b200bsp_score_mse_static accepts (its fixed scratch:
 * about 6.4 MB of static device memory per device). */
#define B200BSP_STATIC_MAX_TILES 8192

/* No counterpart in the reference.  MSE score and gradient as
 * b200bsp_score_mse with the FP32 form, for callers that may not allocate
 * device memory: no context, no allocation; partial sums live in one
 * static device array of the library.  All pointers are device memory on
 * the current device (moving_grad only for B200BSP_MSE_GRAD_NEAREST;
 * score and num_vox may be NULL); the call is ordered on `stream` and
 * returns without waiting.  Grids of more than B200BSP_STATIC_MAX_TILES
 * tiles are rejected (B200BSP_E_UNSUPPORTED).  Every call looks up the
 * array's address in the current context (the first one on a device also
 * loads the library's module there); make the first call before any
 * stream capture.  A CUDA error already pending when the call starts is
 * reported (B200BSP_E_CUDA) and left pending.  Calls whose device work
 * overlaps race on the shared array: issue them on one stream.  Errors
 * are reported through b200bsp_last_error (NULL).  The whole fixed image
 * is the ROI: this entry point takes no fixed or moving ROI mask (a masked
 * registration, the reference's inside_roi test, needs a context and
 * b200bsp_set_roi). */
int b200bsp_score_mse_static (const b200bsp_volume* fixed,
    const b200bsp_volume* moving, const b200bsp_grid* grid, int mse_grad,
    const float* fixed_img, const float* moving_img, const float* moving_grad,
    const float* coeff, float* score, float* grad, int64_t* num_vox,
    void* stream);

/* Text of the last error on this context (or the last create failure when
 * ctx is NULL). */
const char* b200bsp_last_error (const b200bsp_ctx* ctx);

/* ---- batched registrations (no reference counterpart) ----------------
 *
 * A batch groups contexts on one device (uneven volume sizes and grids) so
 * that one CUDA graph launch evaluates all of them (each context's tile
 * pass and finish kernel run on a branch of the graph), and so that their
 * registrations run at once.  The kernels of different contexts take the
 * SMs as they free up.  The Plastimatch counterpart is one registration
 * per process, run one after another. */
typedef struct b200bsp_batch b200bsp_batch;

/* The contexts must be distinct, on one device, with images set; the batch
 * does not own them (destroy it before them). */
int b200bsp_batch_create (b200bsp_ctx* const* ctxs, int n,
    b200bsp_batch** out);
void b200bsp_batch_destroy (b200bsp_batch* batch);
const char* b200bsp_batch_last_error (const b200bsp_batch* batch);

/* MSE score + gradient of every context in one graph launch; coeffs[i],
 * grads[i] (num_coeff floats of context i), scores (n floats) and num_vox
 * (n int64, may be NULL) are device memory.  Blocks until done.  The graph
 * is captured on the first call with a given set of buffers and replayed
 * after that. */
int b200bsp_batch_score_mse (b200bsp_batch* batch, const float* const* coeffs,
    float* const* grads, float* scores, int64_t* num_vox);

/* One L-BFGS registration per context (MSE, similarity weight lambda, no
 * regulariser), all advancing together: each runs b200bsp_optimize_lbfgs's
 * graph-resident optimiser on its context's stream, all at once, so no
 * registration waits for another.  Each follows b200bsp_optimize_lbfgs's
 * trial sequence; coeffs[i] (host or device) holds its start and receives
 * its result, results[i] its status. */
int b200bsp_batch_optimize_lbfgs (b200bsp_batch* batch, float lambda,
    const b200bsp_lbfgs_parms* parms, float* const* coeffs,
    b200bsp_lbfgs_result* results);

#ifdef __cplusplus
}
#endif
#endif
