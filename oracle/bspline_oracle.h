/* CPU restatement of Plastimatch's B-spline registration cost function.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA path is compared
 * against (tests/, __graft_entry__.smoke(), bench.py's cpu_baseline leg);
 * nothing in the product links or calls it.
 *
 * Each function restates one reference routine (file:line given at the
 * definition) in plain C.  The "_f32" entry points reproduce the
 * reference's float arithmetic in the reference's order (compile with
 * -ffp-contract=off), so on the same inputs they agree with the compiled
 * reference bit for bit up to the order of OpenMP reductions.  The "_f64"
 * entry points evaluate the same algorithm entirely in double precision and
 * serve as the error yardstick for the GPU forms. */
#ifndef BSPLINE_ORACLE_H
#define BSPLINE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Volume geometry; step/proj are filled by orc_vol_init. */
typedef struct {
    int64_t dim[3];
    float origin[3];
    float spacing[3];
    float dcos[9];
    float inv_dcos[9];
    float step[9];
    float proj[9];
} orc_vol;

/* B-spline grid over the fixed image (Bspline_header fields). */
typedef struct {
    float img_origin[3];
    float img_spacing[3];
    int64_t img_dim[3];
    int64_t roi_offset[3];
    int64_t roi_dim[3];
    int64_t vox_per_rgn[3];
    float grid_spac[3];
    int64_t rdims[3];
    int64_t cdims[3];
    int64_t num_knots;
    int64_t num_coeff;
} orc_grid;

/* MI histogram parameters (Histogram, EQSP). */
typedef struct {
    int64_t bins;
    float offset;
    float delta;
    /* V-optimal histograms (HIST_VOPT): offset/delta span `keys` fine
       keys and key_lut[key] gives the bin; NULL for equal spacing */
    int64_t keys;
    const int32_t* key_lut;
} orc_hist;

/* An image ROI: a uchar mask volume (x fastest) and its geometry
 * (Bspline_state::fixed_roi / moving_roi).  orc_set_roi makes the MSE and
 * MI routines test them (flavours i and h) until cleared with NULLs; the
 * pointers must stay valid meanwhile. */
typedef struct {
    orc_vol vol;
    const uint8_t* mask;
} orc_roi;
void orc_set_roi (const orc_roi* fixed_roi, const orc_roi* moving_roi);

int orc_vol_init (orc_vol* v, const int64_t dim[3], const float origin[3],
    const float spacing[3], const float dcos[9]);
int orc_grid_init (orc_grid* g, const orc_vol* fixed,
    const int64_t roi_offset[3], const int64_t roi_dim[3],
    const int64_t vox_per_rgn[3]);
void orc_basis_lut (float* lut, int64_t vpr);
void orc_q_lut (float* q_lut, const int64_t vpr[3]);

/* volume_calc_grad: central differences, interleaved xyz. */
void orc_volume_grad (const orc_vol* v, const float* img, float* grad);

/* MSE.  grad_mode 0: reference default flavours g/h/c (dc/dv from the
 * nearest-voxel moving gradient image); grad_mode 1: flavour o (exact
 * derivative of the trilinear interpolant, no moving gradient image). */
int orc_mse_f32 (const orc_grid* g, const orc_vol* fixed, const float* f_img,
    const orc_vol* moving, const float* m_img, const float* m_grad,
    const float* coeff, int grad_mode, float* score, float* grad,
    int64_t* num_vox);
int orc_mse_f64 (const orc_grid* g, const orc_vol* fixed, const float* f_img,
    const orc_vol* moving, const float* m_img, const float* m_grad,
    const float* coeff, int grad_mode, double* score, double* grad,
    int64_t* num_vox);

/* Mattes MI with PVI-8 histograms (flavour g). */
void orc_hist_eqsp (orc_hist* h, const float* img, int64_t n);
/* bspline_initialize_mi_hist_vopt (src/register/joint_histogram.cxx:
 * 195-324): 1000 fine keys over the value range and the bin of each key
 * (key_lut[1000], caller's buffer) chosen by the V-optimal dynamic
 * programme.  h->bins set by the caller (<= 1000). */
void orc_hist_vopt (orc_hist* h, int32_t* key_lut, const float* img,
    int64_t n);
int orc_mi_f32 (const orc_grid* g, const orc_vol* fixed, const float* f_img,
    const orc_vol* moving, const float* m_img, const float* coeff,
    const orc_hist* fh, const orc_hist* mh, float* score, float* grad,
    int64_t* num_vox, double* f_hist, double* m_hist, double* j_hist);
/* Mattes MI with cubic B-spline Parzen windows (no reference
 * implementation; restated from the published method, see the definition).
 * bins >= 5; the value range of each image is mapped with two padding bins
 * at either end. */
typedef struct {
    int64_t bins;
    float f_min, f_delta;    /* fixed: bin = floor((v - f_min) / f_delta) + 2 */
    float m_min, m_delta;    /* moving: window centre (v - m_min) / m_delta + 2 */
} orc_parzen;
void orc_parzen_init (orc_parzen* p, int64_t bins, const float* f_img,
    int64_t nf, const float* m_img, int64_t nm);
int orc_mi_parzen_f64 (const orc_grid* g, const orc_vol* fixed,
    const float* f_img, const orc_vol* moving, const float* m_img,
    const float* coeff, const orc_parzen* p, double* score, double* grad,
    int64_t* num_vox, double* jh);

int orc_mi_f64_pass1 (const orc_grid* g, const orc_vol* fixed,
    const float* f_img, const orc_vol* moving, const float* m_img,
    const float* coeff, const orc_hist* fhp, const orc_hist* mhp,
    int64_t* num_vox, double* fh, double* mh, double* jh);
int orc_mi_f64_pass2 (const orc_grid* g, const orc_vol* fixed,
    const float* f_img, const orc_vol* moving, const float* m_img,
    const float* coeff, const orc_hist* fhp, const orc_hist* mhp,
    int64_t num_vox, const double* fh, const double* mh, const double* jh,
    double* score, double* grad);
int orc_mi_f64 (const orc_grid* g, const orc_vol* fixed, const float* f_img,
    const orc_vol* moving, const float* m_img, const float* coeff,
    const orc_hist* fh, const orc_hist* mh, double* score, double* grad,
    int64_t* num_vox, double* f_hist, double* m_hist, double* j_hist);

/* Analytic regulariser (flavour c).  penalties[] = {curvature, diffusion,
 * lame_1, lame_2, total_displacement, third_order, linear_elastic_multiplier,
 * curvature_mixed_weight}. */
int orc_reg_f32 (const orc_grid* g, const float* coeff,
    const float penalties[8], float* rmetric, float* grad);
int orc_reg_f64 (const orc_grid* g, const float* coeff,
    const float penalties[8], double* rmetric, double* grad);

/* Landmarks.  orc_landmarks_init: the tile p[3n] and in-tile offset q[3n]
 * of each fixed landmark (Bspline_landmarks::initialize); returns the
 * index + 1 of the first landmark outside the fixed image, 0 when all lie
 * inside.  orc_landmarks_f32: bspline_landmarks_score_a in the reference's
 * float arithmetic, lmetric and the gradient ADDED into grad. */
int64_t orc_landmarks_init (const orc_grid* g, const orc_vol* fixed,
    const float* fixed_xyz, int64_t n, int64_t* p, int64_t* q);
void orc_landmarks_f32 (const orc_grid* g, const float* coeff, int64_t n,
    const float* fixed_xyz, const float* moving_xyz, const int64_t* p,
    const int64_t* q, float stiffness, float* lmetric, float* grad);

/* Dense vector field over the ROI (bspline_interpolate_vf) and the warped
 * moving image (bspline_warp, linear interpolation; ROI must be the whole
 * image, returns -2 otherwise). */
int orc_interpolate_vf (const orc_grid* g, const orc_vol* fixed,
    const float* coeff, float* vf);
int orc_warp (const orc_grid* g, const orc_vol* fixed, const orc_vol* moving,
    const float* m_img, const float* coeff, float default_val, float* out,
    float* vf_out);

/* Pyramid resampling: the output geometry of a resample type (0 voxel
 * rate, 1 voxel rate legacy, 2 mm, 3 percent; returns 1 for a plain copy)
 * and the trilinear resampler. */
int orc_resample_geometry (const int64_t dim[3], const float origin[3],
    const float spacing[3], int mode, const float rate[3],
    int64_t odim[3], float oorigin[3], float ospacing[3]);
void orc_resample_li (const int64_t idim[3], const float iorigin[3],
    const float ispacing[3], const float* in, const int64_t odim[3],
    const float oorigin[3], const float ospacing[3], float* out);

#ifdef __cplusplus
}
#endif
#endif
