/* C-ABI driver around Plastimatch's own B-spline cost function, compiled
 * from the reference sources as a CPU oracle (oracle/_ref/libplmref.so).
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/ as the parity checker and by
 * bench.py's reference / cpu_baseline arm.  The product never links it.
 *
 * Each entry point builds the reference's own objects (Volume,
 * Bspline_xform, Bspline_parms, Bspline_state, Bspline_optimize,
 * Metric_state) exactly as Bspline_optimize::optimize() does
 * (src/register/bspline_optimize.cxx:122-153) and then calls the reference
 * flavour function that the caller names, so the numbers are the
 * reference's numbers. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>
#include <fcntl.h>
#include <omp.h>

#include "bspline.h"
#include "bspline_interpolate.h"
#include "bspline_landmarks.h"
#include "bspline_mi.h"
#include "bspline_mse.h"
#include "bspline_optimize.h"
#include "bspline_parms.h"
#include "bspline_regularize.h"
#include "bspline_state.h"
#include "bspline_warp.h"
#include "bspline_xform.h"
#include "joint_histogram.h"
#include "mha_io.h"
#include "metric_state.h"
#include "pointset.h"
#include "regularization_parms.h"
#include "volume.h"
#include "volume_grad.h"
#include "volume_resample.h"

extern "C" {

/* Geometry of one volume: dim, origin (mm), spacing (mm), direction
 * cosines (row-major 3x3), as the reference's Volume constructor takes
 * them (src/base/volume.h:60-67). */
typedef struct {
    int64_t dim[3];
    float origin[3];
    float spacing[3];
    float dcos[9];
} ref_geom;

/* B-spline grid: the arguments of Bspline_xform::initialize
 * (src/base/bspline_xform.cxx:491-507). */
typedef struct {
    int64_t roi_offset[3];
    int64_t roi_dim[3];
    int64_t vox_per_rgn[3];
} ref_grid;

typedef struct {
    float score;            /* bst->ssd.curr_smetric (or total_score) */
    float total_score;      /* bst->ssd.total_score after bspline_score */
    float rmetric;          /* bst->ssd.rmetric */
    int64_t num_vox;        /* bst->ssd.curr_num_vox */
    int64_t num_coeff;
    /* MI only: the joint histogram the flavour built (double) */
    int64_t fixed_bins, moving_bins;
    float f_offset, f_delta, m_offset, m_delta;
} ref_result;

}

/* The reference logs every step to stdout (src/sys/logfile.cxx:45-62);
 * keep the checker quiet by pointing fd 1 at /dev/null for the call. */
class Quiet {
public:
    int saved;
    Quiet () {
        fflush (stdout);
        saved = dup (1);
        int fd = open ("/dev/null", O_WRONLY);
        dup2 (fd, 1);
        close (fd);
    }
    ~Quiet () {
        fflush (stdout);
        dup2 (saved, 1);
        close (saved);
    }
};

static Volume::Pointer
make_volume (const ref_geom* g, const float* img, int planes)
{
    Volume::Pointer v = Volume::New (
        g->dim, g->origin, g->spacing, g->dcos,
        planes == 1 ? PT_FLOAT : PT_VF_FLOAT_INTERLEAVED, planes);
    memcpy (v->img, img, sizeof(float) * planes * v->npix);
    return v;
}

/* Landmark pairs (points in mm) and their stiffness. */
struct Ref_landmarks {
    const float* fixed_xyz;
    const float* moving_xyz;
    int64_t n;
    float stiffness;
};

/* Histogram type of the next MI setups (Bspline_parms::mi_hist_type). */
static Mi_hist_type g_hist_type = HIST_EQSP;

extern "C" void
ref_set_mi_hist_type (int vopt)
{
    g_hist_type = vopt ? HIST_VOPT : HIST_EQSP;
}

struct Ref_setup {
    Labeled_pointset lm_fixed, lm_moving;
    Bspline_xform bxf;
    Bspline_parms parms;
    Regularization_parms rparms;
    Bspline_optimize bod;
    Metric_state::Pointer ms;
};

static void
setup (Ref_setup* s, const ref_geom* fg, const float* fimg,
    const ref_geom* mg, const float* mimg, const float* mgrad,
    const ref_grid* grid, const float* coeff, char flavor,
    int metric_mi, int bins, char reg_impl, float reg_lambda,
    int threads, const Ref_landmarks* lm = 0)
{
    if (threads > 0) omp_set_num_threads (threads);
    float origin[3], spacing[3];
    plm_long dim[3], roi_offset[3], roi_dim[3], vpr[3];
    for (int d = 0; d < 3; d++) {
        origin[d] = fg->origin[d];
        spacing[d] = fg->spacing[d];
        dim[d] = fg->dim[d];
        roi_offset[d] = grid->roi_offset[d];
        roi_dim[d] = grid->roi_dim[d];
        vpr[d] = grid->vox_per_rgn[d];
    }
    float dcos[9];
    memcpy (dcos, fg->dcos, sizeof dcos);
    s->bxf.initialize (origin, spacing, dim, roi_offset, roi_dim, vpr, dcos);
    if (coeff) {
        memcpy (s->bxf.coeff, coeff, sizeof(float) * s->bxf.num_coeff);
    }

    s->parms.threading = BTHR_CPU;
    s->parms.implementation = flavor;
    s->parms.mi_hist_fixed_bins = bins;
    s->parms.mi_hist_moving_bins = bins;
    s->parms.mi_hist_type = g_hist_type;
    s->rparms.implementation = reg_impl;
    s->rparms.curvature_penalty = reg_lambda;
    s->parms.regularization_parms = &s->rparms;

    if (lm && lm->n > 0) {
        /* as bspline_stage.cxx:318-329 sets them up before the state's
           initialize() computes their grid coordinates */
        for (int64_t l = 0; l < lm->n; l++) {
            s->lm_fixed.insert_lps ("", lm->fixed_xyz[3*l],
                lm->fixed_xyz[3*l+1], lm->fixed_xyz[3*l+2]);
            s->lm_moving.insert_lps ("", lm->moving_xyz[3*l],
                lm->moving_xyz[3*l+1], lm->moving_xyz[3*l+2]);
        }
        s->parms.blm->set_landmarks (&s->lm_fixed, &s->lm_moving);
        s->parms.blm->landmark_stiffness = lm->stiffness;
    }

    s->bod.set_bspline_parms (&s->parms);
    s->bod.set_bspline_xform (&s->bxf);
    Bspline_state* bst = s->bod.get_bspline_state ();

    if (fimg) {
        s->ms = Metric_state::New ();
        s->ms->fixed_ss = make_volume (fg, fimg, 1);
        s->ms->moving_ss = make_volume (mg, mimg, 1);
        if (mgrad) {
            s->ms->moving_grad = make_volume (mg, mgrad, 3);
        } else {
            s->ms->moving_grad = volume_gradient (s->ms->moving_ss);
        }
        s->ms->metric_type = metric_mi
            ? SIMILARITY_METRIC_MI_MATTES : SIMILARITY_METRIC_MSE;
        s->ms->metric_lambda = 1.0f;
        bst->similarity_data.push_back (s->ms);
    }
    bst->initialize (&s->bxf, &s->parms);
    if (fimg) {
        bst->initialize_mi_histograms ();
        bst->set_metric_state (s->ms);
    }
}

extern "C" {

/* One similarity-metric evaluation with the named flavour, exactly as the
 * metric loop of bspline_score() runs it (src/register/bspline.cxx:575-616):
 * reset_score, set_metric_state, bspline_score_mse/_mi.  Writes
 * curr_smetric, curr_smetric_grad and curr_num_vox.  For MI, also the
 * histograms (f_hist[bins], m_hist[bins], j_hist[bins*bins], double). */
int
ref_metric (const ref_geom* fg, const float* fimg,
    const ref_geom* mg, const float* mimg, const float* mgrad,
    const ref_grid* grid, const float* coeff, char flavor, int metric_mi,
    int bins, int threads, float* grad, ref_result* res,
    double* f_hist, double* m_hist, double* j_hist)
{
    Quiet q;
    Ref_setup s;
    setup (&s, fg, fimg, mg, mimg, mgrad, grid, coeff, flavor, metric_mi,
        bins, '\0', 0.f, threads);
    Bspline_state* bst = s.bod.get_bspline_state ();
    bst->ssd.reset_score ();
    if (metric_mi) {
        bspline_score_mi (&s.bod);
    } else {
        bspline_score_mse (&s.bod);
    }
    res->score = bst->ssd.curr_smetric;
    res->num_vox = bst->ssd.curr_num_vox;
    res->num_coeff = s.bxf.num_coeff;
    memcpy (grad, bst->ssd.curr_smetric_grad, sizeof(float) * s.bxf.num_coeff);
    if (metric_mi) {
        Joint_histogram* jh = bst->get_mi_hist ();
        res->fixed_bins = jh->fixed.bins;
        res->moving_bins = jh->moving.bins;
        res->f_offset = jh->fixed.offset;
        res->f_delta = jh->fixed.delta;
        res->m_offset = jh->moving.offset;
        res->m_delta = jh->moving.delta;
        if (f_hist) memcpy (f_hist, jh->f_hist, sizeof(double) * jh->fixed.bins);
        if (m_hist) memcpy (m_hist, jh->m_hist, sizeof(double) * jh->moving.bins);
        if (j_hist) memcpy (j_hist, jh->j_hist,
            sizeof(double) * jh->fixed.bins * jh->moving.bins);
    }
    return 0;
}

/* ref_metric with image ROIs: uchar mask volumes (x fastest, any
 * geometry; NULL: none) set on the metric state as a registration stage
 * does (src/register/bspline_stage.cxx:152-205), so the dispatchers route
 * MSE to flavour i (or k for 'c'/'k') and MI to flavour h
 * (bspline_mse.cxx:1879-1887, bspline_mi.cxx:3036-3055). */
int
ref_metric_roi (const ref_geom* fg, const float* fimg,
    const ref_geom* mg, const float* mimg, const float* mgrad,
    const ref_grid* grid, const float* coeff, char flavor, int metric_mi,
    int bins, int threads, const ref_geom* frg, const unsigned char* froi,
    const ref_geom* mrg, const unsigned char* mroi, float* grad,
    ref_result* res, double* f_hist, double* m_hist, double* j_hist)
{
    Quiet q;
    Ref_setup s;
    setup (&s, fg, fimg, mg, mimg, mgrad, grid, coeff, flavor, metric_mi,
        bins, '\0', 0.f, threads);
    Bspline_state* bst = s.bod.get_bspline_state ();
    if (froi) {
        s.ms->fixed_roi = Volume::New (frg->dim, frg->origin, frg->spacing,
            frg->dcos, PT_UCHAR, 1);
        memcpy (s.ms->fixed_roi->img, froi, s.ms->fixed_roi->npix);
    }
    if (mroi) {
        s.ms->moving_roi = Volume::New (mrg->dim, mrg->origin, mrg->spacing,
            mrg->dcos, PT_UCHAR, 1);
        memcpy (s.ms->moving_roi->img, mroi, s.ms->moving_roi->npix);
    }
    bst->set_metric_state (s.ms);
    bst->ssd.reset_score ();
    if (metric_mi) {
        bspline_score_mi (&s.bod);
    } else {
        bspline_score_mse (&s.bod);
    }
    res->score = bst->ssd.curr_smetric;
    res->num_vox = bst->ssd.curr_num_vox;
    res->num_coeff = s.bxf.num_coeff;
    memcpy (grad, bst->ssd.curr_smetric_grad, sizeof(float) * s.bxf.num_coeff);
    if (metric_mi) {
        Joint_histogram* jh = bst->get_mi_hist ();
        res->fixed_bins = jh->fixed.bins;
        res->moving_bins = jh->moving.bins;
        res->f_offset = jh->fixed.offset;
        res->f_delta = jh->fixed.delta;
        res->m_offset = jh->moving.offset;
        res->m_delta = jh->moving.delta;
        if (f_hist) memcpy (f_hist, jh->f_hist, sizeof(double) * jh->fixed.bins);
        if (m_hist) memcpy (m_hist, jh->m_hist, sizeof(double) * jh->moving.bins);
        if (j_hist) memcpy (j_hist, jh->j_hist,
            sizeof(double) * jh->fixed.bins * jh->moving.bins);
    }
    return 0;
}

/* The analytic regulariser alone (flavour 'b' serial or 'c' OpenMP):
 * Bspline_regularize::compute_score into a freshly reset Bspline_score
 * (src/register/bspline_regularize.cxx:95-126).  Writes rmetric and the
 * regulariser's contribution to total_grad. */
int
ref_regularize (const ref_geom* fg, const ref_grid* grid, const float* coeff,
    char reg_impl, float curvature_penalty, int threads, float* grad,
    ref_result* res)
{
    Quiet q;
    Ref_setup s;
    setup (&s, fg, 0, 0, 0, 0, grid, coeff, 'g', 0, 32, reg_impl,
        curvature_penalty, threads);
    Bspline_state* bst = s.bod.get_bspline_state ();
    bst->ssd.reset_score ();
    bst->rst.compute_score (&bst->ssd, &s.rparms, &s.bxf);
    res->rmetric = bst->ssd.rmetric;
    res->num_coeff = s.bxf.num_coeff;
    memcpy (grad, bst->ssd.total_grad, sizeof(float) * s.bxf.num_coeff);
    return 0;
}

/* The whole cost function: bspline_score() (src/register/bspline.cxx:
 * 558-632) with one MSE or MI metric and, when reg_impl != 0, the analytic
 * regulariser.  Writes total_score and total_grad. */
int
ref_score (const ref_geom* fg, const float* fimg,
    const ref_geom* mg, const float* mimg, const float* mgrad,
    const ref_grid* grid, const float* coeff, char flavor, int metric_mi,
    int bins, char reg_impl, float curvature_penalty, int threads,
    float* grad, ref_result* res)
{
    Quiet q;
    Ref_setup s;
    setup (&s, fg, fimg, mg, mimg, mgrad, grid, coeff, flavor, metric_mi,
        bins, reg_impl, curvature_penalty, threads);
    Bspline_state* bst = s.bod.get_bspline_state ();
    bspline_score (&s.bod);
    res->total_score = bst->ssd.total_score;
    res->rmetric = bst->ssd.rmetric;
    res->num_coeff = s.bxf.num_coeff;
    res->score = bst->ssd.metric_record.empty ()
        ? 0.f : bst->ssd.metric_record[0].score;
    memcpy (grad, bst->ssd.total_grad, sizeof(float) * s.bxf.num_coeff);
    return 0;
}

/* The landmark term alone: Bspline_landmarks::initialize through the
 * state's initialize(), then bspline_landmarks_score
 * (src/register/bspline_landmarks.cxx:25-145) into a freshly reset
 * Bspline_score.  Writes lmetric (in res->score) and total_grad. */
int
ref_landmarks (const ref_geom* fg, const ref_grid* grid, const float* coeff,
    const float* fixed_xyz, const float* moving_xyz, int64_t n,
    float stiffness, float* grad, ref_result* res)
{
    Quiet q;
    Ref_setup s;
    Ref_landmarks lm = {fixed_xyz, moving_xyz, n, stiffness};
    setup (&s, fg, 0, 0, 0, 0, grid, coeff, 'g', 0, 32, '\0', 0.f, 0, &lm);
    Bspline_state* bst = s.bod.get_bspline_state ();
    bst->ssd.reset_score ();
    bspline_landmarks_score (&s.parms, bst, &s.bxf);
    res->score = bst->ssd.lmetric;
    res->num_coeff = s.bxf.num_coeff;
    memcpy (grad, bst->ssd.total_grad, sizeof(float) * s.bxf.num_coeff);
    return 0;
}

/* bspline_score() as ref_score, with landmark pairs as well. */
int
ref_score_landmarks (const ref_geom* fg, const float* fimg,
    const ref_geom* mg, const float* mimg, const ref_grid* grid,
    const float* coeff, char flavor, int metric_mi, int bins, char reg_impl,
    float curvature_penalty, const float* fixed_xyz, const float* moving_xyz,
    int64_t n, float stiffness, int threads, float* grad, ref_result* res)
{
    Quiet q;
    Ref_setup s;
    Ref_landmarks lm = {fixed_xyz, moving_xyz, n, stiffness};
    setup (&s, fg, fimg, mg, mimg, 0, grid, coeff, flavor, metric_mi, bins,
        reg_impl, curvature_penalty, threads, &lm);
    Bspline_state* bst = s.bod.get_bspline_state ();
    bspline_score (&s.bod);
    res->total_score = bst->ssd.total_score;
    res->rmetric = bst->ssd.rmetric;
    res->num_coeff = s.bxf.num_coeff;
    res->score = bst->ssd.metric_record.empty ()
        ? 0.f : bst->ssd.metric_record[0].score;
    memcpy (grad, bst->ssd.total_grad, sizeof(float) * s.bxf.num_coeff);
    return 0;
}

/* volume_gradient() (src/base/volume_grad.cxx:9-76): central-difference
 * moving-image gradient, interleaved xyz. */
int
ref_volume_grad (const ref_geom* g, const float* img, float* grad_out)
{
    Quiet q;
    Volume::Pointer v = make_volume (g, img, 1);
    Volume::Pointer gr = volume_gradient (v);
    memcpy (grad_out, gr->img, sizeof(float) * 3 * gr->npix);
    return 0;
}

static void
init_xform (Bspline_xform* bxf, const ref_geom* fg, const ref_grid* grid,
    const float* coeff)
{
    float origin[3], spacing[3], dcos[9];
    plm_long dim[3], roi_offset[3], roi_dim[3], vpr[3];
    for (int d = 0; d < 3; d++) {
        origin[d] = fg->origin[d]; spacing[d] = fg->spacing[d];
        dim[d] = fg->dim[d]; roi_offset[d] = grid->roi_offset[d];
        roi_dim[d] = grid->roi_dim[d]; vpr[d] = grid->vox_per_rgn[d];
    }
    memcpy (dcos, fg->dcos, sizeof dcos);
    bxf->initialize (origin, spacing, dim, roi_offset, roi_dim, vpr, dcos);
    if (coeff) memcpy (bxf->coeff, coeff, sizeof(float) * bxf->num_coeff);
}

/* bspline_interpolate_vf (src/base/bspline_interpolate.cxx:112-142) into a
 * vector-field volume over the fixed image (xyz interleaved). */
int
ref_interpolate_vf (const ref_geom* fg, const ref_grid* grid,
    const float* coeff, float* vf)
{
    Quiet q;
    Bspline_xform bxf;
    init_xform (&bxf, fg, grid, coeff);
    Volume::Pointer v = Volume::New (fg->dim, fg->origin, fg->spacing,
        fg->dcos, PT_VF_FLOAT_INTERLEAVED, 3);
    bspline_interpolate_vf (v.get (), &bxf);
    memcpy (vf, v->img, sizeof(float) * 3 * v->npix);
    return 0;
}

/* bspline_warp (src/base/bspline_warp.cxx:162-227) of a float moving image
 * onto the fixed grid; vf_out (may be NULL) receives the field. */
int
ref_warp (const ref_geom* fg, const ref_geom* mg, const float* mimg,
    const ref_grid* grid, const float* coeff, int linear, float default_val,
    float* out, float* vf_out)
{
    Quiet q;
    Bspline_xform bxf;
    init_xform (&bxf, fg, grid, coeff);
    Volume::Pointer moving = make_volume (mg, mimg, 1);
    Volume::Pointer vout = Volume::New (fg->dim, fg->origin, fg->spacing,
        fg->dcos, PT_FLOAT, 1);
    Volume::Pointer vf;
    if (vf_out) {
        vf = Volume::New (fg->dim, fg->origin, fg->spacing, fg->dcos,
            PT_VF_FLOAT_INTERLEAVED, 3);
    }
    bspline_warp (vout.get (), vf ? vf.get () : 0, &bxf, moving.get (),
        linear, default_val);
    memcpy (out, vout->img, sizeof(float) * vout->npix);
    if (vf_out) memcpy (vf_out, vf->img, sizeof(float) * 3 * vf->npix);
    return 0;
}

/* The resampling step of registration_resample_volume
 * (src/register/registration_resample.cxx:12-59) for resample type mode
 * (0 voxel rate, 1 voxel rate legacy, 2 mm, 3 percent), on a float image.
 * Writes the output geometry; writes the image when out_cap (floats) is
 * large enough.  Returns the output voxel count. */
int64_t
ref_resample (const ref_geom* g, const float* img, int mode,
    const float rate[3], int64_t odim[3], float oorigin[3], float ospacing[3],
    float* out, int64_t out_cap)
{
    Quiet q;
    Volume::Pointer v = make_volume (g, img, 1);
    Volume::Pointer r;
    bool unit = rate[0] == 1.0f && rate[1] == 1.0f && rate[2] == 1.0f;
    if ((mode == 0 || mode == 1) && unit) r = v->clone ();
    else if (mode == 0) r = volume_subsample_vox (v, rate);
    else if (mode == 1) r = volume_subsample_vox_legacy (v, rate);
    else if (mode == 2) r = volume_resample_spacing (v, rate);
    else r = volume_resample_percent (v, rate);
    for (int d = 0; d < 3; d++) {
        odim[d] = r->dim[d];
        oorigin[d] = r->origin[d];
        ospacing[d] = r->spacing[d];
    }
    if (out && out_cap >= r->npix) {
        memcpy (out, r->img, sizeof(float) * r->npix);
    }
    return r->npix;
}

/* Plastimatch's optimiser loop (bspline_optimize, src/register/
 * bspline_optimize.cxx:122-153) with implementation "liblbfgs" and the
 * given iteration / evaluation limits: coeff holds x0 and receives the
 * result; res->total_score the last score bspline_score produced. */
int
ref_optimize (const ref_geom* fg, const float* fimg,
    const ref_geom* mg, const float* mimg, const float* mgrad,
    const ref_grid* grid, float* coeff, char flavor, int metric_mi, int bins,
    char reg_impl, float curvature_penalty, int max_its, int max_feval,
    int threads, ref_result* res)
{
    Quiet q;
    Ref_setup s;
    setup (&s, fg, fimg, mg, mimg, mgrad, grid, coeff, flavor, metric_mi,
        bins, reg_impl, curvature_penalty, threads);
    s.parms.optimization = BOPT_LIBLBFGS;
    s.parms.max_its = max_its;
    s.parms.max_feval = max_feval;
    Bspline_state* bst = s.bod.get_bspline_state ();
    s.bod.optimize ();
    memcpy (coeff, s.bxf.coeff, sizeof(float) * s.bxf.num_coeff);
    res->total_score = bst->ssd.total_score;
    res->num_vox = bst->feval;
    res->num_coeff = s.bxf.num_coeff;
    return bst->it;
}

/* Bspline_xform::save (src/base/bspline_xform.cxx:101-148) of the grid
 * over geometry fg with coefficients coeff. */
int
ref_xform_save (const char* path, const ref_geom* fg, const ref_grid* grid,
    const float* coeff)
{
    Quiet q;
    Bspline_xform bxf;
    init_xform (&bxf, fg, grid, coeff);
    bxf.save (path);
    return 0;
}

/* bspline_xform_load (src/base/bspline_xform.cxx:150-279): geometry, grid
 * and coefficients (coeff may be NULL: sizes only).  Returns num_coeff, or
 * -1 when the reference rejects the file. */
int64_t
ref_xform_load (const char* path, ref_geom* fg, ref_grid* grid, float* coeff,
    int64_t cap)
{
    Quiet q;
    Bspline_xform* bxf = bspline_xform_load (path);
    if (!bxf) return -1;
    const float* dc = bxf->dc.get_matrix ();
    for (int d = 0; d < 3; d++) {
        fg->dim[d] = bxf->img_dim[d];
        fg->origin[d] = bxf->img_origin[d];
        fg->spacing[d] = bxf->img_spacing[d];
        grid->roi_offset[d] = bxf->roi_offset[d];
        grid->roi_dim[d] = bxf->roi_dim[d];
        grid->vox_per_rgn[d] = bxf->vox_per_rgn[d];
    }
    for (int i = 0; i < 9; i++) fg->dcos[i] = dc[i];
    int64_t n = bxf->num_coeff;
    if (coeff && cap >= n) memcpy (coeff, bxf->coeff, sizeof(float) * n);
    delete bxf;
    return n;
}

/* write_mha (src/base/mha_io.cxx:25-103) of a float image (channels 1) or
 * an interleaved vector field (channels 3). */
int
ref_write_mha (const char* path, const ref_geom* g, int channels,
    const float* data)
{
    Quiet q;
    Volume::Pointer v = make_volume (g, data, channels);
    write_mha (path, v.get ());
    return 0;
}

/* read_mha (src/base/mha_io.cxx:105-241) converted to float: geometry,
 * channel count and data (data may be NULL: header only).  Returns the
 * voxel count, or -1 when the file cannot be read. */
int64_t
ref_read_mha (const char* path, ref_geom* g, int* channels, float* data,
    int64_t cap)
{
    Quiet q;
    Volume* v = read_mha (path);
    if (!v) return -1;
    for (int d = 0; d < 3; d++) {
        g->dim[d] = v->dim[d];
        g->origin[d] = v->origin[d];
        g->spacing[d] = v->spacing[d];
    }
    const float* dc = v->direction_cosines.get_matrix ();
    for (int i = 0; i < 9; i++) g->dcos[i] = dc[i];
    *channels = v->pix_type == PT_VF_FLOAT_INTERLEAVED ? 3 : 1;
    int64_t n = v->npix;
    if (data && cap >= n * *channels) {
        if (v->pix_type == PT_VF_FLOAT_INTERLEAVED || v->pix_type == PT_FLOAT) {
            memcpy (data, v->img, sizeof(float) * n * *channels);
        } else {
            v->convert (PT_FLOAT);
            memcpy (data, v->img, sizeof(float) * n);
        }
    }
    delete v;
    return n;
}

/* B-spline grid sizes the reference derives (Bspline_header::set,
 * src/base/bspline_header.cxx:28-62). */
int
ref_grid_dims (const ref_geom* fg, const ref_grid* grid, int64_t rdims[3],
    int64_t cdims[3], int64_t* num_coeff)
{
    Quiet q;
    Bspline_xform bxf;
    float origin[3], spacing[3], dcos[9];
    plm_long dim[3], roi_offset[3], roi_dim[3], vpr[3];
    for (int d = 0; d < 3; d++) {
        origin[d] = fg->origin[d]; spacing[d] = fg->spacing[d];
        dim[d] = fg->dim[d]; roi_offset[d] = grid->roi_offset[d];
        roi_dim[d] = grid->roi_dim[d]; vpr[d] = grid->vox_per_rgn[d];
    }
    memcpy (dcos, fg->dcos, sizeof dcos);
    bxf.initialize (origin, spacing, dim, roi_offset, roi_dim, vpr, dcos);
    for (int d = 0; d < 3; d++) {
        rdims[d] = bxf.rdims[d];
        cdims[d] = bxf.cdims[d];
    }
    *num_coeff = bxf.num_coeff;
    return 0;
}

/* The reference's basis lookup tables (Bspline_xform::allocate,
 * src/base/bspline_xform.cxx:361-488): bx/by/bz_lut [vpr*4] and
 * q_lut [vpr^3 * 64]. */
int
ref_luts (const ref_geom* fg, const ref_grid* grid, float* bx, float* by,
    float* bz, float* q_lut)
{
    Quiet q;
    Bspline_xform bxf;
    float origin[3], spacing[3], dcos[9];
    plm_long dim[3], roi_offset[3], roi_dim[3], vpr[3];
    for (int d = 0; d < 3; d++) {
        origin[d] = fg->origin[d]; spacing[d] = fg->spacing[d];
        dim[d] = fg->dim[d]; roi_offset[d] = grid->roi_offset[d];
        roi_dim[d] = grid->roi_dim[d]; vpr[d] = grid->vox_per_rgn[d];
    }
    memcpy (dcos, fg->dcos, sizeof dcos);
    bxf.initialize (origin, spacing, dim, roi_offset, roi_dim, vpr, dcos);
    memcpy (bx, bxf.bx_lut, sizeof(float) * 4 * vpr[0]);
    memcpy (by, bxf.by_lut, sizeof(float) * 4 * vpr[1]);
    memcpy (bz, bxf.bz_lut, sizeof(float) * 4 * vpr[2]);
    memcpy (q_lut, bxf.q_lut, sizeof(float) * 64 * vpr[0] * vpr[1] * vpr[2]);
    return 0;
}

}

/* L-BFGS-B comes from ITK's netlib port (v3p_netlib_setulb_), which is not
 * vendored with the reference; bspline_optimize.cxx still names it. */
extern "C" void
bspline_optimize_lbfgsb (Bspline_optimize*)
{
    fprintf (stderr, "oracle: reference L-BFGS-B is not available\n");
}
