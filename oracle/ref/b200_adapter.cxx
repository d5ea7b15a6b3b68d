/* The reference-side drop-in of plastimatch_b200, compiled against the
 * reference's own headers (oracle/build_ref.sh) and linked with both the
 * reference build (libplmref.so) and libplastimatch_b200.so.
 *
 * TEST INFRASTRUCTURE: it exists so that a test drives the library exactly
 * as a Plastimatch maintainer would wire it in -- the two functions below
 * are the ones INTEGRATION.md describes (bspline_b200_state_create at
 * Bspline_state's device-state hook, src/register/bspline_state.cxx:
 * 165-212, and the bspline_score_b200 flavour a BTHR_B200 case of
 * bspline_score_mse / bspline_score_mi would call, src/register/
 * bspline_mse.cxx:1876-1962, src/register/bspline_mi.cxx:3036-3141) -- and
 * compares them with the reference's CPU flavours on the same objects. */
#include <stdio.h>
#include <string.h>
#include <omp.h>

#include "bspline.h"
#include "bspline_mi.h"
#include "bspline_mse.h"
#include "bspline_optimize.h"
#include "bspline_parms.h"
#include "bspline_state.h"
#include "bspline_xform.h"
#include "metric_state.h"
#include "volume.h"
#include "volume_grad.h"

#include "../../include/plastimatch_b200.h"

/* ---- what a maintainer adds to Plastimatch -------------------------- */

static void
fill_volume (b200bsp_volume* v, const Volume* vol)
{
    for (int d = 0; d < 3; d++) {
        v->dim[d] = vol->dim[d];
        v->origin[d] = vol->origin[d];
        v->spacing[d] = vol->spacing[d];
    }
    for (int i = 0; i < 9; i++) v->dcos[i] = vol->direction_cosines[i];
}

/* At bspline_cuda_state_create's place: one context per stage, held in
 * Bspline_state::dev_ptrs.  Returns the library's status. */
static int
bspline_b200_state_create (Bspline_state* bst, Bspline_xform* bxf,
    Bspline_parms* parms, Volume* fixed, Volume* moving, Volume* moving_grad)
{
    b200bsp_volume f, m;
    fill_volume (&f, fixed);
    fill_volume (&m, moving);
    b200bsp_grid g;
    for (int d = 0; d < 3; d++) {
        g.roi_offset[d] = bxf->roi_offset[d];
        g.roi_dim[d] = bxf->roi_dim[d];
        g.vox_per_rgn[d] = bxf->vox_per_rgn[d];
    }
    b200bsp_opts o;
    b200bsp_default_opts (&o);
    o.mi_bins = parms->mi_hist_fixed_bins;
    o.mi_hist = parms->mi_hist_type == HIST_VOPT
        ? B200BSP_MI_HIST_VOPT : B200BSP_MI_HIST_EQSP;
    b200bsp_ctx* ctx = 0;
    int rc = b200bsp_create (&f, &m, &g, &o, &ctx);
    if (rc == B200BSP_OK) {
        rc = b200bsp_set_images (ctx, (float*) fixed->img,
            (float*) moving->img, moving_grad ? (float*) moving_grad->img : 0);
    }
    if (rc == B200BSP_OK && (bst->fixed_roi || bst->moving_roi)) {
        b200bsp_volume fr, mr;
        if (bst->fixed_roi) fill_volume (&fr, bst->fixed_roi);
        if (bst->moving_roi) fill_volume (&mr, bst->moving_roi);
        rc = b200bsp_set_roi (ctx,
            bst->fixed_roi ? &fr : 0,
            bst->fixed_roi ? (const uint8_t*) bst->fixed_roi->img : 0,
            bst->moving_roi ? &mr : 0,
            bst->moving_roi ? (const uint8_t*) bst->moving_roi->img : 0);
    }
    if (rc != B200BSP_OK) {
        fprintf (stderr, "b200: %s\n", b200bsp_last_error (ctx));
        b200bsp_destroy (ctx);
        return rc;
    }
    bst->dev_ptrs = ctx;
    return B200BSP_OK;
}

/* The BTHR_B200 flavour: writes the fields the CPU flavours write, so
 * bspline_score() lambda-accumulates and regularises as before. */
static int
bspline_score_b200 (Bspline_optimize* bod)
{
    Bspline_state* bst = bod->get_bspline_state ();
    Bspline_xform* bxf = bod->get_bspline_xform ();
    Bspline_score* ssd = &bst->ssd;
    b200bsp_ctx* ctx = (b200bsp_ctx*) bst->dev_ptrs;
    int64_t nvox = 0;
    int rc = bst->has_metric_type (SIMILARITY_METRIC_MI_MATTES)
        ? b200bsp_score_mi (ctx, bxf->coeff, &ssd->curr_smetric,
              ssd->curr_smetric_grad, &nvox, 0, 0, 0)
        : b200bsp_score_mse (ctx, bxf->coeff, &ssd->curr_smetric,
              ssd->curr_smetric_grad, &nvox);
    if (rc != B200BSP_OK) {
        fprintf (stderr, "b200: %s\n", b200bsp_last_error (ctx));
        return rc;
    }
    ssd->curr_num_vox = nvox;
    return B200BSP_OK;
}

/* ---- the test entry ------------------------------------------------- */

extern "C" {

typedef struct {
    int64_t dim[3];
    float origin[3];
    float spacing[3];
    float dcos[9];
} adapter_geom;

typedef struct {
    int64_t roi_offset[3];
    int64_t roi_dim[3];
    int64_t vox_per_rgn[3];
} adapter_grid;

/* Build the reference's objects as Bspline_optimize::optimize() does
 * (src/register/bspline_optimize.cxx:122-153), then score the same state
 * twice: through the adapter (out_b200) and through the reference's own
 * dispatcher bspline_score_mse / _mi with the CPU flavour `flavor`
 * (out_ref).  Each out block: score, num_vox, gradient[num_coeff].
 * Optional uchar ROI masks (geometry + mask, NULL for none) go onto the
 * metric state.  Returns 0, or the library's status. */
int
adapter_compare (const adapter_geom* fg, const float* fimg,
    const adapter_geom* mg, const float* mimg, const adapter_grid* grid,
    const float* coeff, char flavor, int metric_mi, int bins, int vopt,
    int threads, const adapter_geom* frg, const unsigned char* froi,
    const adapter_geom* mrg, const unsigned char* mroi,
    float* b200_score, int64_t* b200_nvox, float* b200_grad,
    float* ref_score, int64_t* ref_nvox, float* ref_grad)
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
    Bspline_xform bxf;
    bxf.initialize (origin, spacing, dim, roi_offset, roi_dim, vpr, dcos);
    memcpy (bxf.coeff, coeff, sizeof(float) * bxf.num_coeff);
    Bspline_parms parms;
    Regularization_parms rparms;
    parms.threading = BTHR_CPU;
    parms.implementation = flavor;
    parms.mi_hist_fixed_bins = bins;
    parms.mi_hist_moving_bins = bins;
    parms.mi_hist_type = vopt ? HIST_VOPT : HIST_EQSP;
    parms.regularization_parms = &rparms;
    Bspline_optimize bod;
    bod.set_bspline_parms (&parms);
    bod.set_bspline_xform (&bxf);
    Bspline_state* bst = bod.get_bspline_state ();

    Metric_state::Pointer ms = Metric_state::New ();
    ms->fixed_ss = Volume::New (fg->dim, fg->origin, fg->spacing, fg->dcos,
        PT_FLOAT, 1);
    memcpy (ms->fixed_ss->img, fimg, sizeof(float) * ms->fixed_ss->npix);
    ms->moving_ss = Volume::New (mg->dim, mg->origin, mg->spacing, mg->dcos,
        PT_FLOAT, 1);
    memcpy (ms->moving_ss->img, mimg, sizeof(float) * ms->moving_ss->npix);
    ms->moving_grad = volume_gradient (ms->moving_ss);
    if (froi) {
        ms->fixed_roi = Volume::New (frg->dim, frg->origin, frg->spacing,
            frg->dcos, PT_UCHAR, 1);
        memcpy (ms->fixed_roi->img, froi, ms->fixed_roi->npix);
    }
    if (mroi) {
        ms->moving_roi = Volume::New (mrg->dim, mrg->origin, mrg->spacing,
            mrg->dcos, PT_UCHAR, 1);
        memcpy (ms->moving_roi->img, mroi, ms->moving_roi->npix);
    }
    ms->metric_type = metric_mi
        ? SIMILARITY_METRIC_MI_MATTES : SIMILARITY_METRIC_MSE;
    ms->metric_lambda = 1.0f;
    bst->similarity_data.push_back (ms);
    bst->initialize (&bxf, &parms);
    bst->initialize_mi_histograms ();
    bst->set_metric_state (ms);

    int rc = bspline_b200_state_create (bst, &bxf, &parms,
        ms->fixed_ss.get (), ms->moving_ss.get (), ms->moving_grad.get ());
    if (rc == B200BSP_OK) {
        bst->ssd.reset_score ();
        rc = bspline_score_b200 (&bod);
        *b200_score = bst->ssd.curr_smetric;
        *b200_nvox = bst->ssd.curr_num_vox;
        memcpy (b200_grad, bst->ssd.curr_smetric_grad,
            sizeof(float) * bxf.num_coeff);
        b200bsp_destroy ((b200bsp_ctx*) bst->dev_ptrs);
        bst->dev_ptrs = 0;
    }
    bst->ssd.reset_score ();
    if (metric_mi) bspline_score_mi (&bod);
    else bspline_score_mse (&bod);
    *ref_score = bst->ssd.curr_smetric;
    *ref_nvox = bst->ssd.curr_num_vox;
    memcpy (ref_grad, bst->ssd.curr_smetric_grad,
        sizeof(float) * bxf.num_coeff);
    return rc;
}

}
