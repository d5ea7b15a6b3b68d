/* CPU restatement of Plastimatch's B-spline registration cost function.
 *
 * TEST INFRASTRUCTURE ONLY -- the checker for the CUDA path.  Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.
 *
 * Reference file:line anchors are relative to the Plastimatch source tree.
 * Compile with -ffp-contract=off: the _f32 routines keep the reference's
 * float operation order so that they agree with the compiled reference.
 * Parity of this restatement is pinned by tests/test_oracle.py against
 * golden vectors produced by the reference itself (tests/golden/). */
#include "bspline_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* Geometry                                                             */
/* ------------------------------------------------------------------ */

/* 3x3 inverse by cofactors, float (src/base/direction_cosines.cxx:135-158). */
static int
inv3 (float* out, const float* m)
{
    float det = m[0]*(m[4]*m[8]-m[5]*m[7])
        - m[1]*(m[3]*m[8]-m[5]*m[6])
        + m[2]*(m[3]*m[7]-m[4]*m[6]);
    if (fabs (det) < 1e-8) return -1;
    out[0] =  (m[4]*m[8]-m[5]*m[7]) / det;
    out[1] = -(m[1]*m[8]-m[2]*m[7]) / det;
    out[2] =  (m[1]*m[5]-m[2]*m[4]) / det;
    out[3] = -(m[3]*m[8]-m[5]*m[6]) / det;
    out[4] =  (m[0]*m[8]-m[2]*m[6]) / det;
    out[5] = -(m[0]*m[5]-m[2]*m[3]) / det;
    out[6] =  (m[3]*m[7]-m[4]*m[6]) / det;
    out[7] = -(m[0]*m[7]-m[1]*m[6]) / det;
    out[8] =  (m[0]*m[4]-m[1]*m[3]) / det;
    return 0;
}

/* step = dc * spacing (column scale), proj = inv_dc / spacing (row scale)
 * (src/base/direction_matrices.cxx:10-20). */
int
orc_vol_init (orc_vol* v, const int64_t dim[3], const float origin[3],
    const float spacing[3], const float dcos[9])
{
    for (int d = 0; d < 3; d++) {
        v->dim[d] = dim[d];
        v->origin[d] = origin[d];
        v->spacing[d] = spacing[d];
    }
    memcpy (v->dcos, dcos, 9 * sizeof(float));
    if (inv3 (v->inv_dcos, v->dcos)) return -1;
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) {
            v->step[3*i+j] = v->dcos[3*i+j] * spacing[j];
            v->proj[3*i+j] = v->inv_dcos[3*i+j] / spacing[i];
        }
    }
    return 0;
}

/* Bspline_header::set (src/base/bspline_header.cxx:28-62). */
int
orc_grid_init (orc_grid* g, const orc_vol* fixed,
    const int64_t roi_offset[3], const int64_t roi_dim[3],
    const int64_t vox_per_rgn[3])
{
    for (int d = 0; d < 3; d++) {
        if (vox_per_rgn[d] < 1 || roi_dim[d] < 1) return -1;
        g->img_origin[d] = fixed->origin[d];
        g->img_spacing[d] = fixed->spacing[d];
        g->img_dim[d] = fixed->dim[d];
        g->roi_offset[d] = roi_offset[d];
        g->roi_dim[d] = roi_dim[d];
        g->vox_per_rgn[d] = vox_per_rgn[d];
        g->grid_spac[d] = vox_per_rgn[d] * fabsf (fixed->spacing[d]);
        g->rdims[d] = 1 + (roi_dim[d] - 1) / vox_per_rgn[d];
        g->cdims[d] = 3 + g->rdims[d];
    }
    g->num_knots = g->cdims[0] * g->cdims[1] * g->cdims[2];
    g->num_coeff = 3 * g->num_knots;
    return 0;
}

/* Cubic B-spline basis at offset vox_idx/vpr, one of the four pieces t_idx
 * (src/base/bspline_xform.cxx:73-99): float argument, double evaluation. */
static float
basis_eval (int t_idx, int vox_idx, int vpr)
{
    float i = (float) vox_idx / vpr;
    switch (t_idx) {
    case 0: return (1.0/6.0) * (- 1.0 * i*i*i + 3.0 * i*i - 3.0 * i + 1.0);
    case 1: return (1.0/6.0) * (+ 3.0 * i*i*i - 6.0 * i*i + 4.0);
    case 2: return (1.0/6.0) * (- 3.0 * i*i*i + 3.0 * i*i + 3.0 * i + 1.0);
    case 3: return (1.0/6.0) * (+ 1.0 * i*i*i);
    }
    return 0.0;
}

/* bx/by/bz_lut[vpr*4] (src/base/bspline_xform.cxx:468-482). */
void
orc_basis_lut (float* lut, int64_t vpr)
{
    for (int j = 0; j < 4; j++)
        for (int i = 0; i < vpr; i++)
            lut[i*4+j] = basis_eval (j, i, (int) vpr);
}

/* q_lut[vpr^3 * 64] = A x B x C with float cubes
 * (src/base/bspline_xform.cxx:378-430). */
void
orc_q_lut (float* q_lut, const int64_t vpr[3])
{
    float* abc[3];
    for (int d = 0; d < 3; d++) {
        abc[d] = (float*) malloc (sizeof(float) * 4 * vpr[d]);
        for (int64_t i = 0; i < vpr[d]; i++) {
            float ii = ((float) i) / vpr[d];
            float t3 = ii*ii*ii, t2 = ii*ii, t1 = ii;
            abc[d][i*4+0] = (1.0/6.0) * (- 1.0 * t3 + 3.0 * t2 - 3.0 * t1 + 1.0);
            abc[d][i*4+1] = (1.0/6.0) * (+ 3.0 * t3 - 6.0 * t2 + 4.0);
            abc[d][i*4+2] = (1.0/6.0) * (- 3.0 * t3 + 3.0 * t2 + 3.0 * t1 + 1.0);
            abc[d][i*4+3] = (1.0/6.0) * (+ 1.0 * t3);
        }
    }
    int64_t p = 0;
    for (int64_t k = 0; k < vpr[2]; k++)
        for (int64_t j = 0; j < vpr[1]; j++)
            for (int64_t i = 0; i < vpr[0]; i++)
                for (int tz = 0; tz < 4; tz++)
                    for (int ty = 0; ty < 4; ty++)
                        for (int tx = 0; tx < 4; tx++)
                            q_lut[p++] = abc[0][i*4+tx] * abc[1][j*4+ty]
                                * abc[2][k*4+tz];
    for (int d = 0; d < 3; d++) free (abc[d]);
}

static inline int64_t
vidx (const int64_t dim[3], int64_t i, int64_t j, int64_t k)
{
    return i + dim[0] * (j + dim[1] * k);
}

/* ------------------------------------------------------------------ */
/* Moving-image gradient (src/base/volume_grad.cxx:9-76)                */
/* ------------------------------------------------------------------ */
void
orc_volume_grad (const orc_vol* v, const float* ref, float* out)
{
    const float* inv_dc = v->inv_dcos;
    int64_t n = 0;
    for (int64_t k = 0; k < v->dim[2]; k++) {
        int64_t kp = k == 0 ? 0 : k - 1;
        int64_t kn = k == v->dim[2] - 1 ? v->dim[2] - 1 : k + 1;
        for (int64_t j = 0; j < v->dim[1]; j++) {
            int64_t jp = j == 0 ? 0 : j - 1;
            int64_t jn = j == v->dim[1] - 1 ? v->dim[1] - 1 : j + 1;
            for (int64_t i = 0; i < v->dim[0]; i++, n++) {
                int64_t ip = i == 0 ? 0 : i - 1;
                int64_t in = i == v->dim[0] - 1 ? v->dim[0] - 1 : i + 1;
                float* o = &out[3*n];
                float diff;
                o[0] = o[1] = o[2] = 0.f;
                diff = (float) (ref[vidx (v->dim, in, j, k)]
                    - ref[vidx (v->dim, ip, j, k)]) / 2.0 / v->spacing[0];
                o[0] += diff * inv_dc[0]; o[1] += diff * inv_dc[3];
                o[2] += diff * inv_dc[6];
                diff = (float) (ref[vidx (v->dim, i, jn, k)]
                    - ref[vidx (v->dim, i, jp, k)]) / 2.0 / v->spacing[1];
                o[0] += diff * inv_dc[1]; o[1] += diff * inv_dc[4];
                o[2] += diff * inv_dc[7];
                diff = (float) (ref[vidx (v->dim, i, j, kn)]
                    - ref[vidx (v->dim, i, j, kp)]) / 2.0 / v->spacing[2];
                o[0] += diff * inv_dc[2]; o[1] += diff * inv_dc[5];
                o[2] += diff * inv_dc[8];
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* Shared float-precision voxel steps                                   */
/* ------------------------------------------------------------------ */

/* li_clamp (src/base/interpolate.cxx:17-41). */
static inline void
li_clamp_f (float ma, int64_t dmax, int64_t* maf, int64_t* mar,
    float* fa1, float* fa2)
{
    if (ma < 0.f) {
        *maf = 0; *mar = 0; *fa2 = 0.0f;
    } else if (ma >= dmax) {
        *maf = dmax - 1; *mar = dmax; *fa2 = 1.0f;
    } else {
        *maf = (int64_t) floor (ma);
        *mar = (ma >= 0) ? (int64_t) (ma + 0.5) : (int64_t) (-(-ma + 0.5));
        *fa2 = ma - *maf;
    }
    *fa1 = 1.0f - *fa2;
}

/* Volume::is_inside (src/base/volume.cxx:900-906). */
static inline int
inside_f (const float ijk[3], const int64_t dim[3])
{
    for (int d = 0; d < 3; d++) {
        if (ijk[d] <= -0.5 || ijk[d] >= dim[d] - 0.5) return 0;
    }
    return 1;
}

/* bspline_find_correspondence_dcos (src/util/bspline_correspond.cxx:
 * 80-107). */
static inline int
correspond_f (float mijk[3], const float fxyz[3], const float dxyz[3],
    const orc_vol* mv)
{
    float mxyz[3], tmp[3];
    for (int d = 0; d < 3; d++) mxyz[d] = fxyz[d] + dxyz[d];
    for (int d = 0; d < 3; d++) tmp[d] = mxyz[d] - mv->origin[d];
    for (int d = 0; d < 3; d++)
        mijk[d] = tmp[0] * mv->proj[3*d+0] + tmp[1] * mv->proj[3*d+1]
            + tmp[2] * mv->proj[3*d+2];
    return inside_f (mijk, mv->dim);
}

/* Image ROIs (uchar mask volumes with their own geometry), as
 * Bspline_state::fixed_roi / moving_roi hold them.  Set for the duration of
 * one oracle call by orc_set_roi (NULL: none). */
static const orc_roi* g_froi = 0;
static const orc_roi* g_mroi = 0;
/* set while the double-precision MI histogram pass runs: its fixed ROI
 * test takes LOOP_X's accumulated positions, as the reference's does */
static int g_roi_pass1 = 0;

void
orc_set_roi (const orc_roi* fixed_roi, const orc_roi* moving_roi)
{
    g_froi = fixed_roi;
    g_mroi = moving_roi;
}

/* inside_roi (src/util/bspline_correspond.cxx:52-74): project the world
 * position into the ROI volume, clamp each index to [0, dim - 1]
 * (float_to_plm_long_clamp, :11-50; floor inside), read the mask. */
static inline int
inside_roi_f (const float xyz[3], const orc_roi* r)
{
    float tmp[3], pf[3];
    int64_t p[3];
    const orc_vol* v = &r->vol;
    for (int d = 0; d < 3; d++) tmp[d] = xyz[d] - v->origin[d];
    for (int d = 0; d < 3; d++)
        pf[d] = tmp[0] * v->proj[3*d+0] + tmp[1] * v->proj[3*d+1]
            + tmp[2] * v->proj[3*d+2];
    for (int d = 0; d < 3; d++) {
        if (pf[d] < 0.f) p[d] = 0;
        else if (pf[d] >= v->dim[d]) p[d] = v->dim[d] - 1;
        else p[d] = (int64_t) floor (pf[d]);
    }
    return (int) r->mask[vidx (v->dim, p[0], p[1], p[2])];
}

/* bspline_find_correspondence_dcos_roi (src/util/bspline_correspond.cxx:
 * 112-145): the inside test, then the moving ROI at the moving position. */
static inline int
correspond_roi_f (float mijk[3], const float fxyz[3], const float dxyz[3],
    const orc_vol* mv)
{
    if (!correspond_f (mijk, fxyz, dxyz, mv)) return 0;
    if (!g_mroi) return 1;
    float mxyz[3];
    for (int d = 0; d < 3; d++) mxyz[d] = fxyz[d] + dxyz[d];
    return inside_roi_f (mxyz, g_mroi);
}

/* li_value (src/base/interpolate.cxx:135-158). */
static inline float
li_value_f (const float f1[3], const float f2[3], int64_t mvf,
    const float* m, const int64_t dim[3])
{
    int64_t dx = dim[0], dxy = dim[0] * dim[1];
    float a = f1[0] * f1[1] * f1[2] * m[mvf];
    float b = f2[0] * f1[1] * f1[2] * m[mvf+1];
    float c = f1[0] * f2[1] * f1[2] * m[mvf+dx];
    float d = f2[0] * f2[1] * f1[2] * m[mvf+dx+1];
    float e = f1[0] * f1[1] * f2[2] * m[mvf+dxy];
    float f = f2[0] * f1[1] * f2[2] * m[mvf+dxy+1];
    float g = f1[0] * f2[1] * f2[2] * m[mvf+dxy+dx];
    float h = f2[0] * f2[1] * f2[2] * m[mvf+dxy+dx+1];
    return a + b + c + d + e + f + g + h;
}

/* li_value_dx/dy/dz (src/base/interpolate.cxx:161-257). */
static inline void
li_value_d_f (float out[3], const float f1[3], const float f2[3],
    const float inv_r[3], int64_t mvf, const float* m, const int64_t dim[3])
{
    int64_t dx = dim[0], dxy = dim[0] * dim[1];
    float m0 = m[mvf], m1 = m[mvf+1], m2 = m[mvf+dx], m3 = m[mvf+dx+1];
    float m4 = m[mvf+dxy], m5 = m[mvf+dxy+1], m6 = m[mvf+dxy+dx];
    float m7 = m[mvf+dxy+dx+1];
    float rx = inv_r[0], ry = inv_r[1], rz = inv_r[2];
    out[0] = -rx * f1[1] * f1[2] * m0 + rx * f1[1] * f1[2] * m1
        + -rx * f2[1] * f1[2] * m2 + rx * f2[1] * f1[2] * m3
        + -rx * f1[1] * f2[2] * m4 + rx * f1[1] * f2[2] * m5
        + -rx * f2[1] * f2[2] * m6 + rx * f2[1] * f2[2] * m7;
    out[1] = -f1[0] * ry * f1[2] * m0 + -f2[0] * ry * f1[2] * m1
        + f1[0] * ry * f1[2] * m2 + f2[0] * ry * f1[2] * m3
        + -f1[0] * ry * f2[2] * m4 + -f2[0] * ry * f2[2] * m5
        + f1[0] * ry * f2[2] * m6 + f2[0] * ry * f2[2] * m7;
    out[2] = -f1[0] * f1[1] * rz * m0 + -f2[0] * f1[1] * rz * m1
        + -f1[0] * f2[1] * rz * m2 + -f2[0] * f2[1] * rz * m3
        + f1[0] * f1[1] * rz * m4 + f2[0] * f1[1] * rz * m5
        + f1[0] * f2[1] * rz * m6 + f2[0] * f2[1] * rz * m7;
}

/* Field at one voxel: bspline_interp_pix_c
 * (src/base/bspline_interpolate.cxx:78-110). */
static inline void
interp_pix_c (float out[3], const orc_grid* g, const float* coeff,
    const int64_t tile[3], const int64_t q[3], const float* bx,
    const float* by, const float* bz)
{
    const int64_t* cd = g->cdims;
    out[0] = out[1] = out[2] = 0;
    for (int k = 0; k < 4; k++) {
        float C = bz[q[2]*4+k];
        for (int j = 0; j < 4; j++) {
            float B = by[q[1]*4+j] * C;
            for (int i = 0; i < 4; i++) {
                float A = bx[q[0]*4+i] * B;
                int64_t cidx = 3 * ((tile[2] + k) * cd[1] * cd[0]
                    + (tile[1] + j) * cd[0] + (tile[0] + i));
                out[0] += A * coeff[cidx+0];
                out[1] += A * coeff[cidx+1];
                out[2] += A * coeff[cidx+2];
            }
        }
    }
}

/* bspline_update_sets_b (src/register/bspline.cxx:347-374). */
static inline void
update_sets_b (float* sx, float* sy, float* sz, const int64_t q[3],
    const float dc_dv[3], const float* bx, const float* by, const float* bz)
{
    int m = 0;
    for (int k = 0; k < 4; k++) {
        float C = bz[q[2]*4+k];
        for (int j = 0; j < 4; j++) {
            float B = by[q[1]*4+j] * C;
            for (int i = 0; i < 4; i++) {
                float A = bx[q[0]*4+i] * B;
                sx[m] += dc_dv[0] * A;
                sy[m] += dc_dv[1] * A;
                sz[m] += dc_dv[2] * A;
                m++;
            }
        }
    }
}

/* Tile sets -> knot-major slots: bspline_sort_sets + find_knots
 * (src/register/bspline.cxx:214-250, 377-398). */
static void
sort_sets (float* cx, float* cy, float* cz, const float* sx, const float* sy,
    const float* sz, const int64_t tile[3], const orc_grid* g)
{
    const int64_t* cd = g->cdims;
    int sidx = 0;
    for (int k = 0; k < 4; k++)
        for (int j = 0; j < 4; j++)
            for (int i = 0; i < 4; i++, sidx++) {
                int64_t kidx = (tile[2] + k) * cd[0] * cd[1]
                    + (tile[1] + j) * cd[0] + (tile[0] + i);
                cx[64*kidx + sidx] = sx[sidx];
                cy[64*kidx + sidx] = sy[sidx];
                cz[64*kidx + sidx] = sz[sidx];
            }
}

/* bspline_condense_smetric_grad (src/register/bspline.cxx:400-413). */
static void
condense (float* grad, const float* cx, const float* cy, const float* cz,
    int64_t num_knots)
{
    for (int64_t kidx = 0; kidx < num_knots; kidx++) {
        for (int s = 0; s < 64; s++) {
            grad[3*kidx+0] += cx[64*kidx + s];
            grad[3*kidx+1] += cy[64*kidx + s];
            grad[3*kidx+2] += cz[64*kidx + s];
        }
    }
}

/* bspline_score_normalize (src/register/bspline_mse.cxx:43-72). */
static void
normalize_f (float* score, float* grad, int64_t n, double raw,
    int64_t num_vox)
{
    if (num_vox < 1) {
        *score = FLT_MAX;
        for (int64_t i = 0; i < n; i++) grad[i] = 0;
    } else {
        *score = raw / num_vox;
        for (int64_t i = 0; i < n; i++) grad[i] = 2 * grad[i] / num_vox;
    }
}

/* ------------------------------------------------------------------ */
/* MSE, float, reference order                                          */
/* ------------------------------------------------------------------ */

/* grad_mode 0: bspline_score_g_mse (src/register/bspline_mse.cxx:519-720),
 * tiles in index order (the reference runs them under OpenMP; only the
 * double score reduction order differs). */
static int
mse_g_f32 (const orc_grid* g, const orc_vol* fx, const float* f_img,
    const orc_vol* mv, const float* m_img, const float* m_grad,
    const float* coeff, float* score, float* grad, int64_t* num_vox_out)
{
    const int64_t* vpr = g->vox_per_rgn;
    float* bx = (float*) malloc (sizeof(float) * 4 * vpr[0]);
    float* by = (float*) malloc (sizeof(float) * 4 * vpr[1]);
    float* bz = (float*) malloc (sizeof(float) * 4 * vpr[2]);
    orc_basis_lut (bx, vpr[0]);
    orc_basis_lut (by, vpr[1]);
    orc_basis_lut (bz, vpr[2]);
    size_t csz = (size_t) 64 * g->num_knots;
    float* cx = (float*) calloc (csz, sizeof(float));
    float* cy = (float*) calloc (csz, sizeof(float));
    float* cz = (float*) calloc (csz, sizeof(float));
    if (!bx || !by || !bz || !cx || !cy || !cz) return -1;

    int64_t num_vox = 0;
    double score_acc = 0;
    int64_t ntiles = g->rdims[0] * g->rdims[1] * g->rdims[2];
    for (int64_t t = 0; t < ntiles; t++) {
        int64_t tile[3], q[3];
        float sx[64], sy[64], sz[64];
        memset (sx, 0, sizeof sx);
        memset (sy, 0, sizeof sy);
        memset (sz, 0, sizeof sz);
        tile[2] = t / (g->rdims[0] * g->rdims[1]);
        tile[1] = (t - tile[2] * g->rdims[0] * g->rdims[1]) / g->rdims[0];
        tile[0] = t - tile[2] * g->rdims[0] * g->rdims[1]
            - tile[1] * g->rdims[0];
        for (q[2] = 0; q[2] < vpr[2]; q[2]++)
        for (q[1] = 0; q[1] < vpr[1]; q[1]++)
        for (q[0] = 0; q[0] < vpr[0]; q[0]++) {
            int64_t fijk[3];
            float fxyz[3], dxyz[3], mijk[3], li1[3], li2[3], dc_dv[3];
            int64_t mf[3], mr[3];
            int skip = 0;
            for (int d = 0; d < 3; d++) {
                fijk[d] = g->roi_offset[d] + vpr[d] * tile[d] + q[d];
                if (fijk[d] >= g->roi_offset[d] + g->roi_dim[d]) skip = 1;
            }
            if (skip) continue;
            for (int d = 0; d < 3; d++)
                fxyz[d] = g->img_origin[d] + fijk[0] * fx->step[3*d+0]
                    + fijk[1] * fx->step[3*d+1] + fijk[2] * fx->step[3*d+2];
            /* flavour i (bspline_mse.cxx:82-288): the fixed ROI at the
               fixed position, the moving ROI at the moving position */
            if (g_froi && !inside_roi_f (fxyz, g_froi)) continue;
            int64_t fidx = vidx (fx->dim, fijk[0], fijk[1], fijk[2]);
            interp_pix_c (dxyz, g, coeff, tile, q, bx, by, bz);
            if (!correspond_roi_f (mijk, fxyz, dxyz, mv)) continue;
            for (int d = 0; d < 3; d++)
                li_clamp_f (mijk[d], mv->dim[d] - 1, &mf[d], &mr[d],
                    &li1[d], &li2[d]);
            int64_t mvf = vidx (mv->dim, mf[0], mf[1], mf[2]);
            int64_t mvr = vidx (mv->dim, mr[0], mr[1], mr[2]);
            float m_val = li_value_f (li1, li2, mvf, m_img, mv->dim);
            float diff = m_val - f_img[fidx];
            score_acc += diff * diff;
            num_vox++;
            dc_dv[0] = diff * m_grad[3*mvr+0];
            dc_dv[1] = diff * m_grad[3*mvr+1];
            dc_dv[2] = diff * m_grad[3*mvr+2];
            update_sets_b (sx, sy, sz, q, dc_dv, bx, by, bz);
        }
        sort_sets (cx, cy, cz, sx, sy, sz, tile, g);
    }
    memset (grad, 0, sizeof(float) * g->num_coeff);
    condense (grad, cx, cy, cz, g->num_knots);
    normalize_f (score, grad, g->num_coeff, score_acc, num_vox);
    *num_vox_out = num_vox;
    free (bx); free (by); free (bz); free (cx); free (cy); free (cz);
    return 0;
}

/* grad_mode 1: bspline_score_o_mse (src/register/bspline_mse.cxx:946-1130):
 * voxel scan with incremental world positions (LOOP_Z/Y/X,
 * src/base/volume_macros.h:34-76), field from q_lut/c_lut
 * (bspline_interp_pix_b, src/base/bspline_interpolate.cxx:50-76), gradient
 * from the trilinear derivative, per-voxel scatter (Bspline_score::
 * update_grad_b, src/register/bspline_score.cxx:145-170). */
static int
mse_o_f32 (const orc_grid* g, const orc_vol* fx, const float* f_img,
    const orc_vol* mv, const float* m_img, const float* coeff, float* score,
    float* grad, int64_t* num_vox_out)
{
    const int64_t* vpr = g->vox_per_rgn;
    const int64_t* cd = g->cdims;
    int64_t nq = vpr[0] * vpr[1] * vpr[2];
    float* q_lut = (float*) malloc (sizeof(float) * 64 * nq);
    if (!q_lut) return -1;
    orc_q_lut (q_lut, vpr);
    float inv_r[3];
    for (int d = 0; d < 3; d++) inv_r[d] = 1.0 / mv->spacing[d];
    memset (grad, 0, sizeof(float) * g->num_coeff);
    double score_acc = 0.;
    int64_t num_vox = 0;
    int64_t fijk[3], p[3], q[3];
    float fxyz[3];
    const float* st = fx->step;
    const float* org = fx->origin;
    for (fijk[2] = 0, fxyz[2] = org[2]; fijk[2] < fx->dim[2];
         ++fijk[2], fxyz[2] = org[2] + fijk[2]*st[2*3+2]) {
        p[2] = fijk[2] / vpr[2]; q[2] = fijk[2] % vpr[2];
        for (fijk[1] = 0, fxyz[1] = org[1] + fijk[2]*st[1*3+2];
             fijk[1] < fx->dim[1];
             ++fijk[1],
             fxyz[2] = org[2] + fijk[2]*st[2*3+2] + fijk[1]*st[2*3+1],
             fxyz[1] = org[1] + fijk[2]*st[1*3+2] + fijk[1]*st[1*3+1]) {
            p[1] = fijk[1] / vpr[1]; q[1] = fijk[1] % vpr[1];
            for (fijk[0] = 0,
                 fxyz[0] = org[0] + fijk[2]*st[0*3+2] + fijk[1]*st[0*3+1];
                 fijk[0] < fx->dim[0];
                 ++fijk[0], fxyz[0] += st[0], fxyz[1] += st[3],
                 fxyz[2] += st[6]) {
                p[0] = fijk[0] / vpr[0]; q[0] = fijk[0] % vpr[0];
                int64_t qidx = vidx (vpr, q[0], q[1], q[2]);
                const float* ql = &q_lut[64*qidx];
                float dxyz[3] = {0, 0, 0}, mijk[3], li1[3], li2[3], dc_dv[3];
                int64_t mf[3], mr[3];
                int m = 0;
                for (int k = 0; k < 4; k++)
                    for (int j = 0; j < 4; j++)
                        for (int i = 0; i < 4; i++, m++) {
                            int64_t cidx = 3 * ((p[2]+k) * cd[1] * cd[0]
                                + (p[1]+j) * cd[0] + (p[0]+i));
                            dxyz[0] += ql[m] * coeff[cidx+0];
                            dxyz[1] += ql[m] * coeff[cidx+1];
                            dxyz[2] += ql[m] * coeff[cidx+2];
                        }
                if (!correspond_f (mijk, fxyz, dxyz, mv)) continue;
                for (int d = 0; d < 3; d++)
                    li_clamp_f (mijk[d], mv->dim[d] - 1, &mf[d], &mr[d],
                        &li1[d], &li2[d]);
                int64_t mvf = vidx (mv->dim, mf[0], mf[1], mf[2]);
                float m_val = li_value_f (li1, li2, mvf, m_img, mv->dim);
                float md[3];
                li_value_d_f (md, li1, li2, inv_r, mvf, m_img, mv->dim);
                int64_t fv = vidx (fx->dim, fijk[0], fijk[1], fijk[2]);
                float diff = m_val - f_img[fv];
                dc_dv[0] = diff * md[0];
                dc_dv[1] = diff * md[1];
                dc_dv[2] = diff * md[2];
                m = 0;
                for (int k = 0; k < 4; k++)
                    for (int j = 0; j < 4; j++)
                        for (int i = 0; i < 4; i++, m++) {
                            int64_t cidx = 3 * ((p[2]+k) * cd[1] * cd[0]
                                + (p[1]+j) * cd[0] + (p[0]+i));
                            grad[cidx+0] += dc_dv[0] * ql[m];
                            grad[cidx+1] += dc_dv[1] * ql[m];
                            grad[cidx+2] += dc_dv[2] * ql[m];
                        }
                score_acc += diff * diff;
                num_vox++;
            }
        }
    }
    normalize_f (score, grad, g->num_coeff, score_acc, num_vox);
    *num_vox_out = num_vox;
    free (q_lut);
    return 0;
}

int
orc_mse_f32 (const orc_grid* g, const orc_vol* fixed, const float* f_img,
    const orc_vol* moving, const float* m_img, const float* m_grad,
    const float* coeff, int grad_mode, float* score, float* grad,
    int64_t* num_vox)
{
    if (grad_mode == 0)
        return mse_g_f32 (g, fixed, f_img, moving, m_img, m_grad, coeff,
            score, grad, num_vox);
    return mse_o_f32 (g, fixed, f_img, moving, m_img, coeff, score, grad,
        num_vox);
}

/* ------------------------------------------------------------------ */
/* Double-precision evaluation of the same algorithms                   */
/* ------------------------------------------------------------------ */

typedef struct {
    double origin[3];
    double step[9];
    double proj[9];
    int64_t dim[3];
    double spacing[3];
} vol64;

static int
vol64_init (vol64* o, const orc_vol* v)
{
    double m[9], inv[9];
    for (int i = 0; i < 9; i++) m[i] = v->dcos[i];
    double det = m[0]*(m[4]*m[8]-m[5]*m[7]) - m[1]*(m[3]*m[8]-m[5]*m[6])
        + m[2]*(m[3]*m[7]-m[4]*m[6]);
    if (fabs (det) < 1e-8) return -1;
    inv[0] =  (m[4]*m[8]-m[5]*m[7]) / det;
    inv[1] = -(m[1]*m[8]-m[2]*m[7]) / det;
    inv[2] =  (m[1]*m[5]-m[2]*m[4]) / det;
    inv[3] = -(m[3]*m[8]-m[5]*m[6]) / det;
    inv[4] =  (m[0]*m[8]-m[2]*m[6]) / det;
    inv[5] = -(m[0]*m[5]-m[2]*m[3]) / det;
    inv[6] =  (m[3]*m[7]-m[4]*m[6]) / det;
    inv[7] = -(m[0]*m[7]-m[1]*m[6]) / det;
    inv[8] =  (m[0]*m[4]-m[1]*m[3]) / det;
    for (int d = 0; d < 3; d++) {
        o->origin[d] = v->origin[d];
        o->dim[d] = v->dim[d];
        o->spacing[d] = v->spacing[d];
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            o->step[3*i+j] = m[3*i+j] * (double) v->spacing[j];
            o->proj[3*i+j] = inv[3*i+j] / (double) v->spacing[i];
        }
    return 0;
}

static void
basis_lut64 (double* lut, int64_t vpr)
{
    for (int64_t i = 0; i < vpr; i++) {
        double u = (double) i / (double) vpr;
        lut[i*4+0] = (1.0/6.0) * (1.0 - u) * (1.0 - u) * (1.0 - u);
        lut[i*4+1] = (1.0/6.0) * (3.0*u*u*u - 6.0*u*u + 4.0);
        lut[i*4+2] = (1.0/6.0) * (-3.0*u*u*u + 3.0*u*u + 3.0*u + 1.0);
        lut[i*4+3] = (1.0/6.0) * u*u*u;
    }
}

typedef struct {
    int ok;
    int64_t mvf, mvr;
    double w1[3], w2[3];
    int clamped[3];          /* li_clamp held the position at an end */
} tri64;

/* One voxel's correspondence + clamp in double: the same decisions as
 * bspline_find_correspondence_dcos / is_inside / li_clamp. */
static inline tri64
locate64 (const double fxyz[3], const double dxyz[3], const vol64* mv)
{
    tri64 r;
    double mijk[3];
    for (int d = 0; d < 3; d++) {
        double t0 = fxyz[0] + dxyz[0] - mv->origin[0];
        double t1 = fxyz[1] + dxyz[1] - mv->origin[1];
        double t2 = fxyz[2] + dxyz[2] - mv->origin[2];
        mijk[d] = t0 * mv->proj[3*d+0] + t1 * mv->proj[3*d+1]
            + t2 * mv->proj[3*d+2];
    }
    r.ok = 1;
    for (int d = 0; d < 3; d++)
        if (mijk[d] <= -0.5 || mijk[d] >= mv->dim[d] - 0.5) r.ok = 0;
    if (!r.ok) return r;
    int64_t f[3], rr[3];
    for (int d = 0; d < 3; d++) {
        double ma = mijk[d];
        int64_t dmax = mv->dim[d] - 1;
        r.clamped[d] = ma < 0. || ma >= dmax;
        if (ma < 0.) { f[d] = 0; rr[d] = 0; r.w2[d] = 0.; }
        else if (ma >= dmax) { f[d] = dmax - 1; rr[d] = dmax; r.w2[d] = 1.; }
        else {
            f[d] = (int64_t) floor (ma);
            rr[d] = (int64_t) (ma + 0.5);
            r.w2[d] = ma - f[d];
        }
        r.w1[d] = 1. - r.w2[d];
    }
    r.mvf = vidx (mv->dim, f[0], f[1], f[2]);
    r.mvr = vidx (mv->dim, rr[0], rr[1], rr[2]);
    return r;
}

/* The moving ROI at the moving position, decided in float as the
 * reference does. */
static inline int
moving_roi64 (const double fxyz[3], const double dxyz[3])
{
    if (!g_mroi) return 1;
    float mxyz[3];
    for (int d = 0; d < 3; d++) mxyz[d] = (float) fxyz[d] + (float) dxyz[d];
    return inside_roi_f (mxyz, g_mroi);
}

static inline void
corner_weights64 (double w[8], const tri64* t)
{
    for (int c = 0; c < 8; c++) {
        w[c] = ((c & 1) ? t->w2[0] : t->w1[0])
            * ((c & 2) ? t->w2[1] : t->w1[1])
            * ((c & 4) ? t->w2[2] : t->w1[2]);
    }
}

static inline int64_t
corner_index (int64_t mvf, int c, const int64_t dim[3])
{
    return mvf + ((c & 1) ? 1 : 0) + ((c & 2) ? dim[0] : 0)
        + ((c & 4) ? dim[0] * dim[1] : 0);
}

/* Tile loop shared by the double-precision metrics: visits every ROI voxel
 * tile by tile (LOOP_THRU_VOL_TILES order) and hands the voxel's world
 * position, displacement and tile-local basis weights to `visit`. */
typedef void (*voxel_fn) (void* ctx, int64_t fidx, const double fxyz[3],
    const double dxyz[3], double* dc_dv_out, int* has_grad);

static void
tile_loop64 (const orc_grid* g, const vol64* fx, const float* coeff,
    voxel_fn visit, void* ctx, double* grad)
{
    const int64_t* vpr = g->vox_per_rgn;
    const int64_t* cd = g->cdims;
    double* lut[3];
    for (int d = 0; d < 3; d++) {
        lut[d] = (double*) malloc (sizeof(double) * 4 * vpr[d]);
        basis_lut64 (lut[d], vpr[d]);
    }
    if (grad) memset (grad, 0, sizeof(double) * g->num_coeff);
    int64_t ntiles = g->rdims[0] * g->rdims[1] * g->rdims[2];
    for (int64_t t = 0; t < ntiles; t++) {
        int64_t tile[3], q[3];
        tile[2] = t / (g->rdims[0] * g->rdims[1]);
        tile[1] = (t / g->rdims[0]) % g->rdims[1];
        tile[0] = t % g->rdims[0];
        double sets[64][3];
        memset (sets, 0, sizeof sets);
        for (q[2] = 0; q[2] < vpr[2]; q[2]++)
        for (q[1] = 0; q[1] < vpr[1]; q[1]++)
        for (q[0] = 0; q[0] < vpr[0]; q[0]++) {
            int64_t fijk[3];
            int skip = 0;
            for (int d = 0; d < 3; d++) {
                fijk[d] = g->roi_offset[d] + vpr[d] * tile[d] + q[d];
                if (fijk[d] >= g->roi_offset[d] + g->roi_dim[d]) skip = 1;
            }
            if (skip) continue;
            double fxyz[3], dxyz[3] = {0, 0, 0}, dc_dv[3];
            for (int d = 0; d < 3; d++)
                fxyz[d] = (double) g->img_origin[d]
                    + fijk[0] * fx->step[3*d+0] + fijk[1] * fx->step[3*d+1]
                    + fijk[2] * fx->step[3*d+2];
            if (g_froi) {
                /* the ROI decision in the reference's float positions:
                   POSITION_FROM_COORDS, or in the whole-image histogram
                   scan the position LOOP_Z/Y/X accumulate along x
                   (src/base/volume_macros.h:38-97) */
                float fxyz_f[3];
                if (g_roi_pass1) {
                    float s[9];
                    for (int i = 0; i < 9; i++) s[i] = (float) fx->step[i];
                    fxyz_f[0] = g->img_origin[0] + fijk[2] * s[2] + fijk[1] * s[1];
                    fxyz_f[1] = g->img_origin[1] + fijk[2] * s[5] + fijk[1] * s[4];
                    fxyz_f[2] = g->img_origin[2] + fijk[2] * s[8] + fijk[1] * s[7];
                    for (int64_t i = 0; i < fijk[0]; i++) {
                        fxyz_f[0] += s[0];
                        fxyz_f[1] += s[3];
                        fxyz_f[2] += s[6];
                    }
                } else {
                    for (int d = 0; d < 3; d++)
                        fxyz_f[d] = g->img_origin[d]
                            + fijk[0] * (float) fx->step[3*d+0]
                            + fijk[1] * (float) fx->step[3*d+1]
                            + fijk[2] * (float) fx->step[3*d+2];
                }
                if (!inside_roi_f (fxyz_f, g_froi)) continue;
            }
            double w[64];
            int m = 0;
            for (int k = 0; k < 4; k++)
                for (int j = 0; j < 4; j++)
                    for (int i = 0; i < 4; i++, m++) {
                        w[m] = lut[0][q[0]*4+i] * lut[1][q[1]*4+j]
                            * lut[2][q[2]*4+k];
                        int64_t cidx = 3 * ((tile[2]+k) * cd[1] * cd[0]
                            + (tile[1]+j) * cd[0] + (tile[0]+i));
                        dxyz[0] += w[m] * coeff[cidx+0];
                        dxyz[1] += w[m] * coeff[cidx+1];
                        dxyz[2] += w[m] * coeff[cidx+2];
                    }
            int64_t fidx = vidx (fx->dim, fijk[0], fijk[1], fijk[2]);
            int has_grad = 0;
            visit (ctx, fidx, fxyz, dxyz, dc_dv, &has_grad);
            if (has_grad && grad) {
                for (m = 0; m < 64; m++) {
                    sets[m][0] += dc_dv[0] * w[m];
                    sets[m][1] += dc_dv[1] * w[m];
                    sets[m][2] += dc_dv[2] * w[m];
                }
            }
        }
        if (grad) {
            int m = 0;
            for (int k = 0; k < 4; k++)
                for (int j = 0; j < 4; j++)
                    for (int i = 0; i < 4; i++, m++) {
                        int64_t kidx = (tile[2]+k) * cd[1] * cd[0]
                            + (tile[1]+j) * cd[0] + (tile[0]+i);
                        grad[3*kidx+0] += sets[m][0];
                        grad[3*kidx+1] += sets[m][1];
                        grad[3*kidx+2] += sets[m][2];
                    }
        }
    }
    for (int d = 0; d < 3; d++) free (lut[d]);
}

typedef struct {
    const vol64* mv;
    const float* f_img;
    const float* m_img;
    const float* m_grad;
    int grad_mode;
    double score;
    int64_t num_vox;
} mse64_ctx;

static void
mse64_visit (void* vctx, int64_t fidx, const double fxyz[3],
    const double dxyz[3], double* dc_dv, int* has_grad)
{
    mse64_ctx* c = (mse64_ctx*) vctx;
    tri64 t = locate64 (fxyz, dxyz, c->mv);
    if (!t.ok || !moving_roi64 (fxyz, dxyz)) return;
    double w[8], mval = 0;
    corner_weights64 (w, &t);
    for (int k = 0; k < 8; k++)
        mval += w[k] * c->m_img[corner_index (t.mvf, k, c->mv->dim)];
    double diff = mval - (double) c->f_img[fidx];
    c->score += diff * diff;
    c->num_vox++;
    if (c->grad_mode == 0) {
        for (int d = 0; d < 3; d++)
            dc_dv[d] = diff * (double) c->m_grad[3*t.mvr + d];
    } else {
        /* derivative of the trilinear interpolant / spacing */
        double g[3] = {0, 0, 0};
        for (int k = 0; k < 8; k++) {
            double mk = c->m_img[corner_index (t.mvf, k, c->mv->dim)];
            double sx = (k & 1) ? 1. : -1., sy = (k & 2) ? 1. : -1.;
            double sz = (k & 4) ? 1. : -1.;
            double wx = (k & 1) ? t.w2[0] : t.w1[0];
            double wy = (k & 2) ? t.w2[1] : t.w1[1];
            double wz = (k & 4) ? t.w2[2] : t.w1[2];
            g[0] += sx * wy * wz * mk;
            g[1] += wx * sy * wz * mk;
            g[2] += wx * wy * sz * mk;
        }
        for (int d = 0; d < 3; d++)
            dc_dv[d] = diff * g[d] / c->mv->spacing[d];
    }
    *has_grad = 1;
}

int
orc_mse_f64 (const orc_grid* g, const orc_vol* fixed, const float* f_img,
    const orc_vol* moving, const float* m_img, const float* m_grad,
    const float* coeff, int grad_mode, double* score, double* grad,
    int64_t* num_vox)
{
    vol64 fx, mv;
    if (vol64_init (&fx, fixed) || vol64_init (&mv, moving)) return -1;
    mse64_ctx c = { &mv, f_img, m_img, m_grad, grad_mode, 0., 0 };
    tile_loop64 (g, &fx, coeff, mse64_visit, &c, grad);
    *num_vox = c.num_vox;
    if (c.num_vox < 1) {
        *score = FLT_MAX;
        memset (grad, 0, sizeof(double) * g->num_coeff);
        return 0;
    }
    *score = c.score / c.num_vox;
    for (int64_t i = 0; i < g->num_coeff; i++)
        grad[i] = 2. * grad[i] / c.num_vox;
    return 0;
}

/* ------------------------------------------------------------------ */
/* Mattes MI, PVI-8 (flavour g)                                          */
/* ------------------------------------------------------------------ */

/* bspline_initialize_mi_hist_eqsp (src/register/joint_histogram.cxx:
 * 115-139). */
void
orc_hist_eqsp (orc_hist* h, const float* img, int64_t n)
{
    float mn = img[0], mx = img[0];
    for (int64_t i = 0; i < n; i++) {
        if (img[i] < mn) mn = img[i];
        else if (img[i] > mx) mx = img[i];
    }
    h->delta = (mx - mn) / (h->bins - 1);
    h->offset = mn - 0.5 * h->delta;
    h->keys = 0;
    h->key_lut = 0;
}

static inline int
bin_of (float v, const orc_hist* h)
{
    int b = (int) floor ((v - h->offset) / h->delta);
    return h->key_lut ? h->key_lut[b] : b;
}

/* vopt_bin_error (src/register/joint_histogram.cxx:61-79): the squared
 * error of one bin spanning keys [start, end] from the prefix tables;
 * DBL_MAX for a bin holding less than one voxel. */
static double
vopt_err (int64_t start, int64_t end, const double* s, const double* ssq,
    const double* cnt)
{
    double sq = ssq[end] - ssq[start];
    double d = s[end] - s[start];
    double w = (double) end - (double) start + 1.0;
    double n = cnt[end] - cnt[start];
    double v = sq - (d * d) / w;
    if (n < 1.0) return DBL_MAX;
    return v;
}

void
orc_hist_vopt (orc_hist* h, int32_t* key_lut, const float* img, int64_t n)
{
    const int64_t K = 1000, B = h->bins;
    double* hist = (double*) calloc (K, sizeof(double));
    double* avg = (double*) calloc (K, sizeof(double));
    double* s = (double*) malloc (K * sizeof(double));
    double* ssq = (double*) malloc (K * sizeof(double));
    double* cnt = (double*) malloc (K * sizeof(double));
    double* err = (double*) calloc (B * K, sizeof(double));
    int64_t* trk = (int64_t*) calloc (B * K, sizeof(int64_t));
    float mn = img[0], mx = img[0];
    for (int64_t i = 1; i < n; i++) {
        if (img[i] < mn) mn = img[i];
        else if (img[i] > mx) mx = img[i];
    }
    h->keys = K;
    h->delta = (mx - mn) / (K - 1);
    h->offset = mn - 0.5 * h->delta;
    for (int64_t i = 0; i < n; i++) {
        int b = (int) floor ((img[i] - h->offset) / h->delta);
        hist[b]++;
        avg[b] += img[i] - h->offset;
    }
    for (int64_t i = 0; i < K; i++) {
        if (hist[i] > 0) avg[i] = avg[i] / hist[i];
        else if (i > 0) avg[i] = avg[i-1];
    }
    s[0] = avg[0];
    ssq[0] = avg[0] * avg[0];
    cnt[0] = hist[0];
    for (int64_t i = 1; i < K; i++) {
        s[i] = s[i-1] + avg[i];
        ssq[i] = ssq[i-1] + avg[i] * avg[i];
        cnt[i] = cnt[i-1] + hist[i];
    }
    for (int64_t i = 0; i < K; i++) err[i] = vopt_err (0, i, s, ssq, cnt);
    for (int64_t j = 1; j < B; j++) {
        for (int64_t i = 0; i < K; i++) {
            err[K*j+i] = DBL_MAX;
            trk[K*j+i] = 0;
            for (int64_t k = 0; k < i; k++) {
                double c = err[K*(j-1)+k] + vopt_err (k + 1, i, s, ssq, cnt);
                if (c <= err[K*j+i]) {
                    err[K*j+i] = c;
                    trk[K*j+i] = k;
                }
            }
        }
    }
    for (int64_t i = 0; i < K; i++) key_lut[i] = 0;
    int64_t curr = K - 1;
    for (int64_t j = B - 1; j >= 0; j--) {
        int64_t next = trk[K*j+curr];
        int64_t bottom = j == 0 ? 0 : next + 1;
        for (int64_t i = bottom; i <= curr; i++) key_lut[i] = (int32_t) j;
        curr = next;
    }
    h->key_lut = key_lut;
    free (hist); free (avg); free (s); free (ssq); free (cnt); free (err);
    free (trk);
}

/* Joint_histogram::add_pvi_8 (src/register/joint_histogram.cxx:423-486). */
static inline void
add_pvi_8 (double* fh, double* mh, double* jh, const orc_hist* fhp,
    const orc_hist* mhp, float fval, const float* m_img, int64_t mvf,
    const int64_t dim[3], const float li1[3], const float li2[3])
{
    float w[8];
    int64_t n[8];
    w[0] = li1[0] * li1[1] * li1[2];
    w[1] = li2[0] * li1[1] * li1[2];
    w[2] = li1[0] * li2[1] * li1[2];
    w[3] = li2[0] * li2[1] * li1[2];
    w[4] = li1[0] * li1[1] * li2[2];
    w[5] = li2[0] * li1[1] * li2[2];
    w[6] = li1[0] * li2[1] * li2[2];
    w[7] = li2[0] * li2[1] * li2[2];
    n[0] = mvf; n[1] = n[0] + 1; n[2] = n[0] + dim[0]; n[3] = n[2] + 1;
    n[4] = n[0] + dim[0]*dim[1]; n[5] = n[4] + 1; n[6] = n[4] + dim[0];
    n[7] = n[6] + 1;
    int fb = bin_of (fval, fhp);
    fh[fb]++;
    int64_t off = (int64_t) fb * mhp->bins;
    for (int pv = 0; pv < 8; pv++) {
        int mb = bin_of (m_img[n[pv]], mhp);
        mh[mb] += w[pv];
        jh[off + mb] += w[pv];
    }
}

/* mi_hist_score_omp (src/register/bspline_mi.cxx:285-309), serial. */
static float
mi_score (const double* fh, const double* mh, const double* jh,
    const orc_hist* fhp, const orc_hist* mhp, int64_t num_vox)
{
    double fnv = (double) num_vox, score = 0;
    double thresh = 0.001 / (mhp->bins * fhp->bins);
    for (int64_t jb = 0; jb < fhp->bins * mhp->bins; jb++) {
        int64_t mb = jb % mhp->bins, fb = jb / mhp->bins;
        if (jh[jb] > thresh)
            score -= jh[jb] * logf (fnv * jh[jb] / (mh[mb] * fh[fb]));
    }
    return (float) (score / fnv);
}

/* bspline_mi_pvi_8_dc_dv_dcos (src/register/bspline_mi.txx:9-120),
 * including its in-place projection of dc_dv through proj. */
static inline void
mi_dc_dv (float dc_dv[3], const double* fh, const double* mh,
    const double* jh, const orc_hist* fhp, const orc_hist* mhp, float fval,
    const float* m_img, int64_t mvf, const orc_vol* mv, float num_vox_f,
    float smetric, const float li1[3], const float li2[3])
{
    float dw[24];
    int64_t n[8];
    const int64_t* dim = mv->dim;
    dc_dv[0] = dc_dv[1] = dc_dv[2] = 0.0f;
    n[0] = mvf; n[1] = n[0] + 1; n[2] = n[0] + dim[0]; n[3] = n[2] + 1;
    n[4] = n[0] + dim[0]*dim[1]; n[5] = n[4] + 1; n[6] = n[4] + dim[0];
    n[7] = n[6] + 1;
    dw[0] = (-1) * li1[1] * li1[2]; dw[1] = li1[0] * (-1) * li1[2];
    dw[2] = li1[0] * li1[1] * (-1);
    dw[3] = (+1) * li1[1] * li1[2]; dw[4] = li2[0] * (-1) * li1[2];
    dw[5] = li2[0] * li1[1] * (-1);
    dw[6] = (-1) * li2[1] * li1[2]; dw[7] = li1[0] * (+1) * li1[2];
    dw[8] = li1[0] * li2[1] * (-1);
    dw[9] = (+1) * li2[1] * li1[2]; dw[10] = li2[0] * (+1) * li1[2];
    dw[11] = li2[0] * li2[1] * (-1);
    dw[12] = (-1) * li1[1] * li2[2]; dw[13] = li1[0] * (-1) * li2[2];
    dw[14] = li1[0] * li1[1] * (+1);
    dw[15] = (+1) * li1[1] * li2[2]; dw[16] = li2[0] * (-1) * li2[2];
    dw[17] = li2[0] * li1[1] * (+1);
    dw[18] = (-1) * li2[1] * li2[2]; dw[19] = li1[0] * (+1) * li2[2];
    dw[20] = li1[0] * li2[1] * (+1);
    dw[21] = (+1) * li2[1] * li2[2]; dw[22] = li2[0] * (+1) * li2[2];
    dw[23] = li2[0] * li2[1] * (+1);
    int fb = bin_of (fval, fhp);
    int64_t off = (int64_t) fb * mhp->bins;
    for (int pv = 0; pv < 8; pv++) {
        int mb = bin_of (m_img[n[pv]], mhp);
        int64_t jb = off + mb;
        if (jh[jb] > 0.0001) {
            float dS_dP = logf ((num_vox_f * jh[jb]) / (fh[fb] * mh[mb]))
                - smetric;
            dc_dv[0] -= dw[3*pv+0] * dS_dP;
            dc_dv[1] -= dw[3*pv+1] * dS_dP;
            dc_dv[2] -= dw[3*pv+2] * dS_dP;
        }
    }
    dc_dv[0] = dc_dv[0] / num_vox_f;
    dc_dv[1] = dc_dv[1] / num_vox_f;
    dc_dv[2] = dc_dv[2] / num_vox_f;
    const float* pr = mv->proj;
    dc_dv[0] = dc_dv[0] * pr[0] + dc_dv[1] * pr[1] + dc_dv[2] * pr[2];
    dc_dv[1] = dc_dv[0] * pr[3] + dc_dv[1] * pr[4] + dc_dv[2] * pr[5];
    dc_dv[2] = dc_dv[0] * pr[6] + dc_dv[1] * pr[7] + dc_dv[2] * pr[8];
}

/* bspline_score_g_mi (src/register/bspline_mi.cxx:1505-1750); with image
 * ROIs set, bspline_score_h_mi (:1232-1504), which adds the fixed ROI test
 * at the fixed position and the moving ROI test at the moving position to
 * both passes.  Pass 1 is the voxel scan over the whole fixed image with
 * incremental world positions and tile index fijk / vox_per_rgn; pass 2 is
 * the tile loop over the grid's ROI.  Pass 1's tile index is in range only
 * when the grid starts at voxel 0 and its tiles cover the image (returns -2
 * otherwise; the reference reads past its tables there). */
int
orc_mi_f32 (const orc_grid* g, const orc_vol* fx, const float* f_img,
    const orc_vol* mv, const float* m_img, const float* coeff,
    const orc_hist* fhp, const orc_hist* mhp, float* score, float* grad,
    int64_t* num_vox_out, double* fh, double* mh, double* jh)
{
    const int64_t* vpr = g->vox_per_rgn;
    for (int d = 0; d < 3; d++)
        if (g->roi_offset[d] != 0 || g->rdims[d] * vpr[d] < fx->dim[d])
            return -2;
    float* bx = (float*) malloc (sizeof(float) * 4 * vpr[0]);
    float* by = (float*) malloc (sizeof(float) * 4 * vpr[1]);
    float* bz = (float*) malloc (sizeof(float) * 4 * vpr[2]);
    orc_basis_lut (bx, vpr[0]);
    orc_basis_lut (by, vpr[1]);
    orc_basis_lut (bz, vpr[2]);
    memset (fh, 0, sizeof(double) * fhp->bins);
    memset (mh, 0, sizeof(double) * mhp->bins);
    memset (jh, 0, sizeof(double) * fhp->bins * mhp->bins);
    int64_t num_vox = 0;

    /* pass 1 */
    int64_t fijk[3], p[3], q[3];
    float fxyz[3];
    const float* st = fx->step;
    const float* org = fx->origin;
    for (fijk[2] = 0, fxyz[2] = org[2]; fijk[2] < fx->dim[2];
         ++fijk[2], fxyz[2] = org[2] + fijk[2]*st[2*3+2]) {
        p[2] = fijk[2] / vpr[2]; q[2] = fijk[2] % vpr[2];
        for (fijk[1] = 0, fxyz[1] = org[1] + fijk[2]*st[1*3+2];
             fijk[1] < fx->dim[1];
             ++fijk[1],
             fxyz[2] = org[2] + fijk[2]*st[2*3+2] + fijk[1]*st[2*3+1],
             fxyz[1] = org[1] + fijk[2]*st[1*3+2] + fijk[1]*st[1*3+1]) {
            p[1] = fijk[1] / vpr[1]; q[1] = fijk[1] % vpr[1];
            for (fijk[0] = 0,
                 fxyz[0] = org[0] + fijk[2]*st[0*3+2] + fijk[1]*st[0*3+1];
                 fijk[0] < fx->dim[0];
                 ++fijk[0], fxyz[0] += st[0], fxyz[1] += st[3],
                 fxyz[2] += st[6]) {
                p[0] = fijk[0] / vpr[0]; q[0] = fijk[0] % vpr[0];
                float dxyz[3], mijk[3], li1[3], li2[3];
                int64_t mf[3], mr[3];
                if (g_froi && !inside_roi_f (fxyz, g_froi)) continue;
                interp_pix_c (dxyz, g, coeff, p, q, bx, by, bz);
                if (!correspond_roi_f (mijk, fxyz, dxyz, mv)) continue;
                for (int d = 0; d < 3; d++)
                    li_clamp_f (mijk[d], mv->dim[d] - 1, &mf[d], &mr[d],
                        &li1[d], &li2[d]);
                int64_t fidx = vidx (fx->dim, fijk[0], fijk[1], fijk[2]);
                int64_t mvf = vidx (mv->dim, mf[0], mf[1], mf[2]);
                add_pvi_8 (fh, mh, jh, fhp, mhp, f_img[fidx], m_img, mvf,
                    mv->dim, li1, li2);
                num_vox++;
            }
        }
    }
    float smetric = mi_score (fh, mh, jh, fhp, mhp, num_vox);
    float num_vox_f = (float) num_vox;

    /* pass 2 */
    size_t csz = (size_t) 64 * g->num_knots;
    float* cx = (float*) calloc (csz, sizeof(float));
    float* cy = (float*) calloc (csz, sizeof(float));
    float* cz = (float*) calloc (csz, sizeof(float));
    int64_t ntiles = g->rdims[0] * g->rdims[1] * g->rdims[2];
    for (int64_t t = 0; t < ntiles; t++) {
        int64_t tile[3];
        float sx[64], sy[64], sz[64];
        memset (sx, 0, sizeof sx);
        memset (sy, 0, sizeof sy);
        memset (sz, 0, sizeof sz);
        tile[2] = t / (g->rdims[0] * g->rdims[1]);
        tile[1] = (t - tile[2] * g->rdims[0] * g->rdims[1]) / g->rdims[0];
        tile[0] = t - tile[2] * g->rdims[0] * g->rdims[1]
            - tile[1] * g->rdims[0];
        for (q[2] = 0; q[2] < vpr[2]; q[2]++)
        for (q[1] = 0; q[1] < vpr[1]; q[1]++)
        for (q[0] = 0; q[0] < vpr[0]; q[0]++) {
            int skip = 0;
            for (int d = 0; d < 3; d++) {
                fijk[d] = g->roi_offset[d] + vpr[d] * tile[d] + q[d];
                if (fijk[d] >= g->roi_offset[d] + g->roi_dim[d]) skip = 1;
            }
            if (skip) continue;
            float fx3[3], dxyz[3], mijk[3], li1[3], li2[3], dc_dv[3];
            int64_t mf[3], mr[3];
            for (int d = 0; d < 3; d++)
                fx3[d] = g->img_origin[d] + fijk[0] * st[3*d+0]
                    + fijk[1] * st[3*d+1] + fijk[2] * st[3*d+2];
            if (g_froi && !inside_roi_f (fx3, g_froi)) continue;
            interp_pix_c (dxyz, g, coeff, tile, q, bx, by, bz);
            if (!correspond_roi_f (mijk, fx3, dxyz, mv)) continue;
            for (int d = 0; d < 3; d++)
                li_clamp_f (mijk[d], mv->dim[d] - 1, &mf[d], &mr[d],
                    &li1[d], &li2[d]);
            int64_t fidx = vidx (fx->dim, fijk[0], fijk[1], fijk[2]);
            int64_t mvf = vidx (mv->dim, mf[0], mf[1], mf[2]);
            mi_dc_dv (dc_dv, fh, mh, jh, fhp, mhp, f_img[fidx], m_img, mvf,
                mv, num_vox_f, smetric, li1, li2);
            update_sets_b (sx, sy, sz, q, dc_dv, bx, by, bz);
        }
        sort_sets (cx, cy, cz, sx, sy, sz, tile, g);
    }
    memset (grad, 0, sizeof(float) * g->num_coeff);
    condense (grad, cx, cy, cz, g->num_knots);
    *score = smetric;
    *num_vox_out = num_vox;
    free (bx); free (by); free (bz); free (cx); free (cy); free (cz);
    return 0;
}

typedef struct {
    const vol64* mv;
    const float* f_img;
    const float* m_img;
    const orc_hist* fhp;
    const orc_hist* mhp;
    double* fh; double* mh; double* jh;
    int pass;
    double num_vox_f;
    double smetric;
    int64_t num_vox;
} mi64_ctx;

static void
mi64_visit (void* vctx, int64_t fidx, const double fxyz[3],
    const double dxyz[3], double* dc_dv, int* has_grad)
{
    mi64_ctx* c = (mi64_ctx*) vctx;
    tri64 t = locate64 (fxyz, dxyz, c->mv);
    if (!t.ok || !moving_roi64 (fxyz, dxyz)) return;
    double w[8];
    corner_weights64 (w, &t);
    int fb = bin_of (c->f_img[fidx], c->fhp);
    int64_t off = (int64_t) fb * c->mhp->bins;
    if (c->pass == 1) {
        c->fh[fb] += 1.;
        for (int k = 0; k < 8; k++) {
            int mb = bin_of (c->m_img[corner_index (t.mvf, k, c->mv->dim)],
                c->mhp);
            c->mh[mb] += w[k];
            c->jh[off + mb] += w[k];
        }
        c->num_vox++;
        return;
    }
    double g[3] = {0, 0, 0};
    for (int k = 0; k < 8; k++) {
        int mb = bin_of (c->m_img[corner_index (t.mvf, k, c->mv->dim)],
            c->mhp);
        int64_t jb = off + mb;
        if (c->jh[jb] > 0.0001) {
            double dS = log (c->num_vox_f * c->jh[jb]
                / (c->fh[fb] * c->mh[mb])) - c->smetric;
            double sx = (k & 1) ? 1. : -1., sy = (k & 2) ? 1. : -1.;
            double sz = (k & 4) ? 1. : -1.;
            double wx = (k & 1) ? t.w2[0] : t.w1[0];
            double wy = (k & 2) ? t.w2[1] : t.w1[1];
            double wz = (k & 4) ? t.w2[2] : t.w1[2];
            g[0] -= sx * wy * wz * dS;
            g[1] -= wx * sy * wz * dS;
            g[2] -= wx * wy * sz * dS;
        }
    }
    for (int d = 0; d < 3; d++) g[d] /= c->num_vox_f;
    /* same in-place projection as the reference */
    const double* pr = c->mv->proj;
    g[0] = g[0] * pr[0] + g[1] * pr[1] + g[2] * pr[2];
    g[1] = g[0] * pr[3] + g[1] * pr[4] + g[2] * pr[5];
    g[2] = g[0] * pr[6] + g[1] * pr[7] + g[2] * pr[8];
    dc_dv[0] = g[0]; dc_dv[1] = g[1]; dc_dv[2] = g[2];
    *has_grad = 1;
}

/* Pass 1 alone over the grid's ROI: histograms (cleared first) and the
 * voxel count.  Summed over slabs that tile an ROI they give that ROI's
 * pass 1 (up to the order of the double additions). */
int
orc_mi_f64_pass1 (const orc_grid* g, const orc_vol* fixed, const float* f_img,
    const orc_vol* moving, const float* m_img, const float* coeff,
    const orc_hist* fhp, const orc_hist* mhp, int64_t* num_vox, double* fh,
    double* mh, double* jh)
{
    vol64 fx, mv;
    if (vol64_init (&fx, fixed) || vol64_init (&mv, moving)) return -1;
    memset (fh, 0, sizeof(double) * fhp->bins);
    memset (mh, 0, sizeof(double) * mhp->bins);
    memset (jh, 0, sizeof(double) * fhp->bins * mhp->bins);
    mi64_ctx c = { &mv, f_img, m_img, fhp, mhp, fh, mh, jh, 1, 0., 0., 0 };
    g_roi_pass1 = 1;
    tile_loop64 (g, &fx, coeff, mi64_visit, &c, 0);
    g_roi_pass1 = 0;
    *num_vox = c.num_vox;
    return 0;
}

/* Pass 2 over the grid's ROI with given histograms and voxel count (e.g.
 * summed over slabs): the score from them and this ROI's gradient. */
int
orc_mi_f64_pass2 (const orc_grid* g, const orc_vol* fixed, const float* f_img,
    const orc_vol* moving, const float* m_img, const float* coeff,
    const orc_hist* fhp, const orc_hist* mhp, int64_t num_vox,
    const double* fh, const double* mh, const double* jh, double* score,
    double* grad)
{
    vol64 fx, mv;
    if (vol64_init (&fx, fixed) || vol64_init (&mv, moving)) return -1;
    mi64_ctx c = { &mv, f_img, m_img, fhp, mhp, (double*) fh, (double*) mh,
        (double*) jh, 2, 0., 0., num_vox };
    double fnv = (double) num_vox, s = 0;
    double thresh = 0.001 / (mhp->bins * fhp->bins);
    for (int64_t jb = 0; jb < fhp->bins * mhp->bins; jb++) {
        int64_t mb = jb % mhp->bins, fb = jb / mhp->bins;
        if (jh[jb] > thresh) s -= jh[jb] * log (fnv * jh[jb] / (mh[mb] * fh[fb]));
    }
    c.smetric = s / fnv;
    c.num_vox_f = fnv;
    tile_loop64 (g, &fx, coeff, mi64_visit, &c, grad);
    *score = c.smetric;
    return 0;
}

int
orc_mi_f64 (const orc_grid* g, const orc_vol* fixed, const float* f_img,
    const orc_vol* moving, const float* m_img, const float* coeff,
    const orc_hist* fhp, const orc_hist* mhp, double* score, double* grad,
    int64_t* num_vox, double* fh, double* mh, double* jh)
{
    /* pass 1 scans the whole fixed image (see orc_mi_f32) */
    orc_grid g1 = *g;
    for (int d = 0; d < 3; d++) {
        if (g->roi_offset[d] != 0 || g->rdims[d] * g->vox_per_rgn[d]
            < fixed->dim[d]) return -2;
        g1.roi_dim[d] = fixed->dim[d];
    }
    int rc = orc_mi_f64_pass1 (&g1, fixed, f_img, moving, m_img, coeff, fhp,
        mhp, num_vox, fh, mh, jh);
    if (rc) return rc;
    return orc_mi_f64_pass2 (g, fixed, f_img, moving, m_img, coeff, fhp, mhp,
        *num_vox, fh, mh, jh, score, grad);
}

/* ------------------------------------------------------------------ */
/* Mattes MI with cubic B-spline Parzen windows                          */
/* ------------------------------------------------------------------ */

/* Plastimatch implements Mattes MI only with partial-volume (PVI-8)
 * binning; this is the Parzen-window form of the published method: Mattes,
 * Haynor, Vesselle, Lewellen, Eubank, "PET-CT image registration in the
 * chest using free-form deformations", IEEE Trans. Med. Imaging 22(1),
 * 120-128 (2003), section II.B-C.  The joint histogram takes a zero-order
 * B-spline window on the fixed intensity and a cubic B-spline window on
 * the moving intensity at the warped position; the marginals are its sums;
 * the cost is S = -sum p log(p / (p_f p_m)); and since the fixed marginal
 * does not depend on the transform,
 *   dS/dmu = 1/(N delta_m) sum_x [sum_k beta3'(k - u(x)) log(p(i(x), k) /
 *            p_m(k))] grad m(T(x)) . dT(x)/dmu,
 * with u(x) the moving value's continuous bin index.  The spatial gradient
 * is that of the trilinear interpolant, rotated to world coordinates
 * (proj^T times the index-space gradient), and zero along an axis where
 * li_clamp holds the position at the image's end (the value is constant
 * there). */

void
orc_parzen_init (orc_parzen* p, int64_t bins, const float* f_img, int64_t nf,
    const float* m_img, int64_t nm)
{
    float fmin = f_img[0], fmax = f_img[0], mmin = m_img[0], mmax = m_img[0];
    for (int64_t i = 1; i < nf; i++) {
        if (f_img[i] < fmin) fmin = f_img[i];
        if (f_img[i] > fmax) fmax = f_img[i];
    }
    for (int64_t i = 1; i < nm; i++) {
        if (m_img[i] < mmin) mmin = m_img[i];
        if (m_img[i] > mmax) mmax = m_img[i];
    }
    p->bins = bins;
    p->f_min = fmin;
    p->m_min = mmin;
    p->f_delta = fmax > fmin ? (fmax - fmin) / (float) (bins - 4) : 1.0f;
    p->m_delta = mmax > mmin ? (mmax - mmin) / (float) (bins - 4) : 1.0f;
}

/* centred cubic B-spline and its derivative */
static double
bspline3 (double t)
{
    double a = fabs (t);
    if (a < 1.0) return 2.0 / 3.0 - a * a + 0.5 * a * a * a;
    if (a < 2.0) return (2.0 - a) * (2.0 - a) * (2.0 - a) / 6.0;
    return 0.0;
}

static double
bspline3_d (double t)
{
    double a = fabs (t), sg = t < 0 ? -1.0 : 1.0;
    if (a < 1.0) return -2.0 * t + 1.5 * t * a;
    if (a < 2.0) return -sg * 0.5 * (2.0 - a) * (2.0 - a);
    return 0.0;
}

/* fixed bin in float arithmetic, as the device computes it */
static int64_t
parzen_fbin (const orc_parzen* p, float v)
{
    int64_t b = (int64_t) floorf ((v - p->f_min) / p->f_delta) + 2;
    if (b < 2) b = 2;
    if (b > p->bins - 3) b = p->bins - 3;
    return b;
}

typedef struct {
    const vol64* mv;
    const float* f_img;
    const float* m_img;
    const orc_parzen* p;
    double* jh;
    const double* lut;       /* pass 2: log(p / p_m) per joint bin */
    double scale;            /* pass 2: 1 / (N delta_m) */
    int pass;
    int64_t num_vox;
} parzen64_ctx;

static void
parzen64_visit (void* vctx, int64_t fidx, const double fxyz[3],
    const double dxyz[3], double* dc_dv, int* has_grad)
{
    parzen64_ctx* c = (parzen64_ctx*) vctx;
    tri64 t = locate64 (fxyz, dxyz, c->mv);
    if (!t.ok) return;
    const int64_t B = c->p->bins;
    double w[8], mval = 0, mk[8];
    corner_weights64 (w, &t);
    for (int k = 0; k < 8; k++) {
        mk[k] = c->m_img[corner_index (t.mvf, k, c->mv->dim)];
        mval += w[k] * mk[k];
    }
    const int64_t fb = parzen_fbin (c->p, c->f_img[fidx]);
    const double u = (mval - (double) c->p->m_min) / (double) c->p->m_delta + 2.0;
    int64_t k0 = (int64_t) floor (u);
    if (k0 > B - 3) k0 = B - 3;
    if (k0 < 1) k0 = 1;
    if (c->pass == 1) {
        for (int j = 0; j < 4; j++) {
            const int64_t kb = k0 - 1 + j;
            c->jh[fb * B + kb] += bspline3 ((double) kb - u);
        }
        c->num_vox++;
        return;
    }
    double s = 0;
    for (int j = 0; j < 4; j++) {
        const int64_t kb = k0 - 1 + j;
        s += bspline3_d ((double) kb - u) * c->lut[fb * B + kb];
    }
    /* index-space gradient of the trilinear interpolant, then proj^T */
    double gi[3] = {0, 0, 0};
    for (int k = 0; k < 8; k++) {
        double sx = (k & 1) ? 1. : -1., sy = (k & 2) ? 1. : -1.;
        double sz = (k & 4) ? 1. : -1.;
        double wx = (k & 1) ? t.w2[0] : t.w1[0];
        double wy = (k & 2) ? t.w2[1] : t.w1[1];
        double wz = (k & 4) ? t.w2[2] : t.w1[2];
        gi[0] += sx * wy * wz * mk[k];
        gi[1] += wx * sy * wz * mk[k];
        gi[2] += wx * wy * sz * mk[k];
    }
    /* where li_clamp holds the position, the value does not move with it */
    for (int d = 0; d < 3; d++) if (t.clamped[d]) gi[d] = 0;
    for (int j = 0; j < 3; j++) {
        double gw = 0;
        for (int d = 0; d < 3; d++) gw += c->mv->proj[3*d+j] * gi[d];
        dc_dv[j] = c->scale * s * gw;
    }
    *has_grad = 1;
}

int
orc_mi_parzen_f64 (const orc_grid* g, const orc_vol* fixed,
    const float* f_img, const orc_vol* moving, const float* m_img,
    const float* coeff, const orc_parzen* p, double* score, double* grad,
    int64_t* num_vox, double* jh)
{
    vol64 fx, mv;
    if (p->bins < 5 || vol64_init (&fx, fixed) || vol64_init (&mv, moving)) {
        return -1;
    }
    const int64_t B = p->bins;
    memset (jh, 0, sizeof(double) * B * B);
    parzen64_ctx c = { &mv, f_img, m_img, p, jh, 0, 0., 1, 0 };
    tile_loop64 (g, &fx, coeff, parzen64_visit, &c, 0);
    *num_vox = c.num_vox;
    if (c.num_vox < 1) {
        *score = FLT_MAX;
        memset (grad, 0, sizeof(double) * g->num_coeff);
        return 0;
    }
    const double N = (double) c.num_vox;
    double* pf = (double*) calloc (B, sizeof(double));
    double* pm = (double*) calloc (B, sizeof(double));
    double* lut = (double*) calloc (B * B, sizeof(double));
    for (int64_t i = 0; i < B; i++)
        for (int64_t k = 0; k < B; k++) {
            pf[i] += jh[i * B + k] / N;
            pm[k] += jh[i * B + k] / N;
        }
    double s = 0;
    for (int64_t i = 0; i < B; i++)
        for (int64_t k = 0; k < B; k++) {
            double pj = jh[i * B + k] / N;
            if (pj > 0) {
                s -= pj * log (pj / (pf[i] * pm[k]));
                lut[i * B + k] = log (pj / pm[k]);
            }
        }
    *score = s;
    c.pass = 2;
    c.lut = lut;
    c.scale = 1.0 / (N * (double) p->m_delta);
    tile_loop64 (g, &fx, coeff, parzen64_visit, &c, grad);
    free (pf);
    free (pm);
    free (lut);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Analytic regulariser                                                 */
/* ------------------------------------------------------------------ */

/* eval_integral (src/register/bspline_regularize_analytic.cxx:166-198):
 * V[j][i] = integral over one grid interval of the product of polynomial
 * rows j of Qn1 and i of Qn2. */
static void
eval_integral (double* V, const double* Qn1, const double* Qn2, double gs)
{
    double I[7] = { gs, (1.0/2.0)*(gs*gs), (1.0/3.0)*(gs*gs*gs),
        (1.0/4.0)*(gs*gs*gs*gs), (1.0/5.0)*(gs*gs*gs*gs*gs),
        (1.0/6.0)*(gs*gs*gs*gs*gs*gs), (1.0/7.0)*(gs*gs*gs*gs*gs*gs*gs) };
    for (int j = 0; j < 4; j++)
        for (int i = 0; i < 4; i++) {
            double S[16];
            for (int a = 0; a < 4; a++)
                for (int b = 0; b < 4; b++)
                    S[4*a+b] = Qn1[4*j+a] * Qn2[4*i+b];
            V[4*j+i] = (I[0] * S[0]) + (I[1] * (S[1] + S[4]))
                + (I[2] * (S[2] + S[5] + S[8]))
                + (I[3] * (S[3] + S[6] + S[9] + S[12]))
                + (I[4] * (S[7] + S[10] + S[13]))
                + (I[5] * (S[11] + S[14])) + (I[6] * (S[15]));
        }
}

static void
mat44 (double* out, const double* a, const double* b)
{
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            double s = 0;
            for (int k = 0; k < 4; k++) s += a[4*i+k] * b[4*k+j];
            out[4*i+j] = s;
        }
}

/* init_analytic (src/register/bspline_regularize_analytic.cxx:200-280):
 * Q[axis][order] = B * R(axis) * delta(order). */
static void
init_q (double Q[3][4][16], const orc_grid* g)
{
    static const double B[16] = {
        1.0/6.0, -1.0/2.0,  1.0/2.0, -1.0/6.0,
        2.0/3.0,  0.0    , -1.0    ,  1.0/2.0,
        1.0/6.0,  1.0/2.0,  1.0/2.0, -1.0/2.0,
        0.0    ,  0.0    ,  0.0    ,  1.0/6.0 };
    static const double D1[16] = { 0,0,0,0, 1,0,0,0, 0,2,0,0, 0,0,3,0 };
    static const double D2[16] = { 0,0,0,0, 0,0,0,0, 2,0,0,0, 0,6,0,0 };
    static const double D3[16] = { 0,0,0,0, 0,0,0,0, 0,0,0,0, 6,0,0,0 };
    for (int a = 0; a < 3; a++) {
        double r = 1.0 / g->grid_spac[a];
        double R[16] = { 1,0,0,0, 0,r,0,0, 0,0,r*r,0, 0,0,0,r*r*r };
        mat44 (Q[a][0], B, R);
        mat44 (Q[a][1], Q[a][0], D1);
        mat44 (Q[a][2], Q[a][0], D2);
        mat44 (Q[a][3], Q[a][0], D3);
    }
}

/* get_Vmatrix (src/register/bspline_regularize_analytic.cxx:282-337):
 * V = X (x) Y (x) Z over the tile's 64 knot slots. */
static void
get_vmatrix (double* V, const double* X, const double* Y, const double* Z)
{
    for (int a = 0; a < 4; a++) for (int b = 0; b < 4; b++)
    for (int c = 0; c < 4; c++) for (int d = 0; d < 4; d++)
    for (int e = 0; e < 4; e++) for (int f = 0; f < 4; f++)
        V[64*(16*a + 4*c + e) + (16*b + 4*d + f)]
            = X[4*a+b] * (Y[4*c+d] * Z[4*e+f]);
}

/* The 32 weighted V matrices of Bspline_regularize::analytic_init
 * (src/register/bspline_regularize_analytic.cxx:637-940): for each,
 * the (x, y, z) derivative orders of its two factors and its weight. */
typedef struct { int xa, xb, ya, yb, za, zb; int wsel; } vterm;

static const vterm VTERMS[32] = {
    {2,2, 0,0, 0,0, 0}, {0,0, 2,2, 0,0, 0}, {0,0, 0,0, 2,2, 0},
    {1,1, 1,1, 0,0, 1}, {1,1, 0,0, 1,1, 1}, {0,0, 1,1, 1,1, 1},
    {1,1, 0,0, 0,0, 2}, {0,0, 1,1, 0,0, 2}, {0,0, 0,0, 1,1, 2},
    {1,0, 0,1, 0,0, 3}, {0,1, 1,0, 0,0, 4}, {1,0, 0,0, 0,1, 3},
    {0,1, 0,0, 1,0, 4}, {0,0, 1,0, 0,1, 3}, {0,0, 0,1, 1,0, 4},
    {1,1, 0,0, 0,0, 5}, {0,0, 1,1, 0,0, 5}, {0,0, 0,0, 1,1, 5},
    {1,1, 0,0, 0,0, 6}, {0,0, 1,1, 0,0, 6}, {0,0, 0,0, 1,1, 6},
    {0,0, 0,0, 0,0, 7},
    {3,3, 0,0, 0,0, 8}, {0,0, 3,3, 0,0, 8}, {0,0, 0,0, 3,3, 8},
    {2,2, 1,1, 0,0, 8}, {2,2, 0,0, 1,1, 8}, {0,0, 2,2, 1,1, 8},
    {1,1, 2,2, 0,0, 8}, {1,1, 0,0, 2,2, 8}, {0,0, 1,1, 2,2, 8},
    {1,1, 1,1, 1,1, 8},
};

static double
vterm_weight (int wsel, const float* pen)
{
    float curv = pen[0], diff = pen[1], l1 = pen[2], l2 = pen[3];
    float disp = pen[4], third = pen[5], lem = pen[6], mixed = pen[7];
    switch (wsel) {
    case 0: return curv;
    case 1: return curv * mixed;
    case 2: return diff;
    case 3: return l1 * lem;
    case 4: return l2 * lem;
    case 5: return (lem) * (2*l1 + l2)/2;
    case 6: return (lem) * (l1)/2;
    case 7: return disp;
    case 8: return third;
    }
    return 0;
}

static double*
build_vmats (const orc_grid* g, const float* pen)
{
    double Q[3][4][16];
    init_q (Q, g);
    double* V = (double*) malloc (sizeof(double) * 32 * 4096);
    for (int t = 0; t < 32; t++) {
        const vterm* v = &VTERMS[t];
        double X[16], Y[16], Z[16];
        eval_integral (X, Q[0][v->xa], Q[0][v->xb], (double) g->grid_spac[0]);
        eval_integral (Y, Q[1][v->ya], Q[1][v->yb], (double) g->grid_spac[1]);
        eval_integral (Z, Q[2][v->za], Q[2][v->zb], (double) g->grid_spac[2]);
        get_vmatrix (&V[4096*t], X, Y, Z);
        double lam = vterm_weight (v->wsel, pen);
        for (int j = 0; j < 4096; j++) V[4096*t + j] = lam * V[4096*t + j];
    }
    return V;
}

/* region_smoothness_omp / region_smoothness_elastic_omp
 * (src/register/bspline_regularize_analytic.cxx:362-397, 516-600) for one
 * tile: returns S, accumulates dS/dp into sets[64*3]. */
static double
region_plain (double* sets, const double* Vt, const float* coeff,
    const int64_t* knots)
{
    double S = 0.0;
    double X[64] = {0}, Y[64] = {0}, Z[64] = {0};
    for (int j = 0; j < 64; j++) {
        for (int i = 0; i < 64; i++) {
            X[j] += coeff[3*knots[i]+0] * Vt[64*j + i];
            Y[j] += coeff[3*knots[i]+1] * Vt[64*j + i];
            Z[j] += coeff[3*knots[i]+2] * Vt[64*j + i];
        }
        S += X[j] * coeff[3*knots[j]+0];
        S += Y[j] * coeff[3*knots[j]+1];
        S += Z[j] * coeff[3*knots[j]+2];
        sets[3*j+0] += 2 * X[j];
        sets[3*j+1] += 2 * Y[j];
        sets[3*j+2] += 2 * Z[j];
    }
    return S;
}

static double
region_elastic (double* sets, const double* V, const float* coeff,
    const int64_t* knots)
{
    double S = 0.0;
    const double *V9 = &V[4096*9], *V10 = &V[4096*10], *V11 = &V[4096*11];
    const double *V12 = &V[4096*12], *V13 = &V[4096*13], *V14 = &V[4096*14];
    const double *V15 = &V[4096*15], *V16 = &V[4096*16], *V17 = &V[4096*17];
    const double *V18 = &V[4096*18], *V19 = &V[4096*19], *V20 = &V[4096*20];
    for (int j = 0; j < 64; j++) {
        double X1=0,Y1=0,X2=0,Y2=0,X3=0,Z3=0,X4=0,Z4=0,Y5=0,Z5=0,Y6=0,Z6=0;
        double X7=0,Y7=0,Z7=0,X8=0,Y8=0,Z8=0,X9=0,Y9=0,Z9=0;
        for (int i = 0; i < 64; i++) {
            double cx = coeff[3*knots[i]+0], cy = coeff[3*knots[i]+1];
            double cz = coeff[3*knots[i]+2];
            int o = 64*j + i;
            X1 += cx * V9[o];  X2 += cx * V10[o]; X3 += cx * V11[o];
            X4 += cx * V12[o]; Y5 += cy * V13[o]; Y6 += cy * V14[o];
            Y1 += cy * V9[o];  Y2 += cy * V10[o]; Z3 += cz * V11[o];
            Z4 += cz * V12[o]; Z5 += cz * V13[o]; Z6 += cz * V14[o];
            X7 += cx * V15[o]; Y8 += cy * V16[o]; Z9 += cz * V17[o];
            Y7 += cy * V18[o]; Z7 += cz * V18[o]; X8 += cx * V19[o];
            Z8 += cz * V19[o]; X9 += cx * V20[o]; Y9 += cy * V20[o];
        }
        double cx = coeff[3*knots[j]+0], cy = coeff[3*knots[j]+1];
        double cz = coeff[3*knots[j]+2];
        S += X1 * cy; S += X2 * cy; S += X3 * cz; S += X4 * cz;
        S += Y5 * cz; S += Y6 * cz; S += X7 * cx; S += Y8 * cy;
        S += Z9 * cz; S += Y7 * cy; S += Z7 * cz; S += X8 * cx;
        S += Z8 * cz; S += X9 * cx; S += Y9 * cy;
        sets[3*j+0] += Y1 + Y2 + Z3 + Z4 + 2 * X7 + 2 * X8 + 2 * X9;
        sets[3*j+1] += X1 + X2 + Z5 + Z6 + 2 * Y8 + 2 * Y7 + 2 * Y9;
        sets[3*j+2] += X3 + X4 + Y5 + Y6 + 2 * Z9 + 2 * Z7 + 2 * Z8;
    }
    return S;
}

/* One tile, terms in the reference's order: V0..V8, the elastic group
 * V9..V20, then V21..V31 (src/register/bspline_regularize_analytic.cxx:
 * 968-996).  The per-term partial scores are summed as the reference's
 * `S += region_smoothness_omp (...)` does. */
static double
region (double* sets, const double* V, const float* coeff,
    const int64_t* knots)
{
    double S = 0.0;
    for (int t = 0; t <= 8; t++)
        S += region_plain (sets, &V[4096*t], coeff, knots);
    S += region_elastic (sets, V, coeff, knots);
    for (int t = 21; t < 32; t++)
        S += region_plain (sets, &V[4096*t], coeff, knots);
    return S;
}

/* compute_score_analytic_omp (src/register/bspline_regularize_analytic.cxx:
 * 942-1007): the V matrices applied tile by tile in the reference's order
 * (all 21 plain terms, then the elastic group, then the last 11).  The
 * double per-tile sets are condensed per knot (reg_update_grad,
 * :122-137) into a float gradient when out_f != 0, else a double one. */
static int
reg_common (const orc_grid* g, const float* coeff, const float* pen,
    double* rmetric, float* out_f, double* out_d)
{
    double* V = build_vmats (g, pen);
    int64_t n = g->rdims[0] * g->rdims[1] * g->rdims[2];
    size_t csz = (size_t) 3 * 64 * g->num_knots;
    double* cond = (double*) calloc (csz, sizeof(double));
    if (!V || !cond) return -1;
    const int64_t* cd = g->cdims;
    double S = 0;
    for (int64_t t = 0; t < n; t++) {
        int64_t knots[64], tl[3];
        int64_t ntx = cd[0] - 3, nty = cd[1] - 3, ntz = cd[2] - 3;
        tl[0] = t % ntx;
        tl[1] = ((t - tl[0]) / ntx) % nty;
        tl[2] = (((t - tl[0]) / ntx) / nty) % ntz;
        int idx = 0;
        for (int k = 0; k < 4; k++)
            for (int j = 0; j < 4; j++)
                for (int i = 0; i < 4; i++)
                    knots[idx++] = cd[0]*cd[1]*(tl[2]+k) + cd[0]*(tl[1]+j)
                        + (tl[0]+i);
        double sets[3*64];
        memset (sets, 0, sizeof sets);
        S += region (sets, V, coeff, knots);
        for (int s = 0; s < 64; s++) {
            cond[3*(64*knots[s]+s)+0] = sets[3*s+0];
            cond[3*(64*knots[s]+s)+1] = sets[3*s+1];
            cond[3*(64*knots[s]+s)+2] = sets[3*s+2];
        }
    }
    for (int64_t k = 0; k < g->num_knots; k++) {
        for (int s = 0; s < 64; s++) {
            for (int c = 0; c < 3; c++) {
                if (out_f) out_f[3*k+c] += cond[3*(64*k+s)+c];
                else out_d[3*k+c] += cond[3*(64*k+s)+c];
            }
        }
    }
    *rmetric = S;
    free (V);
    free (cond);
    return 0;
}

int
orc_reg_f32 (const orc_grid* g, const float* coeff, const float pen[8],
    float* rmetric, float* grad)
{
    double S;
    memset (grad, 0, sizeof(float) * g->num_coeff);
    int rc = reg_common (g, coeff, pen, &S, grad, 0);
    *rmetric = (float) S;
    return rc;
}

int
orc_reg_f64 (const orc_grid* g, const float* coeff, const float pen[8],
    double* rmetric, double* grad)
{
    memset (grad, 0, sizeof(double) * g->num_coeff);
    return reg_common (g, coeff, pen, rmetric, 0, grad);
}

/* ------------------------------------------------------------------ */
/* Dense vector field and warp                                          */
/* ------------------------------------------------------------------ */

/* Field at one voxel from the q_lut weights of its offset in the tile:
 * bspline_interp_pix / bspline_interp_pix_b
 * (src/base/bspline_interpolate.cxx:21-76), knots in (k, j, i) order. */
static inline void
interp_pix_q (float out[3], const orc_grid* g, const float* coeff,
    const int64_t p[3], const float* q)
{
    const int64_t* cd = g->cdims;
    int m = 0;
    out[0] = out[1] = out[2] = 0;
    for (int k = 0; k < 4; k++)
        for (int j = 0; j < 4; j++)
            for (int i = 0; i < 4; i++, m++) {
                int64_t cidx = 3 * ((p[2] + k) * cd[1] * cd[0]
                    + (p[1] + j) * cd[0] + (p[0] + i));
                out[0] += q[m] * coeff[cidx+0];
                out[1] += q[m] * coeff[cidx+1];
                out[2] += q[m] * coeff[cidx+2];
            }
}

/* bspline_interpolate_vf (src/base/bspline_interpolate.cxx:112-142): the
 * field at every ROI voxel (tile and offset counted from the ROI corner),
 * zero elsewhere; vf is xyz-interleaved over the fixed image. */
int
orc_interpolate_vf (const orc_grid* g, const orc_vol* fixed,
    const float* coeff, float* vf)
{
    const int64_t* vpr = g->vox_per_rgn;
    const int64_t* dim = fixed->dim;
    float* q_lut = (float*) malloc (sizeof(float) * 64 * vpr[0] * vpr[1] * vpr[2]);
    if (!q_lut) return -1;
    orc_q_lut (q_lut, vpr);
    memset (vf, 0, sizeof(float) * 3 * dim[0] * dim[1] * dim[2]);
    for (int64_t k = 0; k < g->roi_dim[2]; k++)
    for (int64_t j = 0; j < g->roi_dim[1]; j++)
    for (int64_t i = 0; i < g->roi_dim[0]; i++) {
        int64_t p[3] = {i / vpr[0], j / vpr[1], k / vpr[2]};
        int64_t qidx = (i % vpr[0]) + vpr[0] * ((j % vpr[1])
            + vpr[1] * (k % vpr[2]));
        int64_t v = (k + g->roi_offset[2]) * dim[0] * dim[1]
            + (j + g->roi_offset[1]) * dim[0] + (i + g->roi_offset[0]);
        interp_pix_q (&vf[3*v], g, coeff, p, &q_lut[qidx*64]);
    }
    free (q_lut);
    return 0;
}

/* bspline_warp_dcos with linear interpolation on a float image
 * (src/base/bspline_warp.cxx:28-160): every fixed voxel gets the trilinear
 * moving value at its displaced position, or default_val outside the
 * moving image; positions advance along x as LOOP_X does.  The reference
 * takes the tile from the absolute voxel index, so this is defined only
 * when the ROI is the whole image (returns -2 otherwise).  vf_out (may be
 * NULL) receives the field. */
int
orc_warp (const orc_grid* g, const orc_vol* fx, const orc_vol* mv,
    const float* m_img, const float* coeff, float default_val, float* out,
    float* vf_out)
{
    const int64_t* vpr = g->vox_per_rgn;
    const int64_t* dim = fx->dim;
    for (int d = 0; d < 3; d++)
        if (g->roi_offset[d] != 0 || g->roi_dim[d] != dim[d]) return -2;
    float* q_lut = (float*) malloc (sizeof(float) * 64 * vpr[0] * vpr[1] * vpr[2]);
    if (!q_lut) return -1;
    orc_q_lut (q_lut, vpr);
    int64_t npix = dim[0] * dim[1] * dim[2];
    for (int64_t v = 0; v < npix; v++) out[v] = default_val;
    if (vf_out) memset (vf_out, 0, sizeof(float) * 3 * npix);
    const float* st = fx->step;
    const float* org = fx->origin;
    int64_t fijk[3];
    float fxyz[3];
    for (fijk[2] = 0; fijk[2] < dim[2]; fijk[2]++) {
        fxyz[2] = org[2] + fijk[2] * st[2*3+2];
        for (fijk[1] = 0, fxyz[1] = org[1] + fijk[2] * st[1*3+2];
             fijk[1] < dim[1];
             ++fijk[1],
             fxyz[2] = org[2] + fijk[2] * st[2*3+2] + fijk[1] * st[2*3+1],
             fxyz[1] = org[1] + fijk[2] * st[1*3+2] + fijk[1] * st[1*3+1]) {
            for (fijk[0] = 0,
                 fxyz[0] = org[0] + fijk[2] * st[0*3+2] + fijk[1] * st[0*3+1];
                 fijk[0] < dim[0];
                 ++fijk[0], fxyz[0] += st[0], fxyz[1] += st[3],
                 fxyz[2] += st[6]) {
                int64_t p[3], qidx;
                float dxyz[3], mijk[3], li1[3], li2[3];
                int64_t mf[3], mr[3];
                for (int d = 0; d < 3; d++) p[d] = fijk[d] / vpr[d];
                qidx = (fijk[0] % vpr[0]) + vpr[0] * ((fijk[1] % vpr[1])
                    + vpr[1] * (fijk[2] % vpr[2]));
                interp_pix_q (dxyz, g, coeff, p, &q_lut[qidx*64]);
                int64_t fv = vidx (dim, fijk[0], fijk[1], fijk[2]);
                if (vf_out) {
                    vf_out[3*fv+0] = dxyz[0];
                    vf_out[3*fv+1] = dxyz[1];
                    vf_out[3*fv+2] = dxyz[2];
                }
                if (!correspond_f (mijk, fxyz, dxyz, mv)) continue;
                for (int d = 0; d < 3; d++)
                    li_clamp_f (mijk[d], mv->dim[d] - 1, &mf[d], &mr[d],
                        &li1[d], &li2[d]);
                out[fv] = li_value_f (li1, li2,
                    vidx (mv->dim, mf[0], mf[1], mf[2]), m_img, mv->dim);
            }
        }
    }
    free (q_lut);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Pyramid resampling                                                   */
/* ------------------------------------------------------------------ */

static int64_t
round_long (double x)       /* ROUND_PLM_LONG (src/sys/plm_math.h:53-54) */
{
    return (x >= 0) ? (int64_t) (x + 0.5) : (int64_t) (-(-x + 0.5));
}

/* Output geometry of registration_resample_volume
 * (src/register/registration_resample.cxx:12-59) for resample type mode:
 * 0 voxel rate (volume_subsample_vox, src/base/volume_resample.cxx:297-315),
 * 1 voxel rate, legacy (volume_subsample_vox_legacy, :337-357),
 * 2 millimetres (volume_resample_spacing, :381-393),
 * 3 percent (volume_resample_percent, :395-413).
 * Returns 1 when the reference clones the input instead (voxel rate 1). */
int
orc_resample_geometry (const int64_t dim[3], const float origin[3],
    const float spacing[3], int mode, const float rate[3],
    int64_t odim[3], float oorigin[3], float ospacing[3])
{
    if ((mode == 0 || mode == 1) && rate[0] == 1.0f && rate[1] == 1.0f
        && rate[2] == 1.0f) {
        for (int d = 0; d < 3; d++) {
            odim[d] = dim[d]; oorigin[d] = origin[d]; ospacing[d] = spacing[d];
        }
        return 1;
    }
    for (int d = 0; d < 3; d++) {
        if (mode == 0) {
            int64_t r = round_long (rate[d]);
            odim[d] = (dim[d] + r - 1) / r;
            oorigin[d] = origin[d];
            ospacing[d] = spacing[d] * r;
        } else if (mode == 1) {
            float in_size = dim[d] * spacing[d];
            odim[d] = dim[d] / (int64_t) rate[d];
            if (odim[d] < 1) odim[d] = 1;
            ospacing[d] = in_size / odim[d];
            oorigin[d] = (float) (origin[d] - 0.5 * spacing[d]
                + 0.5 * ospacing[d]);
        } else if (mode == 2) {
            float in_size = (dim[d] - 1) * spacing[d];
            odim[d] = 1 + round_long (in_size / rate[d]);
            oorigin[d] = origin[d];
            ospacing[d] = rate[d];
        } else {
            float in_size = (dim[d] - 1) * spacing[d];
            odim[d] = 1 + round_long (rate[d] * (dim[d] - 1));
            ospacing[d] = odim[d] == 1 ? in_size : in_size / (odim[d] - 1);
            oorigin[d] = origin[d];
        }
    }
    return 0;
}

/* volume_resample_float_li (src/base/volume_resample.cxx:70-136): output
 * positions advance by the output spacing from the output origin (direction
 * cosines ignored, as the reference does), the input index is
 * (position - origin) / spacing, a voxel whose rounded index falls outside
 * the input is 0, the rest are trilinear (li_clamp, LI_VALUE). */
void
orc_resample_li (const int64_t idim[3], const float iorigin[3],
    const float ispacing[3], const float* in, const int64_t odim[3],
    const float oorigin[3], const float ospacing[3], float* out)
{
    int64_t v = 0;
    float x, y, z, ijk[3];
    int64_t k, j, i;
    for (k = 0, z = oorigin[2]; k < odim[2]; k++, z += ospacing[2]) {
        ijk[2] = (z - iorigin[2]) / ispacing[2];
        int64_t zi = round_long (ijk[2]);
        for (j = 0, y = oorigin[1]; j < odim[1]; j++, y += ospacing[1]) {
            ijk[1] = (y - iorigin[1]) / ispacing[1];
            int64_t yi = round_long (ijk[1]);
            for (i = 0, x = oorigin[0]; i < odim[0]; i++, x += ospacing[0], v++) {
                ijk[0] = (x - iorigin[0]) / ispacing[0];
                int64_t xi = round_long (ijk[0]);
                if (zi < 0 || zi >= idim[2] || yi < 0 || yi >= idim[1]
                    || xi < 0 || xi >= idim[0]) {
                    out[v] = 0.0f;
                    continue;
                }
                int64_t f[3], r[3];
                float l1[3], l2[3];
                for (int d = 0; d < 3; d++)
                    li_clamp_f (ijk[d], idim[d] - 1, &f[d], &r[d], &l1[d],
                        &l2[d]);
                out[v] = li_value_f (l1, l2, vidx (idim, f[0], f[1], f[2]),
                    in, idim);
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* Landmarks                                                          */

/* Bspline_landmarks::initialize (src/register/bspline_landmarks.cxx:
 * 150-204): landmark position relative to the image origin, projected to
 * voxel coordinates by the fixed image's proj matrix (PROJECT_X/Y/Z,
 * src/base/volume_macros.h:76-81), truncated toward zero, split into tile
 * and offset by vox_per_rgn.  The tile comes from the absolute voxel
 * index, not from the ROI. */
int64_t
orc_landmarks_init (const orc_grid* g, const orc_vol* fixed,
    const float* fixed_xyz, int64_t n, int64_t* p, int64_t* q)
{
    for (int64_t l = 0; l < n; l++) {
        float xyz[3];
        for (int d = 0; d < 3; d++) {
            xyz[d] = fixed_xyz[3*l+d] - g->img_origin[d];
        }
        for (int d = 0; d < 3; d++) {
            const float* pr = fixed->proj + 3 * d;
            float ijk = xyz[0] * pr[0] + xyz[1] * pr[1] + xyz[2] * pr[2];
            if (!(ijk > -1.f && ijk < (float) g->img_dim[d])) return l + 1;
            int64_t v = (int64_t) ijk;
            if (v < 0 || v >= g->img_dim[d]) return l + 1;
            p[3*l+d] = v / g->vox_per_rgn[d];
            q[3*l+d] = v % g->vox_per_rgn[d];
        }
    }
    return 0;
}

/* bspline_landmarks_score_a (src/register/bspline_landmarks.cxx:25-134):
 * field at the landmark (bspline_interp_pix over q_lut,
 * src/base/bspline_interpolate.cxx:21-48), residual moving - (fixed +
 * field), squared distance summed in float, dc/dv = -(stiffness / n) *
 * residual added to the 64 knots (Bspline_score::update_grad,
 * src/register/bspline_score.cxx:117-143); lmetric = sum / n. */
void
orc_landmarks_f32 (const orc_grid* g, const float* coeff, int64_t n,
    const float* fixed_xyz, const float* moving_xyz, const int64_t* p,
    const int64_t* q, float stiffness, float* lmetric, float* grad)
{
    const int64_t* vpr = g->vox_per_rgn;
    const int64_t* cd = g->cdims;
    float* q_lut = (float*) malloc (sizeof(float) * 64
        * vpr[0] * vpr[1] * vpr[2]);
    orc_q_lut (q_lut, vpr);
    float land_score = 0.f;
    const float land_grad_coeff = stiffness / (float) n;
    for (int64_t l = 0; l < n; l++) {
        const int64_t* pl = p + 3 * l;
        const int64_t qidx = q[3*l+0] + vpr[0] * (q[3*l+1] + vpr[1] * q[3*l+2]);
        const float* ql = q_lut + 64 * qidx;
        float dxyz[3] = {0.f, 0.f, 0.f};
        int m = 0;
        for (int k = 0; k < 4; k++)
            for (int j = 0; j < 4; j++)
                for (int i = 0; i < 4; i++) {
                    int64_t cidx = 3 * ((pl[2] + k) * cd[1] * cd[0]
                        + (pl[1] + j) * cd[0] + (pl[0] + i));
                    dxyz[0] += ql[m] * coeff[cidx+0];
                    dxyz[1] += ql[m] * coeff[cidx+1];
                    dxyz[2] += ql[m] * coeff[cidx+2];
                    m++;
                }
        float diff[3], dc_dv[3];
        for (int d = 0; d < 3; d++) {
            float mxyz = fixed_xyz[3*l+d] + dxyz[d];
            diff[d] = moving_xyz[3*l+d] - mxyz;
        }
        float l_dist = diff[0]*diff[0] + diff[1]*diff[1] + diff[2]*diff[2];
        land_score += l_dist;
        for (int d = 0; d < 3; d++) dc_dv[d] = - land_grad_coeff * diff[d];
        m = 0;
        for (int k = 0; k < 4; k++)
            for (int j = 0; j < 4; j++)
                for (int i = 0; i < 4; i++) {
                    int64_t cidx = 3 * ((pl[2] + k) * cd[1] * cd[0]
                        + (pl[1] + j) * cd[0] + (pl[0] + i));
                    grad[cidx+0] += dc_dv[0] * ql[m];
                    grad[cidx+1] += dc_dv[1] * ql[m];
                    grad[cidx+2] += dc_dv[2] * ql[m];
                    m++;
                }
    }
    free (q_lut);
    *lmetric = land_score / (float) n;
}
