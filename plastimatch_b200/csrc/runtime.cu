// Host runtime of libplastimatch_b200: the C ABI declared in
// include/plastimatch_b200.h.
//
// A context owns every device buffer one registration stage needs
// (allocated in b200bsp_create / b200bsp_set_images, none afterwards), the
// geometry in the reference's float arithmetic, and a CUDA stream.  One
// evaluation is a short fixed sequence of kernel launches on that stream:
//   [H2D coefficients] -> tile kernel (FP32 or tensor-core form)
//   -> reduce_score -> gather_grad -> [D2H score + gradient]
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/plastimatch_b200.h"
#include "kernels.cuh"
#include "mi.cuh"
#include "regularize.cuh"

using namespace b200;

static thread_local std::string g_create_error;
// b200bsp_debug_fail_alloc: the n-th device allocation of the next
// b200bsp_create calls on this thread fails as if the device were full
static thread_local int g_fail_alloc = 0;

struct b200bsp_ctx {
    int device = 0;
    b200bsp_opts opts;
    b200bsp_volume fixed, moving;
    b200bsp_grid grid;
    BspGeom geom;
    int64_t num_coeff = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;

    float* d_fixed = nullptr;
    float* d_moving = nullptr;
    float* d_mgrad = nullptr;
    float* d_out = nullptr;           // field / warp staging (host outputs)
    float4* d_mgrad4 = nullptr;       // TC form, nearest gradient: padded copy
    float* d_coeff = nullptr;
    float* d_luts = nullptr;
    float* d_grad = nullptr;
    double* d_grad64 = nullptr;
    float* d_part = nullptr;
    double* d_score_part = nullptr;
    int* d_count_part = nullptr;
    DevResult* d_res = nullptr;
    int* d_err = nullptr;
    void* d_qlut = nullptr;
    float* d_inv_dc = nullptr;
    DevResult* h_res = nullptr;
    DevResult* h_res_dev = nullptr;   // device alias of h_res (mapped)
    float* h_scalar = nullptr;

    PartLayout lay;
    TcPlan plan;
    // the x-lane tensor-core MSE kernel (mse_xl.cu): pinned, chosen by the
    // autotuner, or needed for image ROIs; pref_xl is the choice without
    // ROIs, restored when they are removed
    bool use_xl = false;
    bool pref_xl = false;
    bool has_xl = false;
    XlPlan xplan;
    PartLayout xlay;
    void* d_xtab = nullptr;
    unsigned wait_limit = XL_DEFAULT_WAIT_LIMIT;
    int withhold_mma = 0;     // b200bsp_set_wait_limit's testing aid
    // b200bsp_score's device path: the regulariser on a second stream,
    // overlapping the tile kernel, its gradient kept in double
    double* d_reg_grad64 = nullptr;
    float* d_total = nullptr;
    int tc_grid = 0;          // CTAs of the tile kernel; 0: plan.grid
    int sm_count = 148;
    // bumped by every change to what an evaluation launches (kernel
    // choice, ROIs, images, wait limit, grid): a recorded graph of
    // evaluations is stale once it moves
    unsigned gen = 0;
    // b200bsp_score's regulariser: a second stream, and the fork and join
    // of it around the MSE kernel
    cudaStream_t aux_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // the optimiser's device workspace, kept between runs (optimize.cu)
    void* opt_ws = nullptr;
    void (*opt_ws_free) (void*) = nullptr;
    int nscore_parts = 0;
    bool images_set = false;

    MiState mi;
    RegState reg;

    // image ROIs (b200bsp_set_roi): the fixed ROI's test per fixed voxel,
    // the moving ROI's mask; geom.fmask / geom.mroi point at them
    uint8_t* d_fmask = nullptr;
    uint8_t* d_mroi = nullptr;

    // landmark pairs (b200bsp_set_landmarks)
    int lm_n = 0;
    float lm_stiffness = 1.f;
    int* d_lm_p = nullptr;            // tile of each fixed landmark [3n]
    float* d_lm_w = nullptr;          // its q_lut row [64n]
    float* d_lm_fm = nullptr;         // fixed xyz, moving xyz [6n]
    float* d_lm_dc = nullptr;         // dc/dv + squared distance [4n], lmetric

    bool timing = false;
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    float last_total_ms = 0.f, last_main_ms = 0.f;
    int last_launches = 0;
    std::string err;
};

// ------------------------------------------------------------------ util --

static int
fail (b200bsp_ctx* c, int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start (ap, fmt);
    vsnprintf (buf, sizeof buf, fmt, ap);
    va_end (ap);
    if (c) c->err = buf; else g_create_error = buf;
    return code;
}

// SMs left to b200bsp_score's regulariser beside the MSE kernel
constexpr int REG_SIDE_SMS = 12;

#define CK(call)                                                        \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) {                                        \
            return fail (c, e_ == cudaErrorMemoryAllocation             \
                ? B200BSP_E_OOM : B200BSP_E_CUDA, "%s: %s", #call,      \
                cudaGetErrorString (e_));                               \
        }                                                               \
    } while (0)

static bool
is_device_ptr (const void* p)
{
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes (&a, p) != cudaSuccess) {
        cudaGetLastError ();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Device address of host memory the GPU can write in place (page-locked and
// mapped, as cudaMallocHost / cudaHostAlloc memory is under unified
// addressing), else nullptr.
static void*
mapped_alias (void* p)
{
    if (!p) return nullptr;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes (&a, p) != cudaSuccess) {
        cudaGetLastError ();
        return nullptr;
    }
    return a.type == cudaMemoryTypeHost ? a.devicePointer : nullptr;
}

// Make `p` the context's tensor-core plan: the partial-gradient layout of
// its batches and the number of score parts follow it.
static void
use_tc_plan (b200bsp_ctx* c, const TcPlan& p)
{
    const BspGeom& g = c->geom;
    c->plan = p;
    PartLayout& L = c->lay;
    L.bx = p.bx; L.by = 1; L.bz = 1;
    L.nbx = (g.rdims[0] + L.bx - 1) / L.bx;
    L.nby = g.rdims[1];
    L.nbz = g.rdims[2];
    L.kx = L.bx + 3; L.ky = 4; L.kz = 4;
    L.slots = 1;
    c->nscore_parts = p.nbatches;
}

// Make `p` the context's x-lane plan and batch layout.
static void
use_xl_plan (b200bsp_ctx* c, const XlPlan& p)
{
    const BspGeom& g = c->geom;
    c->xplan = p;
    PartLayout& L = c->xlay;
    L.bx = p.T; L.by = 1; L.bz = 1;
    L.nbx = p.nbx; L.nby = g.rdims[1]; L.nbz = g.rdims[2];
    L.kx = p.T + 3; L.ky = 4; L.kz = 4;
    L.slots = 1;
}

// Cofactor inverse in float (Plastimatch src/base/direction_cosines.cxx:
// 135-158); the caller rejects |det| < 1e-8 as the reference does.
static bool
inv3f (float* out, const float* m)
{
    float det = m[0]*(m[4]*m[8]-m[5]*m[7]) - m[1]*(m[3]*m[8]-m[5]*m[6])
        + m[2]*(m[3]*m[7]-m[4]*m[6]);
    if (std::fabs (det) < 1e-8) return false;
    out[0] =  (m[4]*m[8]-m[5]*m[7]) / det;
    out[1] = -(m[1]*m[8]-m[2]*m[7]) / det;
    out[2] =  (m[1]*m[5]-m[2]*m[4]) / det;
    out[3] = -(m[3]*m[8]-m[5]*m[6]) / det;
    out[4] =  (m[0]*m[8]-m[2]*m[6]) / det;
    out[5] = -(m[0]*m[5]-m[2]*m[3]) / det;
    out[6] =  (m[3]*m[7]-m[4]*m[6]) / det;
    out[7] = -(m[0]*m[7]-m[1]*m[6]) / det;
    out[8] =  (m[0]*m[4]-m[1]*m[3]) / det;
    return true;
}

// Cubic B-spline basis table bx/by/bz_lut[vpr*4] as Bspline_xform::allocate
// builds it (src/base/bspline_xform.cxx:73-99, 468-482): float argument,
// double evaluation, rounded to float.
static void
basis_lut (float* lut, int vpr)
{
    for (int j = 0; j < 4; j++) {
        for (int v = 0; v < vpr; v++) {
            float i = (float) v / vpr;
            double r = 0;
            switch (j) {
            case 0: r = (1.0/6.0) * (- 1.0 * i*i*i + 3.0 * i*i - 3.0 * i + 1.0); break;
            case 1: r = (1.0/6.0) * (+ 3.0 * i*i*i - 6.0 * i*i + 4.0); break;
            case 2: r = (1.0/6.0) * (- 3.0 * i*i*i + 3.0 * i*i + 3.0 * i + 1.0); break;
            case 3: r = (1.0/6.0) * (+ 1.0 * i*i*i); break;
            }
            lut[v*4+j] = (float) r;
        }
    }
}

// ------------------------------------------------------------- lifecycle --

extern "C" void
b200bsp_default_opts (b200bsp_opts* o)
{
    memset (o, 0, sizeof *o);
    o->form = B200BSP_FORM_TC;
    o->mse_grad = B200BSP_MSE_GRAD_NEAREST;
    o->mi_bins = 32;
    o->device = 0;
}

extern "C" const char*
b200bsp_version (void)
{
    return "plastimatch_b200 0.1 (sm_100a)";
}

static int
check_volume (const b200bsp_volume* v, const char* what)
{
    long long n = 1;
    for (int d = 0; d < 3; d++) {
        if (v->dim[d] < 2) {
            return fail (nullptr, B200BSP_E_BADARG,
                "%s: dim[%d] = %lld, need >= 2", what, d, (long long) v->dim[d]);
        }
        if (!(v->spacing[d] != 0.f) || !std::isfinite (v->spacing[d])) {
            return fail (nullptr, B200BSP_E_BADARG, "%s: bad spacing", what);
        }
        n *= v->dim[d];
    }
    if (n >= (1LL << 31)) {
        return fail (nullptr, B200BSP_E_UNSUPPORTED,
            "%s: %lld voxels; volumes must have < 2^31 voxels", what, n);
    }
    return B200BSP_OK;
}

static void
free_all (b200bsp_ctx* c)
{
    cudaFree (c->d_fixed); cudaFree (c->d_moving); cudaFree (c->d_mgrad);
    cudaFree (c->d_out);
    cudaFree (c->d_mgrad4);
    if (c->ev_fork) cudaEventDestroy (c->ev_fork);
    if (c->ev_join) cudaEventDestroy (c->ev_join);
    if (c->aux_stream) cudaStreamDestroy (c->aux_stream);
    cudaFree (c->d_coeff); cudaFree (c->d_luts); cudaFree (c->d_grad);
    cudaFree (c->d_grad64); cudaFree (c->d_part); cudaFree (c->d_score_part);
    cudaFree (c->d_count_part); cudaFree (c->d_res); cudaFree (c->d_err);
    cudaFree (c->d_qlut); cudaFree (c->d_xtab); cudaFree (c->d_inv_dc);
    cudaFree (c->d_lm_p); cudaFree (c->d_lm_w); cudaFree (c->d_lm_fm);
    cudaFree (c->d_lm_dc);
    cudaFree (c->d_fmask); cudaFree (c->d_mroi);
    cudaFreeHost (c->h_res); cudaFreeHost (c->h_scalar);
    mi_free (&c->mi);
    reg_free (&c->reg);
    if (c->opt_ws_free) c->opt_ws_free (c->opt_ws);
    c->opt_ws = nullptr;
    for (auto& e : c->ev) if (e) cudaEventDestroy (e);
    cudaFree (c->d_reg_grad64);
    cudaFree (c->d_total);
    if (c->own_stream) cudaStreamDestroy (c->own_stream);
}

namespace b200 {

// The checks and geometry of b200bsp_create for the context-free
// b200bsp_score_mse_static: fills g and the three basis tables (x, y, z
// back to back, *nlut floats).  Errors go to the no-context error text.
int
static_geometry (const b200bsp_volume* fixed, const b200bsp_volume* moving,
    const b200bsp_grid* grid, BspGeom* out, float* luts, int* nlut)
{
    int rc = check_volume (fixed, "fixed");
    if (rc) return rc;
    rc = check_volume (moving, "moving");
    if (rc) return rc;
    for (int d = 0; d < 3; d++) {
        if (grid->vox_per_rgn[d] < 1 || grid->vox_per_rgn[d] > 64
            || grid->roi_dim[d] < 1 || grid->roi_offset[d] < 0
            || grid->roi_offset[d] + grid->roi_dim[d] > fixed->dim[d]) {
            return fail (nullptr, B200BSP_E_BADARG,
                "grid axis %d: need 1 <= vox_per_rgn <= 64 and the ROI "
                "inside the fixed image", d);
        }
    }
    float finv[9], minv[9];
    if (!inv3f (finv, fixed->dcos) || !inv3f (minv, moving->dcos)) {
        return fail (nullptr, B200BSP_E_BADARG,
            "singular matrix of direction cosines");
    }
    BspGeom g = {};
    long long ntiles = 1, nknots = 1;
    for (int d = 0; d < 3; d++) {
        g.fdim[d] = (int) fixed->dim[d];
        g.img_origin[d] = fixed->origin[d];
        g.mdim[d] = (int) moving->dim[d];
        g.morigin[d] = moving->origin[d];
        g.minv_spacing[d] = (float) (1.0 / moving->spacing[d]);
        g.roi_off[d] = (int) grid->roi_offset[d];
        g.roi_dim[d] = (int) grid->roi_dim[d];
        g.vpr[d] = (int) grid->vox_per_rgn[d];
        g.rdims[d] = 1 + (g.roi_dim[d] - 1) / g.vpr[d];
        g.cdims[d] = g.rdims[d] + 3;
        g.m_hi[d] = (float) moving->dim[d] - 0.5f;
        g.m_fmax[d] = (float) (moving->dim[d] - 2);
        ntiles *= g.rdims[d];
        nknots *= g.cdims[d];
    }
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) {
            g.fstep[3*i+j] = fixed->dcos[3*i+j] * fixed->spacing[j];
            g.mproj[3*i+j] = minv[3*i+j] / moving->spacing[i];
        }
    }
    g.ntiles = (int) ntiles;
    g.nknots = (int) nknots;
    basis_lut (luts, g.vpr[0]);
    basis_lut (luts + 4 * g.vpr[0], g.vpr[1]);
    basis_lut (luts + 4 * (g.vpr[0] + g.vpr[1]), g.vpr[2]);
    *nlut = 4 * (g.vpr[0] + g.vpr[1] + g.vpr[2]);
    *out = g;
    return B200BSP_OK;
}

int
static_fail (int code, const char* msg)
{
    return fail (nullptr, code, "%s", msg);
}

// The stream a context's work is ordered on (its own or the caller's).
cudaStream_t
ctx_stream (const b200bsp_ctx* c)
{
    return c->stream;
}

int
ctx_device (const b200bsp_ctx* c)
{
    return c->device;
}

// Landmark count (0: none set) and stiffness, for the optimiser's
// objective.
int
ctx_landmarks (const b200bsp_ctx* c, float* stiffness)
{
    if (stiffness) *stiffness = c->lm_stiffness;
    return c->lm_n;
}

unsigned
ctx_generation (const b200bsp_ctx* c)
{
    return c->gen;
}

// The optimiser's workspace slot: kept by the context, freed with it.
void*
ctx_opt_ws (const b200bsp_ctx* c)
{
    return c->opt_ws;
}

void
ctx_set_opt_ws (b200bsp_ctx* c, void* ws, void (*release) (void*))
{
    if (c->opt_ws_free && c->opt_ws && c->opt_ws != ws) {
        c->opt_ws_free (c->opt_ws);
    }
    c->opt_ws = ws;
    c->opt_ws_free = release;
}

// The device-side error flag of the tile kernel (nullptr for the FP32
// form, which has no bounded waits).
int*
ctx_err_flag (b200bsp_ctx* c)
{
    return c->opts.form == B200BSP_FORM_TC ? c->d_err : nullptr;
}

// Record a device error flag read by a caller that checked it (clears it).
int
ctx_report_device_error (b200bsp_ctx* c, int e)
{
    if (!e) return B200BSP_OK;
    cudaMemsetAsync (c->d_err, 0, sizeof (int), c->stream);
    return fail (c, B200BSP_E_TIMEOUT,
        "a bounded device-side wait gave up (code %d)", e);
}

} // namespace b200

extern "C" int
b200bsp_create (const b200bsp_volume* fixed, const b200bsp_volume* moving,
    const b200bsp_grid* grid, const b200bsp_opts* opts, b200bsp_ctx** out)
{
    b200bsp_ctx* c = nullptr;
    if (!fixed || !moving || !grid || !out) {
        return fail (nullptr, B200BSP_E_BADARG, "null argument");
    }
    *out = nullptr;
    int rc = check_volume (fixed, "fixed");
    if (rc) return rc;
    rc = check_volume (moving, "moving");
    if (rc) return rc;
    b200bsp_opts o;
    if (opts) o = *opts; else b200bsp_default_opts (&o);
    if (o.form != B200BSP_FORM_TC && o.form != B200BSP_FORM_FP32) {
        return fail (nullptr, B200BSP_E_BADARG, "unknown form %d", o.form);
    }
    if (o.mse_grad != 0 && o.mse_grad != 1) {
        return fail (nullptr, B200BSP_E_BADARG, "unknown mse_grad %d", o.mse_grad);
    }
    if (o.mi_window != B200BSP_MI_PVI8 && o.mi_window != B200BSP_MI_PARZEN) {
        return fail (nullptr, B200BSP_E_BADARG, "unknown mi_window %d",
            o.mi_window);
    }
    if (o.mi_window == B200BSP_MI_PARZEN && o.mi_bins < 5) {
        return fail (nullptr, B200BSP_E_BADARG,
            "Parzen-window MI needs at least 5 bins");
    }
    if (o.mi_hist != B200BSP_MI_HIST_EQSP && o.mi_hist != B200BSP_MI_HIST_VOPT) {
        return fail (nullptr, B200BSP_E_BADARG, "unknown mi_hist %d", o.mi_hist);
    }
    if (o.mi_hist == B200BSP_MI_HIST_VOPT && o.mi_window != B200BSP_MI_PVI8) {
        return fail (nullptr, B200BSP_E_BADARG,
            "V-optimal bins are a PVI-8 histogram type");
    }
    if (o.mi_bins < 2 || o.mi_bins > MI_MAX_BINS) {
        return fail (nullptr, B200BSP_E_BADARG, "mi_bins must be in [2, %d]",
            MI_MAX_BINS);
    }
    for (int d = 0; d < 3; d++) {
        if (grid->vox_per_rgn[d] < 1 || grid->vox_per_rgn[d] > 64
            || grid->roi_dim[d] < 1 || grid->roi_offset[d] < 0
            || grid->roi_offset[d] + grid->roi_dim[d] > fixed->dim[d]) {
            return fail (nullptr, B200BSP_E_BADARG,
                "grid axis %d: need 1 <= vox_per_rgn <= 64 and the ROI "
                "inside the fixed image", d);
        }
    }
    int ndev = 0;
    if (cudaGetDeviceCount (&ndev) != cudaSuccess || o.device < 0
        || o.device >= ndev) {
        cudaGetLastError ();
        return fail (nullptr, B200BSP_E_CUDA, "no CUDA device %d", o.device);
    }

    c = new b200bsp_ctx ();
    c->opts = o;
    c->fixed = *fixed;
    c->moving = *moving;
    c->grid = *grid;
    c->device = o.device;
    if (cudaSetDevice (o.device) != cudaSuccess) {
        delete c;
        return fail (nullptr, B200BSP_E_CUDA, "cudaSetDevice failed");
    }

    // Geometry in the reference's float arithmetic.
    BspGeom& g = c->geom;
    float finv[9], minv[9];
    if (!inv3f (finv, fixed->dcos) || !inv3f (minv, moving->dcos)) {
        delete c;
        return fail (nullptr, B200BSP_E_BADARG,
            "singular matrix of direction cosines");
    }
    long long ntiles = 1, nknots = 1;
    for (int d = 0; d < 3; d++) {
        g.fdim[d] = (int) fixed->dim[d];
        g.img_origin[d] = fixed->origin[d];
        g.mdim[d] = (int) moving->dim[d];
        g.morigin[d] = moving->origin[d];
        g.minv_spacing[d] = (float) (1.0 / moving->spacing[d]);
        g.roi_off[d] = (int) grid->roi_offset[d];
        g.roi_dim[d] = (int) grid->roi_dim[d];
        g.vpr[d] = (int) grid->vox_per_rgn[d];
        g.rdims[d] = 1 + (g.roi_dim[d] - 1) / g.vpr[d];
        g.cdims[d] = g.rdims[d] + 3;
        g.m_hi[d] = (float) moving->dim[d] - 0.5f;
        g.m_fmax[d] = (float) (moving->dim[d] - 2);
        ntiles *= g.rdims[d];
        nknots *= g.cdims[d];
    }
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) {
            g.fstep[3*i+j] = fixed->dcos[3*i+j] * fixed->spacing[j];
            g.mproj[3*i+j] = minv[3*i+j] / moving->spacing[i];
        }
    }
    g.ntiles = (int) ntiles;
    g.nknots = (int) nknots;
    c->num_coeff = 3 * nknots;

    // Device buffers that do not depend on the form.
    size_t nf = (size_t) g.fdim[0] * g.fdim[1] * g.fdim[2];
    size_t nm = (size_t) g.mdim[0] * g.mdim[1] * g.mdim[2];
    int rc2 = B200BSP_OK;
    auto alloc = [&](void** p, size_t bytes) {
        if (rc2) return;
        if (g_fail_alloc > 0 && --g_fail_alloc == 0) {
            rc2 = fail (c, B200BSP_E_OOM, "cudaMalloc(%zu): injected failure",
                bytes);
            return;
        }
        cudaError_t e = cudaMalloc (p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError ();
            rc2 = fail (c, B200BSP_E_OOM, "cudaMalloc(%zu): %s", bytes,
                cudaGetErrorString (e));
        }
    };
    alloc ((void**) &c->d_fixed, nf * sizeof (float));
    alloc ((void**) &c->d_moving, nm * sizeof (float));
    if (o.mse_grad == 0) alloc ((void**) &c->d_mgrad, 3 * nm * sizeof (float));
    int sm_count = 148;
    cudaDeviceGetAttribute (&sm_count, cudaDevAttrMultiProcessorCount, o.device);
    c->sm_count = sm_count;
    if (o.tc_kernel < 0 || o.tc_kernel > B200BSP_TC_KERNEL_TILE) {
        rc2 = fail (c, B200BSP_E_BADARG, "tc_kernel %d unknown", o.tc_kernel);
    } else if (o.form == B200BSP_FORM_TC
               && o.tc_kernel != B200BSP_TC_KERNEL_TILE) {
        // AUTO starts on the tile kernel (the faster one where both were
        // measured: 256x256x128 at vpr 5 and 64^3 at vpr 8); image ROIs
        // and the autotuner move it to the x-lane kernel
        c->has_xl = xl_plan (g, &c->xplan, sm_count);
        c->use_xl = c->pref_xl = c->has_xl
            && o.tc_kernel == B200BSP_TC_KERNEL_XLANE;
        if (!c->has_xl && o.tc_kernel == B200BSP_TC_KERNEL_XLANE) {
            rc2 = fail (c, B200BSP_E_UNSUPPORTED,
                "x-lane kernel: vox_per_rgn[1] = %d outside 3..10", g.vpr[1]);
        }
    }
    if (o.wait_limit < 0) {
        rc2 = fail (c, B200BSP_E_BADARG, "wait_limit must be >= 0");
    } else if (o.wait_limit > 0) {
        c->wait_limit = (unsigned) o.wait_limit;
    }
    // the tile kernel's 16-byte moving-gradient copy, wherever the tile
    // kernel may run
    if (o.mse_grad == 0 && o.form == B200BSP_FORM_TC
        && !(c->has_xl && o.tc_kernel == B200BSP_TC_KERNEL_XLANE)) {
        alloc ((void**) &c->d_mgrad4, nm * sizeof (float4));
    }
    alloc ((void**) &c->d_coeff, c->num_coeff * sizeof (float));
    alloc ((void**) &c->d_grad, c->num_coeff * sizeof (float));
    alloc ((void**) &c->d_grad64, c->num_coeff * sizeof (double));
    alloc ((void**) &c->d_reg_grad64, c->num_coeff * sizeof (double));
    alloc ((void**) &c->d_total, sizeof (float));
    alloc ((void**) &c->d_res, sizeof (DevResult));
    alloc ((void**) &c->d_err, sizeof (int));
    alloc ((void**) &c->d_inv_dc, 9 * sizeof (float));
    int nlut = 4 * (g.vpr[0] + g.vpr[1] + g.vpr[2]);
    alloc ((void**) &c->d_luts, nlut * sizeof (float));
    if (!rc2 && (cudaMallocHost ((void**) &c->h_res, sizeof (DevResult)) != cudaSuccess
        || cudaMallocHost ((void**) &c->h_scalar, 64) != cudaSuccess)) {
        cudaGetLastError ();
        rc2 = fail (c, B200BSP_E_OOM, "cudaMallocHost failed");
    }
    if (!rc2 && cudaHostGetDevicePointer ((void**) &c->h_res_dev, c->h_res, 0)
        != cudaSuccess) {
        cudaGetLastError ();
        c->h_res_dev = nullptr;          // result block then comes by copy
    }

    // Tile partial-gradient layout of the chosen form.
    size_t part_elems = 0;
    size_t score_parts = 0;
    if (!rc2 && o.form == B200BSP_FORM_TC) {
        if (!tc_plan (g, &c->plan, 2, sm_count)) {
            rc2 = fail (c, B200BSP_E_UNSUPPORTED,
                "tensor-core form: grid with vox_per_rgn (%d,%d,%d) not "
                "supported; use B200BSP_FORM_FP32", g.vpr[0], g.vpr[1], g.vpr[2]);
        } else {
            // buffers for every batch split the autotuner may choose
            for (int e = 0; e <= TC_TUNE_MAX_EXTRA; e++) {
                TcPlan p;
                if (!tc_plan (g, &p, 2, sm_count, e)) continue;
                part_elems = std::max (part_elems,
                    (size_t) p.nbatches * (p.bx + 3) * 16 * 3);
                score_parts = std::max (score_parts, (size_t) p.nbatches);
            }
            use_tc_plan (c, c->plan);
            if (c->has_xl) {
                for (int e = 0; e <= TC_TUNE_MAX_EXTRA; e++) {
                    XlPlan xp;
                    if (!xl_plan (g, &xp, sm_count, e)) continue;
                    part_elems = std::max (part_elems,
                        (size_t) xp.nbatches * (xp.T + 3) * 16 * 3);
                    score_parts = std::max (score_parts,
                        (size_t) xp.score_parts);
                }
                use_xl_plan (c, c->xplan);
            }
        }
    } else if (!rc2) {
        if (mse_fp32_smem_bytes (g) > 200 * 1024) {
            rc2 = fail (c, B200BSP_E_UNSUPPORTED, "tile too large");
        }
        PartLayout& L = c->lay;
        L.bx = L.by = L.bz = 1;
        L.nbx = g.rdims[0]; L.nby = g.rdims[1]; L.nbz = g.rdims[2];
        L.kx = L.ky = L.kz = 4;
        L.slots = 64;
        part_elems = (size_t) 64 * g.ntiles * 3;
        c->nscore_parts = g.ntiles;
    }
    alloc ((void**) &c->d_part, part_elems * sizeof (float));
    score_parts = std::max (score_parts, (size_t) std::max (c->nscore_parts, 1));
    alloc ((void**) &c->d_score_part, score_parts * sizeof (double));
    alloc ((void**) &c->d_count_part, score_parts * sizeof (int));
    if (!rc2 && o.form == B200BSP_FORM_TC) {
        rc2 = tc_build_tables (c->geom, c->plan, &c->d_qlut);
        if (rc2) rc2 = fail (c, rc2, "tensor-core tables: %s", cudaGetErrorString (cudaGetLastError ()));
    }
    if (!rc2 && mi_alloc (&c->mi, c->geom, o.mi_bins, o.mi_window,
            o.mi_hist)) {
        rc2 = fail (c, B200BSP_E_OOM, "MI buffers: out of device memory");
    }
    if (!rc2) {
        // Bspline_xform::grid_spac = vox_per_rgn * |spacing| (float)
        float gsp[3];
        for (int d = 0; d < 3; d++) {
            gsp[d] = (float) g.vpr[d] * std::fabs (c->fixed.spacing[d]);
        }
        if (reg_alloc (&c->reg, c->geom, gsp)) {
            rc2 = fail (c, B200BSP_E_OOM, "regulariser buffers");
        }
    }
    if (rc2) {
        g_create_error = c->err;
        free_all (c);
        delete c;
        return rc2;
    }

    if (cudaStreamCreateWithFlags (&c->own_stream, cudaStreamNonBlocking)
        != cudaSuccess
        || cudaStreamCreateWithFlags (&c->aux_stream, cudaStreamNonBlocking)
        != cudaSuccess
        || cudaEventCreateWithFlags (&c->ev_fork, cudaEventDisableTiming)
        != cudaSuccess
        || cudaEventCreateWithFlags (&c->ev_join, cudaEventDisableTiming)
        != cudaSuccess) {
        cudaGetLastError ();
        free_all (c);
        delete c;
        return fail (nullptr, B200BSP_E_CUDA, "stream create failed");
    }
    c->stream = c->own_stream;

    std::vector<float> luts (nlut);
    basis_lut (luts.data (), g.vpr[0]);
    basis_lut (luts.data () + 4 * g.vpr[0], g.vpr[1]);
    basis_lut (luts.data () + 4 * (g.vpr[0] + g.vpr[1]), g.vpr[2]);
    if (c->has_xl) {
        int rt = xl_build_table (g, c->xplan, luts.data (), &c->d_xtab);
        if (rt) {
            cudaGetLastError ();
            free_all (c);
            delete c;
            return fail (nullptr, rt, "tensor-core x-lane table");
        }
    }
    cudaMemcpy (c->d_luts, luts.data (), nlut * sizeof (float),
        cudaMemcpyHostToDevice);
    cudaMemcpy (c->d_inv_dc, minv, 9 * sizeof (float), cudaMemcpyHostToDevice);
    cudaMemset (c->d_err, 0, sizeof (int));
    if (cudaDeviceSynchronize () != cudaSuccess) {
        std::string e = cudaGetErrorString (cudaGetLastError ());
        free_all (c);
        delete c;
        return fail (nullptr, B200BSP_E_CUDA, "setup: %s", e.c_str ());
    }
    *out = c;
    return B200BSP_OK;
}

extern "C" int
b200bsp_set_wait_limit (b200bsp_ctx* c, int polls, int withhold_mma)
{
    if (!c) return B200BSP_E_BADARG;
    if (polls < 0) return fail (c, B200BSP_E_BADARG, "polls must be >= 0");
    if (withhold_mma && !(c->opts.form == B200BSP_FORM_TC && c->use_xl)) {
        return fail (c, B200BSP_E_UNSUPPORTED,
            "withholding MMAs is a testing aid of the x-lane kernel");
    }
    c->wait_limit = polls > 0 ? (unsigned) polls : XL_DEFAULT_WAIT_LIMIT;
    c->withhold_mma = withhold_mma ? 1 : 0;
    c->gen++;
    return B200BSP_OK;
}

extern "C" void
b200bsp_debug_fail_alloc (int nth)
{
    g_fail_alloc = nth > 0 ? nth : 0;
}

extern "C" int
b200bsp_destroy (b200bsp_ctx* c)
{
    if (!c) return B200BSP_OK;
    cudaSetDevice (c->device);
    if (c->stream) cudaStreamSynchronize (c->stream);
    free_all (c);
    delete c;
    return B200BSP_OK;
}

extern "C" int
b200bsp_grid_info (const b200bsp_ctx* c, int64_t rdims[3], int64_t cdims[3],
    int64_t* num_coeff)
{
    if (!c) return B200BSP_E_BADARG;
    for (int d = 0; d < 3; d++) {
        if (rdims) rdims[d] = c->geom.rdims[d];
        if (cdims) cdims[d] = c->geom.cdims[d];
    }
    if (num_coeff) *num_coeff = c->num_coeff;
    return B200BSP_OK;
}

extern "C" int
b200bsp_set_stream (b200bsp_ctx* c, void* stream)
{
    if (!c) return B200BSP_E_BADARG;
    c->stream = stream ? (cudaStream_t) stream : c->own_stream;
    return B200BSP_OK;
}

static cudaMemcpyKind
kind_to_dev (const void* src)
{
    return is_device_ptr (src) ? cudaMemcpyDeviceToDevice
                               : cudaMemcpyHostToDevice;
}

extern "C" int
b200bsp_set_images (b200bsp_ctx* c, const float* fixed_img,
    const float* moving_img, const float* moving_grad)
{
    if (!c || !fixed_img || !moving_img) {
        return fail (c, B200BSP_E_BADARG, "null image");
    }
    c->gen++;
    CK (cudaSetDevice (c->device));
    const BspGeom& g = c->geom;
    size_t nf = (size_t) g.fdim[0] * g.fdim[1] * g.fdim[2];
    size_t nm = (size_t) g.mdim[0] * g.mdim[1] * g.mdim[2];
    CK (cudaMemcpyAsync (c->d_fixed, fixed_img, nf * sizeof (float),
        kind_to_dev (fixed_img), c->stream));
    CK (cudaMemcpyAsync (c->d_moving, moving_img, nm * sizeof (float),
        kind_to_dev (moving_img), c->stream));
    if (c->opts.mse_grad == 0) {
        if (moving_grad) {
            CK (cudaMemcpyAsync (c->d_mgrad, moving_grad, 3 * nm * sizeof (float),
                kind_to_dev (moving_grad), c->stream));
        } else {
            float sp[3] = {c->moving.spacing[0], c->moving.spacing[1],
                c->moving.spacing[2]};
            CK (launch_volume_grad (g.mdim, sp, c->d_inv_dc, c->d_moving,
                c->d_mgrad, c->stream));
        }
        if (c->d_mgrad4) {
            CK (launch_pad_grad4 (c->d_mgrad, c->d_mgrad4, (long long) nm,
                c->stream));
        }
    }
    int rc = mi_set_images (&c->mi, g, c->d_fixed, c->d_moving, nf, nm,
        c->stream);
    if (rc) return fail (c, rc, "MI histogram setup failed");
    CK (cudaStreamSynchronize (c->stream));
    c->images_set = true;
    return B200BSP_OK;
}

// ------------------------------------------------------------ evaluation --

struct OutPtrs {
    bool dev;
    float* grad;
    double* grad64;
    float* score;
    double* score64;
    long long* nvox;
};

static int
begin_eval (b200bsp_ctx* c, const float* coeff, const float** dcoeff)
{
    if (!c) return B200BSP_E_BADARG;
    if (!c->images_set) return fail (c, B200BSP_E_STATE, "images not set");
    if (!coeff) return fail (c, B200BSP_E_BADARG, "null coefficients");
    CK (cudaSetDevice (c->device));
    if (is_device_ptr (coeff)) {
        *dcoeff = coeff;
    } else {
        CK (cudaMemcpyAsync (c->d_coeff, coeff, c->num_coeff * sizeof (float),
            cudaMemcpyHostToDevice, c->stream));
        *dcoeff = c->d_coeff;
    }
    if (c->timing) {
        if (!c->ev[0]) {
            for (auto& e : c->ev) CK (cudaEventCreate (&e));
        }
        CK (cudaEventRecord (c->ev[0], c->stream));
    }
    c->last_launches = 0;
    return B200BSP_OK;
}

static int
mark_main_done (b200bsp_ctx* c)
{
    if (c->timing) CK (cudaEventRecord (c->ev[1], c->stream));
    return B200BSP_OK;
}

static int
end_eval (b200bsp_ctx* c, bool wait)
{
    if (c->timing) CK (cudaEventRecord (c->ev[2], c->stream));
    if (wait) CK (cudaStreamSynchronize (c->stream));
    if (c->timing && wait) {
        cudaEventElapsedTime (&c->last_main_ms, c->ev[0], c->ev[1]);
        cudaEventElapsedTime (&c->last_total_ms, c->ev[0], c->ev[2]);
    }
    return B200BSP_OK;
}

// The MSE tile pass + reductions, results left in d_res and the given
// gradient outputs (device pointers).
static int
run_mse (b200bsp_ctx* c, const float* dcoeff, float* grad_out,
    double* grad64_out, float* score_out, double* score64_out,
    long long* nvox_out, DevResult* res_host = nullptr,
    const FinishCombine& combine = FinishCombine (),
    cudaEvent_t before_finish = nullptr,
    const std::function<int ()>& after_main = nullptr)
{
    const BspGeom& g = c->geom;
    if (c->opts.form == B200BSP_FORM_FP32) {
        CK (launch_mse_fp32 (g, c->opts.mse_grad, c->d_fixed, c->d_moving,
            c->d_mgrad, dcoeff, c->d_luts, c->d_part, c->d_score_part,
            c->d_count_part, c->stream));
    } else if (c->use_xl) {
        XlPlan plan = c->xplan;
        // a batch's share of the SMs' CTA slots counts two per SM (the
        // tile kernel's); this kernel runs one CTA per SM
        if (c->tc_grid > 0) {
            plan.grid = std::min (std::max (1, c->tc_grid / 2), plan.nbatches);
        }
        CK (launch_mse_xl (g, plan, c->opts.mse_grad, c->d_fixed,
            c->d_moving, c->d_mgrad, dcoeff, c->d_xtab, c->d_luts,
            c->d_part, c->d_score_part, c->d_count_part, c->d_err,
            c->wait_limit, c->withhold_mma, c->stream));
    } else {
        TcPlan plan = c->plan;
        if (c->tc_grid > 0) plan.grid = std::min (c->tc_grid, plan.nbatches);
        CK (launch_mse_tc (g, plan, c->opts.mse_grad, c->d_fixed,
            c->d_moving, c->d_mgrad, c->d_mgrad4, dcoeff, c->d_qlut,
            c->d_part, c->d_score_part, c->d_count_part, c->d_err,
            c->wait_limit, c->stream));
    }
    c->last_launches++;
    int rc = mark_main_done (c);
    if (rc) return rc;
    if (after_main) {
        rc = after_main ();
        if (rc) return rc;
    }
    const bool xl = c->opts.form == B200BSP_FORM_TC && c->use_xl;
    if (before_finish) CK (cudaStreamWaitEvent (c->stream, before_finish, 0));
    CK (launch_finish_mse (g, xl ? c->xlay : c->lay, c->d_part,
        c->d_score_part, c->d_count_part,
        xl ? c->xplan.score_parts : c->nscore_parts,
        c->opts.form == B200BSP_FORM_TC ? c->d_err : nullptr, c->d_res,
        res_host, grad_out, grad64_out, score_out, score64_out, nvox_out,
        c->stream, nullptr, 0, combine));
    c->last_launches += 1;
    return B200BSP_OK;
}

// e: the tile kernel's error flag as the finish kernel copied it into the
// result block; -1 reads it from the device.
static int
check_device_error (b200bsp_ctx* c, int e = -1)
{
    if (c->opts.form != B200BSP_FORM_TC) return B200BSP_OK;
    if (e < 0) {
        e = 0;
        CK (cudaMemcpy (&e, c->d_err, sizeof (int), cudaMemcpyDeviceToHost));
    }
    if (e) {
        cudaMemset (c->d_err, 0, sizeof (int));
        return fail (c, B200BSP_E_TIMEOUT,
            "a bounded device-side wait gave up (code %d)", e);
    }
    return B200BSP_OK;
}

extern "C" int
b200bsp_score_mse (b200bsp_ctx* c, const float* coeff, float* score,
    float* grad, int64_t* num_vox)
{
    const float* dcoeff = nullptr;
    int rc = begin_eval (c, coeff, &dcoeff);
    if (rc) return rc;
    bool dev_out = is_device_ptr (grad) && (!score || is_device_ptr (score))
        && (!num_vox || is_device_ptr (num_vox));
    if (dev_out && is_device_ptr (coeff)) {
        rc = run_mse (c, dcoeff, grad, nullptr, score, nullptr,
            (long long*) num_vox);
        if (rc) return rc;
        return end_eval (c, false);
    }
    // Host outputs: the finish kernel writes the gradient and the result
    // block straight into page-locked mapped memory when it can, else they
    // come back by copy.
    float* g_map = (float*) mapped_alias (grad);
    float* g_dev = is_device_ptr (grad) ? grad : g_map ? g_map : c->d_grad;
    rc = run_mse (c, dcoeff, g_dev, nullptr, nullptr, nullptr, nullptr,
        c->h_res_dev);
    if (rc) return rc;
    if (!c->h_res_dev) {
        CK (cudaMemcpyAsync (c->h_res, c->d_res, sizeof (DevResult),
            cudaMemcpyDeviceToHost, c->stream));
    }
    if (grad && g_dev == c->d_grad) {
        CK (cudaMemcpyAsync (grad, c->d_grad, c->num_coeff * sizeof (float),
            cudaMemcpyDeviceToHost, c->stream));
    }
    rc = end_eval (c, true);
    if (rc) return rc;
    if (score) *score = c->h_res->score_f;
    if (num_vox) *num_vox = c->h_res->num_vox;
    return check_device_error (c, c->h_res->error);
}

extern "C" int
b200bsp_score_mse_f64 (b200bsp_ctx* c, const float* coeff, double* score,
    double* grad, int64_t* num_vox)
{
    const float* dcoeff = nullptr;
    int rc = begin_eval (c, coeff, &dcoeff);
    if (rc) return rc;
    double* g_out = is_device_ptr (grad) ? grad : (double*) mapped_alias (grad);
    rc = run_mse (c, dcoeff, nullptr, g_out ? g_out : c->d_grad64, nullptr,
        nullptr, nullptr, c->h_res_dev);
    if (rc) return rc;
    if (!c->h_res_dev) {
        CK (cudaMemcpyAsync (c->h_res, c->d_res, sizeof (DevResult),
            cudaMemcpyDeviceToHost, c->stream));
    }
    if (grad && !g_out) {
        CK (cudaMemcpyAsync (grad, c->d_grad64, c->num_coeff * sizeof (double),
            cudaMemcpyDeviceToHost, c->stream));
    }
    rc = end_eval (c, true);
    if (rc) return rc;
    if (score) *score = c->h_res->score;
    if (num_vox) *num_vox = c->h_res->num_vox;
    return check_device_error (c, c->h_res->error);
}

extern "C" int
b200bsp_autotune (b200bsp_ctx* c, const float* coeff, int evals, int* tiles)
{
    if (!c) return B200BSP_E_BADARG;
    if (evals < 1) return fail (c, B200BSP_E_BADARG, "evals must be >= 1");
    c->gen++;
    if (c->opts.form != B200BSP_FORM_TC) {
        if (tiles) *tiles = 1;
        return B200BSP_OK;
    }
    const float* dcoeff = nullptr;
    int rc = begin_eval (c, coeff, &dcoeff);
    if (rc) return rc;
    int sm_count = 148;
    cudaDeviceGetAttribute (&sm_count, cudaDevAttrMultiProcessorCount,
        c->device);
    cudaEvent_t e0, e1;
    CK (cudaEventCreate (&e0));
    CK (cudaEventCreate (&e1));
    const TcPlan start = c->plan;
    const bool start_xl = c->use_xl;
    TcPlan best = start;
    bool best_xl = start_xl;
    float best_ms = 0.f;
    auto time_it = [&](float* ms) {
        int r = run_mse (c, dcoeff, c->d_grad, nullptr, nullptr, nullptr,
            nullptr);                                    // warm-up
        if (!r && cudaEventRecord (e0, c->stream) != cudaSuccess) r = B200BSP_E_CUDA;
        for (int i = 0; i < evals && !r; i++) {
            r = run_mse (c, dcoeff, c->d_grad, nullptr, nullptr, nullptr,
                nullptr);
        }
        if (!r && (cudaEventRecord (e1, c->stream) != cudaSuccess
                || cudaEventSynchronize (e1) != cudaSuccess
                || cudaEventElapsedTime (ms, e0, e1) != cudaSuccess)) {
            r = B200BSP_E_CUDA;
        }
        return r;
    };
    // candidates: the x-lane kernel, then each batch split of the tile
    // kernel; ties keep the earlier candidate
    const XlPlan xstart = c->xplan;
    XlPlan xbest = xstart;
    for (int e = 0; e <= TC_TUNE_MAX_EXTRA && c->has_xl && !rc; e++) {
        XlPlan xp;
        if (!xl_plan (c->geom, &xp, sm_count, e)) continue;
        use_xl_plan (c, xp);
        c->use_xl = true;
        float ms = 0.f;
        rc = time_it (&ms);
        if (!rc && (best_ms == 0.f || ms < best_ms)) {
            best_ms = ms;
            best_xl = true;
            xbest = xp;
        }
    }
    c->use_xl = false;
    const bool roi = c->geom.fmask || c->geom.mroi;
    const bool tile_ok = !roi && !(c->has_xl
        && c->opts.tc_kernel == B200BSP_TC_KERNEL_XLANE);
    for (int e = 0; e <= TC_TUNE_MAX_EXTRA && !rc && tile_ok; e++) {
        TcPlan p;
        if (!tc_plan (c->geom, &p, 2, sm_count, e)) continue;
        use_tc_plan (c, p);
        float ms = 0.f;
        rc = time_it (&ms);
        if (!rc && (best_ms == 0.f || ms < best_ms)) {
            best_ms = ms;
            best = p;
            best_xl = false;
        }
    }
    cudaEventDestroy (e0);
    cudaEventDestroy (e1);
    use_tc_plan (c, rc ? start : best);
    if (c->has_xl) use_xl_plan (c, rc ? xstart : xbest);
    c->use_xl = rc ? start_xl : best_xl;
    if (!roi) c->pref_xl = c->use_xl;
    if (rc) {
        cudaGetLastError ();
        return fail (c, rc, "autotuning failed");
    }
    if (tiles) *tiles = c->use_xl ? c->xplan.T : best.bx;
    return check_device_error (c);
}

extern "C" int
b200bsp_mse_kernel (const b200bsp_ctx* c, int* kernel, int* tiles,
    int* batches)
{
    if (!c) return B200BSP_E_BADARG;
    int k = 0, t = 1, b = c->geom.ntiles;
    if (c->opts.form == B200BSP_FORM_TC && c->use_xl) {
        k = B200BSP_TC_KERNEL_XLANE;
        t = c->xplan.T;
        b = c->xplan.nbatches;
    } else if (c->opts.form == B200BSP_FORM_TC) {
        k = B200BSP_TC_KERNEL_TILE;
        t = c->plan.bx;
        b = c->plan.nbatches;
    }
    if (kernel) *kernel = k;
    if (tiles) *tiles = t;
    if (batches) *batches = b;
    return B200BSP_OK;
}

// One or both MI passes on the context's form (tensor-core modes where they
// apply); gradients to grad (float) or grad64 (double), device pointers.
static int
mi_passes_on (b200bsp_ctx* c, const BspGeom& g, const float* dcoeff,
    float* grad, double* grad64, int passes)
{
    const bool roi = g.fmask || g.mroi;
    // the tile kernel's MI passes are the faster ones where both apply
    // (PVI-8, 32 bins, 256x256x128 at vpr 5: 332 + 179 us against 532 +
    // 223 us); the x-lane kernel's when pinned or the tile kernel cannot
    const bool tile_mi = c->opts.form == B200BSP_FORM_TC && !roi
        && c->opts.tc_kernel != B200BSP_TC_KERNEL_XLANE
        && tc_mi_supported (g, c->plan, c->mi.bins);
    if (c->opts.form == B200BSP_FORM_TC && !roi && c->has_xl && !tile_mi
        && xl_mi_supported (c->mi.bins)) {
        XlPlan plan = c->xplan;
        if (c->tc_grid > 0) {
            plan.grid = std::min (std::max (1, c->tc_grid / 2), plan.nbatches);
        }
        return mi_run_xl (&c->mi, g, plan, c->xlay, c->d_xtab, c->d_luts,
            c->d_part, c->d_err, c->wait_limit, dcoeff, c->d_moving,
            c->d_res, grad, grad64, c->stream, &c->last_launches, passes);
    }
    if (tile_mi) {
        TcPlan plan = c->plan;
        if (c->tc_grid > 0) plan.grid = std::min (c->tc_grid, plan.nbatches);
        return mi_run_tc (&c->mi, g, plan, c->lay, c->d_qlut,
            c->d_part, c->d_score_part, c->d_count_part, c->d_err, dcoeff,
            c->d_moving, c->d_res, grad, grad64, c->stream,
            &c->last_launches, passes);
    }
    return mi_run (&c->mi, g, dcoeff, c->d_moving, c->d_luts, c->d_res,
        grad, grad64, c->stream, &c->last_launches, passes);
}

// Whether the PVI-8 histogram pass must scan more than the ROI: the
// reference's flavours g/h scan the whole fixed image with tile index
// ijk / vox_per_rgn (bspline_mi.cxx:1562-1620), which is in range only when
// the grid starts at voxel 0 and its tiles cover the image.  Returns 1
// (whole image differs from the ROI), 0 (ROI is the image) or -1
// (unsupported).
static int
mi_whole_image_pass1 (const b200bsp_ctx* c)
{
    const BspGeom& g = c->geom;
    int differs = 0;
    for (int d = 0; d < 3; d++) {
        if (g.roi_off[d] != 0 || g.rdims[d] * g.vpr[d] < g.fdim[d]) return -1;
        if (g.roi_dim[d] != g.fdim[d]) differs = 1;
    }
    return differs;
}

static int
mi_passes (b200bsp_ctx* c, const float* dcoeff, float* grad, double* grad64,
    int passes)
{
    if (c->opts.mi_window == B200BSP_MI_PVI8 && (passes & MI_PASS_HIST)
        && mi_whole_image_pass1 (c) == 1) {
        // pass 1 over the whole image with the same tile grid, pass 2
        // over the ROI
        BspGeom g1 = c->geom;
        for (int d = 0; d < 3; d++) g1.roi_dim[d] = g1.fdim[d];
        int rc = mi_passes_on (c, g1, dcoeff, grad, grad64, MI_PASS_HIST);
        if (rc || !(passes & MI_PASS_GRAD)) return rc;
        passes = MI_PASS_GRAD;
    }
    return mi_passes_on (c, c->geom, dcoeff, grad, grad64, passes);
}

extern "C" int
b200bsp_score_mi (b200bsp_ctx* c, const float* coeff, float* score,
    float* grad, int64_t* num_vox, double* f_hist, double* m_hist,
    double* j_hist)
{
    if (!c) return B200BSP_E_BADARG;
    if (c->opts.mi_window == B200BSP_MI_PVI8 && mi_whole_image_pass1 (c) < 0) {
        // The reference's histogram pass scans the whole fixed image with
        // tile index ijk / vox_per_rgn; unless the grid starts at voxel 0
        // and covers the image it reads past its tile tables.  (The Parzen
        // variant scans the ROI in both passes.)
        return fail (c, B200BSP_E_UNSUPPORTED,
            "PVI-8 MI needs the grid to start at voxel 0 and its tiles to "
            "cover the fixed image");
    }
    const float* dcoeff = nullptr;
    int rc = begin_eval (c, coeff, &dcoeff);
    if (rc) return rc;
    float* g_dev = is_device_ptr (grad) ? grad : c->d_grad;
    rc = mi_passes (c, dcoeff, g_dev, nullptr, MI_PASS_HIST | MI_PASS_GRAD);
    if (rc) return fail (c, rc, "MI evaluation failed: %s",
        cudaGetErrorString (cudaGetLastError ()));
    mark_main_done (c);
    MiResult mr;
    rc = mi_fetch (&c->mi, c->d_res, f_hist, m_hist, j_hist, c->stream);
    if (rc) return fail (c, rc, "MI fetch failed");
    if (grad && g_dev == c->d_grad) {
        CK (cudaMemcpyAsync (grad, c->d_grad, c->num_coeff * sizeof (float),
            cudaMemcpyDeviceToHost, c->stream));
    }
    rc = end_eval (c, true);
    if (rc) return rc;
    mi_finish (&c->mi, &mr);
    if (score) *score = mr.score_f;
    if (num_vox) *num_vox = mr.num_vox;
    return check_device_error (c);
}

extern "C" int
b200bsp_mi_hist (b200bsp_ctx* c, const float* coeff, int64_t* hist)
{
    if (!c) return B200BSP_E_BADARG;
    if (!hist) return fail (c, B200BSP_E_BADARG, "null histogram buffer");
    const float* dcoeff = nullptr;
    int rc = begin_eval (c, coeff, &dcoeff);
    if (rc) return rc;
    // over the context's ROI (a slab's pass 1; see the header)
    rc = mi_passes_on (c, c->geom, dcoeff, nullptr, nullptr, MI_PASS_HIST);
    if (rc) return fail (c, rc, "MI pass 1 failed: %s",
        cudaGetErrorString (cudaGetLastError ()));
    const int B = c->mi.bins;
    const size_t nh = (size_t) 2 * B + (size_t) B * B + 1;
    CK (cudaMemcpyAsync (hist, c->mi.d_hist, nh * sizeof (int64_t),
        is_device_ptr (hist) ? cudaMemcpyDeviceToDevice
                             : cudaMemcpyDeviceToHost, c->stream));
    rc = end_eval (c, true);
    if (rc) return rc;
    return check_device_error (c);
}

extern "C" int
b200bsp_mi_grad (b200bsp_ctx* c, const float* coeff, const int64_t* hist,
    float* score, double* grad, int64_t* num_vox)
{
    if (!c) return B200BSP_E_BADARG;
    if (!hist || !grad) return fail (c, B200BSP_E_BADARG, "null argument");
    const float* dcoeff = nullptr;
    int rc = begin_eval (c, coeff, &dcoeff);
    if (rc) return rc;
    const int B = c->mi.bins;
    const size_t nh = (size_t) 2 * B + (size_t) B * B + 1;
    CK (cudaMemcpyAsync (c->mi.d_hist, hist, nh * sizeof (int64_t),
        is_device_ptr (hist) ? cudaMemcpyDeviceToDevice
                             : cudaMemcpyHostToDevice, c->stream));
    const bool dev_grad = is_device_ptr (grad);
    rc = mi_passes_on (c, c->geom, dcoeff, nullptr,
        dev_grad ? grad : c->d_grad64, MI_PASS_GRAD);
    if (rc) return fail (c, rc, "MI pass 2 failed: %s",
        cudaGetErrorString (cudaGetLastError ()));
    CK (cudaMemcpyAsync (c->h_res, c->d_res, sizeof (DevResult),
        cudaMemcpyDeviceToHost, c->stream));
    if (!dev_grad) {
        CK (cudaMemcpyAsync (grad, c->d_grad64, c->num_coeff * sizeof (double),
            cudaMemcpyDeviceToHost, c->stream));
    }
    rc = end_eval (c, true);
    if (rc) return rc;
    if (score) *score = c->h_res->score_f;
    if (num_vox) *num_vox = c->h_res->num_vox;
    return check_device_error (c);
}

static int
regularize (b200bsp_ctx* c, const float* coeff,
    const b200bsp_reg_parms* parms, double* rmetric, float* grad)
{
    if (!parms) return fail (c, B200BSP_E_BADARG, "null parms");
    const float* dcoeff = nullptr;
    if (!c) return B200BSP_E_BADARG;
    CK (cudaSetDevice (c->device));
    if (!coeff) return fail (c, B200BSP_E_BADARG, "null coefficients");
    if (is_device_ptr (coeff)) {
        dcoeff = coeff;
    } else {
        CK (cudaMemcpyAsync (c->d_coeff, coeff, c->num_coeff * sizeof (float),
            cudaMemcpyHostToDevice, c->stream));
        dcoeff = c->d_coeff;
    }
    bool dev_grad = is_device_ptr (grad);
    if (grad && !dev_grad) {
        CK (cudaMemcpyAsync (c->d_grad, grad, c->num_coeff * sizeof (float),
            cudaMemcpyHostToDevice, c->stream));
    }
    float* g_dev = grad ? (dev_grad ? grad : c->d_grad) : nullptr;
    int rc = reg_run (&c->reg, c->geom, parms, dcoeff, g_dev, c->stream);
    if (rc) return fail (c, rc, "regulariser failed: %s",
        cudaGetErrorString (cudaGetLastError ()));
    if (grad && !dev_grad) {
        CK (cudaMemcpyAsync (grad, c->d_grad, c->num_coeff * sizeof (float),
            cudaMemcpyDeviceToHost, c->stream));
    }
    double S = 0;
    rc = reg_fetch (&c->reg, &S, c->stream);
    if (rc) return fail (c, rc, "regulariser fetch failed");
    if (rmetric) *rmetric = S;
    return B200BSP_OK;
}

extern "C" int
b200bsp_regularize (b200bsp_ctx* c, const float* coeff,
    const b200bsp_reg_parms* parms, float* rmetric, float* grad)
{
    double S = 0.0;
    const int rc = regularize (c, coeff, parms, &S, grad);
    if (!rc && rmetric) *rmetric = (float) S;
    return rc;
}

extern "C" int
b200bsp_regularize_f64 (b200bsp_ctx* c, const float* coeff,
    const b200bsp_reg_parms* parms, double* rmetric, float* grad)
{
    return regularize (c, coeff, parms, rmetric, grad);
}

// One axis of a q_lut row as Bspline_xform::allocate builds it
// (src/base/bspline_xform.cxx:378-430): float offset, double polynomial,
// rounded to float.
static void
qlut_axis (float out[4], int64_t i, int64_t vpr)
{
    const float ii = ((float) i) / vpr;
    const float t3 = ii * ii * ii, t2 = ii * ii, t1 = ii;
    out[0] = (float) ((1.0/6.0) * (- 1.0 * t3 + 3.0 * t2 - 3.0 * t1 + 1.0));
    out[1] = (float) ((1.0/6.0) * (+ 3.0 * t3 - 6.0 * t2 + 4.0));
    out[2] = (float) ((1.0/6.0) * (- 3.0 * t3 + 3.0 * t2 + 3.0 * t1 + 1.0));
    out[3] = (float) ((1.0/6.0) * (+ 1.0 * t3));
}

static void
free_landmarks (b200bsp_ctx* c)
{
    cudaFree (c->d_lm_p); cudaFree (c->d_lm_w); cudaFree (c->d_lm_fm);
    cudaFree (c->d_lm_dc);
    c->d_lm_p = nullptr; c->d_lm_w = nullptr; c->d_lm_fm = nullptr;
    c->d_lm_dc = nullptr;
    c->lm_n = 0;
}

static bool
roi_geom (const b200bsp_volume* v, RoiGeom* o)
{
    float inv[9];
    if (!inv3f (inv, v->dcos)) return false;
    for (int d = 0; d < 3; d++) {
        if (v->dim[d] < 1 || v->dim[d] > (1 << 30) || !(v->spacing[d] != 0.f)
            || !std::isfinite (v->spacing[d])) {
            return false;
        }
        o->dim[d] = (int) v->dim[d];
        o->origin[d] = v->origin[d];
    }
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) {
            o->step[3*i+j] = v->dcos[3*i+j] * v->spacing[j];
            o->proj[3*i+j] = inv[3*i+j] / v->spacing[i];
        }
    }
    return (long long) o->dim[0] * o->dim[1] * o->dim[2] < (1LL << 31);
}

extern "C" int
b200bsp_set_roi (b200bsp_ctx* c, const b200bsp_volume* fixed_roi,
    const uint8_t* fixed_mask, const b200bsp_volume* moving_roi,
    const uint8_t* moving_mask)
{
    if (!c) return B200BSP_E_BADARG;
    c->gen++;
    if (!fixed_roi != !fixed_mask || !moving_roi != !moving_mask) {
        return fail (c, B200BSP_E_BADARG,
            "an ROI needs both its geometry and its mask");
    }
    RoiGeom fr, mr;
    if ((fixed_roi && !roi_geom (fixed_roi, &fr))
        || (moving_roi && !roi_geom (moving_roi, &mr))) {
        return fail (c, B200BSP_E_BADARG,
            "ROI geometry: need dims >= 1 (< 2^31 voxels), finite nonzero "
            "spacing and invertible direction cosines");
    }
    const bool any = fixed_roi || moving_roi;
    if (any && c->opts.form == B200BSP_FORM_TC && !c->has_xl) {
        return fail (c, B200BSP_E_UNSUPPORTED,
            "image ROIs in the tensor-core form need its x-lane kernel "
            "(3 <= vox_per_rgn[1] <= 10, tc_kernel not TILE); use "
            "B200BSP_FORM_FP32");
    }
    CK (cudaSetDevice (c->device));
    CK (cudaStreamSynchronize (c->stream));
    cudaFree (c->d_fmask);
    cudaFree (c->d_mroi);
    c->d_fmask = nullptr;
    c->d_mroi = nullptr;
    BspGeom& g = c->geom;
    g.fmask = nullptr;
    g.mroi = nullptr;
    if (fixed_roi) {
        const size_t nr = (size_t) fr.dim[0] * fr.dim[1] * fr.dim[2];
        const size_t nf = (size_t) g.fdim[0] * g.fdim[1] * g.fdim[2];
        uint8_t* d_roi = nullptr;
        const bool dev = is_device_ptr (fixed_mask);
        if (!dev) CK (cudaMalloc ((void**) &d_roi, nr));
        CK (cudaMalloc ((void**) &c->d_fmask, nf));
        cudaError_t e = cudaSuccess;
        if (!dev) {
            e = cudaMemcpyAsync (d_roi, fixed_mask, nr, cudaMemcpyHostToDevice,
                c->stream);
        }
        RoiGeom fg;
        for (int d = 0; d < 3; d++) {
            fg.dim[d] = g.fdim[d];
            fg.origin[d] = g.img_origin[d];
        }
        for (int i = 0; i < 9; i++) fg.step[i] = g.fstep[i];
        if (e == cudaSuccess) {
            e = launch_fixed_roi_mask (g.fdim, fg, fr, dev ? fixed_mask : d_roi,
                c->d_fmask, c->stream);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize (c->stream);
        cudaFree (d_roi);
        if (e != cudaSuccess) {
            return fail (c, B200BSP_E_CUDA, "fixed ROI: %s",
                cudaGetErrorString (e));
        }
        g.fmask = c->d_fmask;
    }
    if (moving_roi) {
        const size_t nr = (size_t) mr.dim[0] * mr.dim[1] * mr.dim[2];
        CK (cudaMalloc ((void**) &c->d_mroi, nr));
        CK (cudaMemcpy (c->d_mroi, moving_mask, nr, cudaMemcpyDefault));
        for (int d = 0; d < 3; d++) {
            g.mroi_dim[d] = mr.dim[d];
            g.mroi_origin[d] = mr.origin[d];
        }
        for (int i = 0; i < 9; i++) g.mroi_proj[i] = mr.proj[i];
        g.mroi = c->d_mroi;
    }
    // the tile kernel has no ROI tests: MSE moves to the x-lane kernel while
    // ROIs are set, and back to the choice without them after
    if (c->opts.form == B200BSP_FORM_TC) c->use_xl = any || c->pref_xl;
    return B200BSP_OK;
}

extern "C" int
b200bsp_set_landmarks (b200bsp_ctx* c, const float* fixed_xyz,
    int64_t n_fixed, const float* moving_xyz, int64_t n_moving,
    float stiffness)
{
    if (!c) return B200BSP_E_BADARG;
    CK (cudaSetDevice (c->device));
    // Bspline_landmarks::set_landmarks: the shorter list sets the count
    const int64_t n = n_fixed < n_moving ? n_fixed : n_moving;
    if (n <= 0) {
        CK (cudaStreamSynchronize (c->stream));
        free_landmarks (c);
        return B200BSP_OK;
    }
    if (!fixed_xyz || !moving_xyz) {
        return fail (c, B200BSP_E_BADARG, "null landmark list");
    }
    if (n > (1 << 24)) {
        return fail (c, B200BSP_E_BADARG, "at most 2^24 landmarks");
    }
    // Bspline_landmarks::initialize (src/register/bspline_landmarks.cxx:
    // 150-204): grid coordinates of each fixed landmark, in float, through
    // the fixed image's projection matrix; the voxel index truncates
    // toward zero and must lie inside the image.
    float inv[9], proj[9];
    if (!inv3f (inv, c->fixed.dcos)) {
        return fail (c, B200BSP_E_BADARG, "singular direction cosines");
    }
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) {
            proj[3*i+j] = inv[3*i+j] / c->fixed.spacing[i];
        }
    }
    const BspGeom& g = c->geom;
    std::vector<int> hp ((size_t) 3 * n);
    std::vector<float> hw ((size_t) 64 * n), hfm ((size_t) 6 * n);
    for (int64_t l = 0; l < n; l++) {
        float xyz[3];
        for (int d = 0; d < 3; d++) {
            xyz[d] = fixed_xyz[3*l+d] - c->fixed.origin[d];
        }
        int64_t q[3];
        for (int d = 0; d < 3; d++) {
            const float ijk = xyz[0] * proj[3*d+0] + xyz[1] * proj[3*d+1]
                + xyz[2] * proj[3*d+2];
            // (the range test first: the cast is defined only in range)
            const bool in = ijk > -1.f && ijk < (float) c->fixed.dim[d];
            const int64_t v = in ? (int64_t) ijk : -1;
            if (v < 0 || v >= c->fixed.dim[d]) {
                free_landmarks (c);
                return fail (c, B200BSP_E_BADARG,
                    "fixed landmark %lld outside of the fixed image",
                    (long long) l);
            }
            hp[3*l+d] = (int) (v / g.vpr[d]);
            q[d] = v % g.vpr[d];
            // The reference takes the tile from the absolute voxel index;
            // it must be one of the grid's tiles.
            if (hp[3*l+d] >= g.rdims[d]) {
                free_landmarks (c);
                return fail (c, B200BSP_E_UNSUPPORTED,
                    "fixed landmark %lld lies beyond the grid's tiles",
                    (long long) l);
            }
        }
        float A[4], B[4], C[4];
        qlut_axis (A, q[0], g.vpr[0]);
        qlut_axis (B, q[1], g.vpr[1]);
        qlut_axis (C, q[2], g.vpr[2]);
        for (int tz = 0; tz < 4; tz++)
            for (int ty = 0; ty < 4; ty++)
                for (int tx = 0; tx < 4; tx++)
                    hw[64*l + 16*tz + 4*ty + tx] = A[tx] * B[ty] * C[tz];
        for (int d = 0; d < 3; d++) {
            hfm[6*l+d] = fixed_xyz[3*l+d];
            hfm[6*l+3+d] = moving_xyz[3*l+d];
        }
    }
    CK (cudaStreamSynchronize (c->stream));
    free_landmarks (c);
    CK (cudaMalloc ((void**) &c->d_lm_p, hp.size () * sizeof (int)));
    CK (cudaMalloc ((void**) &c->d_lm_w, hw.size () * sizeof (float)));
    CK (cudaMalloc ((void**) &c->d_lm_fm, hfm.size () * sizeof (float)));
    CK (cudaMalloc ((void**) &c->d_lm_dc, (4 * n + 1) * sizeof (float)));
    CK (cudaMemcpy (c->d_lm_p, hp.data (), hp.size () * sizeof (int),
        cudaMemcpyHostToDevice));
    CK (cudaMemcpy (c->d_lm_w, hw.data (), hw.size () * sizeof (float),
        cudaMemcpyHostToDevice));
    CK (cudaMemcpy (c->d_lm_fm, hfm.data (), hfm.size () * sizeof (float),
        cudaMemcpyHostToDevice));
    c->lm_n = (int) n;
    c->lm_stiffness = stiffness;
    return B200BSP_OK;
}

extern "C" int
b200bsp_landmarks_score (b200bsp_ctx* c, const float* coeff, float* lmetric,
    float* grad)
{
    if (!c) return B200BSP_E_BADARG;
    if (c->lm_n < 1) return fail (c, B200BSP_E_STATE, "no landmarks set");
    if (!coeff) return fail (c, B200BSP_E_BADARG, "null coefficients");
    CK (cudaSetDevice (c->device));
    const float* dcoeff = coeff;
    if (!is_device_ptr (coeff)) {
        CK (cudaMemcpyAsync (c->d_coeff, coeff, c->num_coeff * sizeof (float),
            cudaMemcpyHostToDevice, c->stream));
        dcoeff = c->d_coeff;
    }
    const bool dev_grad = is_device_ptr (grad);
    float* g_dev = dev_grad ? grad : c->d_grad;
    if (grad && !dev_grad) {
        CK (cudaMemcpyAsync (c->d_grad, grad, c->num_coeff * sizeof (float),
            cudaMemcpyHostToDevice, c->stream));
    } else if (!grad) {
        CK (cudaMemsetAsync (c->d_grad, 0, c->num_coeff * sizeof (float),
            c->stream));
    }
    // land_grad_coeff = landmark_stiffness / num_landmarks, in float
    const float grad_coeff = c->lm_stiffness / (float) c->lm_n;
    float* d_lmetric = c->d_lm_dc + 4 * (size_t) c->lm_n;
    CK (launch_landmarks (c->geom, c->lm_n, c->d_lm_p, c->d_lm_w,
        c->d_lm_fm, dcoeff, grad_coeff, c->d_lm_dc, g_dev, d_lmetric,
        c->stream));
    if (grad && !dev_grad) {
        CK (cudaMemcpyAsync (grad, c->d_grad, c->num_coeff * sizeof (float),
            cudaMemcpyDeviceToHost, c->stream));
    }
    float lm = 0.f;
    CK (cudaMemcpyAsync (c->h_scalar, d_lmetric, sizeof (float),
        cudaMemcpyDeviceToHost, c->stream));
    CK (cudaStreamSynchronize (c->stream));
    lm = *c->h_scalar;
    if (lmetric) *lmetric = lm;
    return B200BSP_OK;
}

// bspline_score with MSE and device outputs, stream-ordered: the MSE
// kernel, the regulariser's passes beside it on the context's second
// stream, then the finish kernel that combines them (lambda times the
// metric, plus the regulariser's score and double gradient).  The MSE
// kernel holds every register of the SMs it runs on, so it is launched on
// all but REG_SIDE_SMS of them and the passes (a few microseconds of work
// each, but three dependent launches) run on the rest meanwhile.
static int
score_mse_device (b200bsp_ctx* c, const float* coeff, float lambda,
    const b200bsp_reg_parms* reg, float* total_score, float* total_grad,
    float* smetric, int64_t* num_vox)
{
    const float* dcoeff = nullptr;
    int rc = begin_eval (c, coeff, &dcoeff);
    if (rc) return rc;
    FinishCombine cb;
    cb.lambda = lambda;
    cb.total_score = total_score ? total_score : c->d_total;
    const int grid0 = c->tc_grid;
    if (reg) {
        CK (cudaEventRecord (c->ev_fork, c->stream));
        CK (cudaStreamWaitEvent (c->aux_stream, c->ev_fork, 0));
        cb.reg_grad = c->d_reg_grad64;
        cb.reg_score = c->reg.d_score;
        if (c->opts.form == B200BSP_FORM_TC && grid0 == 0
            && c->sm_count > 2 * REG_SIDE_SMS) {
            c->tc_grid = 2 * (c->sm_count - REG_SIDE_SMS);
        }
    }
    rc = run_mse (c, dcoeff, total_grad, nullptr, smetric, nullptr,
        (long long*) num_vox, nullptr, cb, reg ? c->ev_join : nullptr,
        [&] () {
            // between the MSE kernel's launch and the finish kernel's
            if (!reg) return B200BSP_OK;
            int r = reg_run (&c->reg, c->geom, reg, dcoeff, nullptr,
                c->aux_stream, c->d_reg_grad64);
            if (r) return fail (c, r, "regulariser failed: %s",
                cudaGetErrorString (cudaGetLastError ()));
            CK (cudaEventRecord (c->ev_join, c->aux_stream));
            c->last_launches += c->reg.plan.n1 ? 3 : 1;
            return B200BSP_OK;
        });
    c->tc_grid = grid0;
    if (rc) return rc;
    return end_eval (c, false);
}

// MI's combine on the device, as the finish kernel's for MSE: total_grad =
// 0 + lambda * metric gradient in float, then the regulariser's double
// gradient added with one rounding; total = lambda * score (+ the
// regulariser's score in float), in Bspline_score's order.
__global__ void
mi_combine_kernel (const DevResult* __restrict__ res, float lambda,
    const double* __restrict__ reg_grad, const double* __restrict__ reg_score,
    float* __restrict__ grad, long long n, float* __restrict__ total,
    float* __restrict__ smetric, long long* __restrict__ nvox)
{
    for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x;
         i < n; i += (long long) gridDim.x * blockDim.x) {
        const float t = 0.f + lambda * grad[i];
        grad[i] = reg_grad ? (float) ((double) t + reg_grad[i]) : t;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        float tot = 0.f;
        tot += lambda * res->score_f;
        if (reg_score) tot += (float) *reg_score;
        *total = tot;
        if (smetric) *smetric = res->score_f;
        if (nvox) *nvox = res->num_vox;
    }
}

// bspline_score with MI and device outputs, stream-ordered: both MI
// passes, the regulariser, then mi_combine_kernel (no host round trip, so
// the optimiser can record it in a graph).
static int
score_mi_device (b200bsp_ctx* c, const float* coeff, float lambda,
    const b200bsp_reg_parms* reg, float* total_score, float* total_grad,
    float* smetric, int64_t* num_vox)
{
    if (c->opts.mi_window == B200BSP_MI_PVI8 && mi_whole_image_pass1 (c) < 0) {
        return fail (c, B200BSP_E_UNSUPPORTED,
            "PVI-8 MI needs the grid to start at voxel 0 and its tiles to "
            "cover the fixed image");
    }
    const float* dcoeff = nullptr;
    int rc = begin_eval (c, coeff, &dcoeff);
    if (rc) return rc;
    rc = mi_passes (c, dcoeff, total_grad, nullptr,
        MI_PASS_HIST | MI_PASS_GRAD);
    if (rc) return fail (c, rc, "MI evaluation failed: %s",
        cudaGetErrorString (cudaGetLastError ()));
    mark_main_done (c);
    if (reg) {
        rc = reg_run (&c->reg, c->geom, reg, dcoeff, nullptr, c->stream,
            c->d_reg_grad64);
        if (rc) return fail (c, rc, "regulariser failed: %s",
            cudaGetErrorString (cudaGetLastError ()));
    }
    const long long n = c->num_coeff;
    const unsigned blocks = (unsigned) std::max<long long> (1,
        std::min<long long> ((n + 255) / 256, 4LL * c->sm_count));
    mi_combine_kernel<<<blocks, 256, 0, c->stream>>> (c->d_res, lambda,
        reg ? c->d_reg_grad64 : nullptr, reg ? c->reg.d_score : nullptr,
        total_grad, n, total_score ? total_score : c->d_total, smetric,
        (long long*) num_vox);
    CK (cudaGetLastError ());
    c->last_launches++;
    return end_eval (c, false);
}

extern "C" int
b200bsp_score (b200bsp_ctx* c, const float* coeff, int metric_type,
    float lambda, const b200bsp_reg_parms* reg, float* total_score,
    float* total_grad, float* smetric, int64_t* num_vox)
{
    if (!c || !total_grad) return fail (c, B200BSP_E_BADARG, "null argument");
    if ((metric_type == 0 || metric_type == 1) && c->lm_n == 0
        && is_device_ptr (total_grad)
        && (!total_score || is_device_ptr (total_score))
        && (!smetric || is_device_ptr (smetric))
        && (!num_vox || is_device_ptr (num_vox))) {
        return metric_type == 0
            ? score_mse_device (c, coeff, lambda, reg, total_score,
                total_grad, smetric, num_vox)
            : score_mi_device (c, coeff, lambda, reg, total_score,
                total_grad, smetric, num_vox);
    }
    std::vector<float> g ((size_t) c->num_coeff);
    float s = 0.f;
    int64_t nv = 0;
    int rc = metric_type == 0
        ? b200bsp_score_mse (c, coeff, &s, g.data (), &nv)
        : b200bsp_score_mi (c, coeff, &s, g.data (), &nv, nullptr, nullptr,
            nullptr);
    if (rc) return rc;
    // Bspline_score::accumulate (src/register/bspline_score.cxx:63-74)
    float total = 0.f;
    total += lambda * s;
    for (int64_t i = 0; i < c->num_coeff; i++) g[i] = 0.f + lambda * g[i];
    if (reg) {
        float r = 0.f;
        rc = b200bsp_regularize (c, coeff, reg, &r, g.data ());
        if (rc) return rc;
        total += r;
    }
    if (c->lm_n > 0) {
        // landmark score and gradient (src/register/bspline.cxx:624-628)
        float lm = 0.f;
        rc = b200bsp_landmarks_score (c, coeff, &lm, g.data ());
        if (rc) return rc;
        total += c->lm_stiffness * lm;
    }
    if (is_device_ptr (total_grad)) {
        CK (cudaMemcpy (total_grad, g.data (), c->num_coeff * sizeof (float),
            cudaMemcpyHostToDevice));
    } else {
        memcpy (total_grad, g.data (), c->num_coeff * sizeof (float));
    }
    if (total_score) *total_score = total;
    if (smetric) *smetric = s;
    if (num_vox) *num_vox = nv;
    return B200BSP_OK;
}

// Field and warp share one path: coefficients to the device, outputs
// either written in place (device pointers) or through the staging buffer.
static int
field_warp (b200bsp_ctx* c, const float* coeff, float* vf, float* warped,
    float default_value)
{
    const float* dcoeff = nullptr;
    int rc = begin_eval (c, coeff, &dcoeff);
    if (rc) return rc;
    const BspGeom& g = c->geom;
    const size_t nf = (size_t) g.fdim[0] * g.fdim[1] * g.fdim[2];
    float* out = vf ? vf : warped;
    const size_t bytes = (vf ? 3 : 1) * nf * sizeof (float);
    const bool dev_out = is_device_ptr (out);
    float* target = out;
    if (!dev_out) {
        if (!c->d_out) {
            cudaError_t e = cudaMalloc ((void**) &c->d_out,
                3 * nf * sizeof (float));
            if (e != cudaSuccess) {
                cudaGetLastError ();
                c->d_out = nullptr;
                return fail (c, B200BSP_E_OOM, "staging buffer: %s",
                    cudaGetErrorString (e));
            }
        }
        target = c->d_out;
    }
    bool whole = true;
    for (int d = 0; d < 3; d++) {
        whole = whole && g.roi_off[d] == 0 && g.roi_dim[d] == g.fdim[d];
    }
    if (vf && !whole) CK (cudaMemsetAsync (target, 0, bytes, c->stream));
    CK (launch_field_warp (g, dcoeff, c->d_luts, c->d_moving, default_value,
        vf ? target : nullptr, vf ? nullptr : target, c->stream));
    c->last_launches = 1;
    rc = mark_main_done (c);
    if (rc) return rc;
    if (!dev_out) {
        CK (cudaMemcpyAsync (out, target, bytes, cudaMemcpyDeviceToHost,
            c->stream));
    }
    return end_eval (c, !dev_out);
}

extern "C" int
b200bsp_interpolate_vf (b200bsp_ctx* c, const float* coeff, float* vf)
{
    if (!c) return B200BSP_E_BADARG;
    if (!vf) return fail (c, B200BSP_E_BADARG, "null output");
    return field_warp (c, coeff, vf, nullptr, 0.f);
}

extern "C" int
b200bsp_warp (b200bsp_ctx* c, const float* coeff, float default_value,
    float* warped)
{
    if (!c) return B200BSP_E_BADARG;
    if (!warped) return fail (c, B200BSP_E_BADARG, "null output");
    for (int d = 0; d < 3; d++) {
        if (c->geom.roi_off[d] != 0 || c->geom.roi_dim[d] != c->geom.fdim[d]) {
            return fail (c, B200BSP_E_UNSUPPORTED,
                "warp needs the grid's ROI to be the whole fixed image");
        }
    }
    return field_warp (c, coeff, nullptr, warped, default_value);
}

extern "C" int
b200bsp_volume_grad (const b200bsp_volume* vol, const float* img,
    float* grad_out, int device)
{
    b200bsp_ctx* c = nullptr;
    if (!vol || !img || !grad_out) return fail (c, B200BSP_E_BADARG, "null argument");
    int rc = check_volume (vol, "volume");
    if (rc) return rc;
    float inv[9];
    if (!inv3f (inv, vol->dcos)) {
        return fail (c, B200BSP_E_BADARG, "singular direction cosines");
    }
    CK (cudaSetDevice (device));
    int dim[3] = {(int) vol->dim[0], (int) vol->dim[1], (int) vol->dim[2]};
    size_t n = (size_t) dim[0] * dim[1] * dim[2];
    float *d_img = nullptr, *d_grad = nullptr, *d_inv = nullptr;
    bool in_dev = is_device_ptr (img), out_dev = is_device_ptr (grad_out);
    if (!in_dev) CK (cudaMalloc (&d_img, n * sizeof (float)));
    if (!out_dev) CK (cudaMalloc (&d_grad, 3 * n * sizeof (float)));
    CK (cudaMalloc (&d_inv, 9 * sizeof (float)));
    if (!in_dev) CK (cudaMemcpy (d_img, img, n * sizeof (float), cudaMemcpyHostToDevice));
    CK (cudaMemcpy (d_inv, inv, 9 * sizeof (float), cudaMemcpyHostToDevice));
    float sp[3] = {vol->spacing[0], vol->spacing[1], vol->spacing[2]};
    CK (launch_volume_grad (dim, sp, d_inv, in_dev ? img : d_img,
        out_dev ? grad_out : d_grad, 0));
    CK (cudaDeviceSynchronize ());
    if (!out_dev) CK (cudaMemcpy (grad_out, d_grad, 3 * n * sizeof (float),
        cudaMemcpyDeviceToHost));
    cudaFree (d_img); cudaFree (d_grad); cudaFree (d_inv);
    return B200BSP_OK;
}

extern "C" int
b200bsp_enable_timing (b200bsp_ctx* c, int on)
{
    if (!c) return B200BSP_E_BADARG;
    c->timing = on != 0;
    return B200BSP_OK;
}

extern "C" int
b200bsp_last_timing (const b200bsp_ctx* c, float* ms, int* launches)
{
    if (!c) return B200BSP_E_BADARG;
    if (ms) *ms = c->last_total_ms;
    if (launches) *launches = c->last_launches;
    return B200BSP_OK;
}

extern "C" int
b200bsp_last_main_ms (const b200bsp_ctx* c, float* ms)
{
    if (!c) return B200BSP_E_BADARG;
    if (ms) *ms = c->last_main_ms;
    return B200BSP_OK;
}

extern "C" const char*
b200bsp_last_error (const b200bsp_ctx* c)
{
    return c ? c->err.c_str () : g_create_error.c_str ();
}
