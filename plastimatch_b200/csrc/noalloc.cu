// Context-free MSE score + gradient whose scratch is one fixed-size static
// device array instead of memory obtained at run time.
//
// Who needs it: a host that cannot let a library allocate device memory
// while it runs -- an optimiser loop inside a framework whose caching
// allocator owns the device's memory (a cudaMalloc from outside it can fail
// or fragment its pool, and cudaMalloc/cudaFree synchronise the device), or
// a service that reserves all its memory at start-up and admits no
// allocation afterwards.  Such a caller passes device buffers it already
// owns; this entry point adds nothing to them but the static array below.
//
// The work is that of b200bsp_score_mse with the FP32 form: the tile
// kernel, the fixed-order score reduction and the per-knot gradient gather,
// with their partial sums placed in the static array.  Every partial the
// kernels read is written earlier in the same call (each tile writes all
// 64 slots of its partial gradient, its score and its count; the reduction
// writes the result block; a small kernel writes the basis tables), so
// nothing needs clearing between calls.
//
// One array serves every call on a device: two calls whose device work
// overlaps (different streams, or different host threads) race on it.
// Callers serialise them, e.g. by issuing all calls on one stream.
#include <cstdio>

#include "../../include/plastimatch_b200.h"
#include "kernels.cuh"

namespace b200 {

// Validation and geometry of b200bsp_create, without a context (runtime.cu).
int static_geometry (const b200bsp_volume* fixed, const b200bsp_volume* moving,
    const b200bsp_grid* grid, BspGeom* g, float* luts, int* nlut);
int static_fail (int code, const char* msg);

constexpr int SMAX = B200BSP_STATIC_MAX_TILES;
constexpr size_t align256 (size_t n) { return (n + 255) & ~(size_t) 255; }
constexpr size_t OFF_RES = 0;
constexpr size_t OFF_LUT = align256 (OFF_RES + sizeof (DevResult));
constexpr size_t OFF_SCORE = align256 (OFF_LUT + sizeof (float) * 4 * 3 * 64);
constexpr size_t OFF_COUNT = align256 (OFF_SCORE + sizeof (double) * SMAX);
constexpr size_t OFF_PART = align256 (OFF_COUNT + sizeof (int) * SMAX);
constexpr size_t SCRATCH_BYTES = align256 (OFF_PART
    + sizeof (float) * 64 * 3 * (size_t) SMAX);

static __device__ __align__ (256) unsigned char g_scratch[SCRATCH_BYTES];

struct LutArg {
    float v[4 * 3 * 64];
};

__global__ void
fill_luts_kernel (LutArg a, int n, float* __restrict__ dst)
{
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = a.v[i];
}

// Device address of the static array in the current device's context.
// Looked up on every call (a cheap query) rather than cached: after a
// cudaDeviceReset, or under another driver context on the same ordinal,
// the module is loaded afresh and the array has a new address.
static unsigned char*
scratch_base ()
{
    void* p = nullptr;
    if (cudaGetSymbolAddress (&p, g_scratch) != cudaSuccess) {
        cudaGetLastError ();             // this call's own lookup error
        return nullptr;
    }
    return (unsigned char*) p;
}

static bool
on_device (const void* p, int dev)
{
    cudaPointerAttributes a;
    if (!p || cudaPointerGetAttributes (&a, p) != cudaSuccess) {
        cudaGetLastError ();
        return false;
    }
    return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged)
        && a.device == dev;
}

} // namespace b200

using namespace b200;

extern "C" int
b200bsp_score_mse_static (const b200bsp_volume* fixed,
    const b200bsp_volume* moving, const b200bsp_grid* grid, int mse_grad,
    const float* fixed_img, const float* moving_img, const float* moving_grad,
    const float* coeff, float* score, float* grad, int64_t* num_vox,
    void* stream)
{
    if (!fixed || !moving || !grid) {
        return static_fail (B200BSP_E_BADARG, "null argument");
    }
    if (mse_grad != B200BSP_MSE_GRAD_NEAREST
        && mse_grad != B200BSP_MSE_GRAD_TRILINEAR) {
        return static_fail (B200BSP_E_BADARG, "unknown mse_grad");
    }
    BspGeom g = {};
    float luts[4 * 3 * 64];
    int nlut = 0;
    int rc = static_geometry (fixed, moving, grid, &g, luts, &nlut);
    if (rc) return rc;
    if (g.ntiles > SMAX) {
        char msg[160];
        snprintf (msg, sizeof msg, "static scratch holds %d tiles; this grid "
            "has %d (use a context instead)", SMAX, g.ntiles);
        return static_fail (B200BSP_E_UNSUPPORTED, msg);
    }
    if (mse_fp32_smem_bytes (g) > 200 * 1024) {
        return static_fail (B200BSP_E_UNSUPPORTED, "tile too large");
    }
    // an error the caller's own earlier work left pending is reported, not
    // cleared (and not blamed on this call's launches below)
    const cudaError_t pending = cudaPeekAtLastError ();
    if (pending != cudaSuccess) {
        char msg[200];
        snprintf (msg, sizeof msg, "a CUDA error is already pending: %s",
            cudaGetErrorString (pending));
        return static_fail (B200BSP_E_CUDA, msg);
    }
    int dev = 0;
    if (cudaGetDevice (&dev) != cudaSuccess) {
        cudaGetLastError ();
        return static_fail (B200BSP_E_CUDA, "no current CUDA device");
    }
    const bool need_mgrad = mse_grad == B200BSP_MSE_GRAD_NEAREST;
    if (!on_device (fixed_img, dev) || !on_device (moving_img, dev)
        || !on_device (coeff, dev) || !on_device (grad, dev)
        || (need_mgrad && !on_device (moving_grad, dev))
        || (score && !on_device (score, dev))
        || (num_vox && !on_device (num_vox, dev))) {
        return static_fail (B200BSP_E_BADARG, "images, coefficients, "
            "moving gradient (nearest mode) and outputs must be device "
            "memory on the current device");
    }
    unsigned char* base = scratch_base ();
    if (!base) return static_fail (B200BSP_E_CUDA, "static scratch lookup failed");
    DevResult* res = (DevResult*) (base + OFF_RES);
    float* d_luts = (float*) (base + OFF_LUT);
    double* score_part = (double*) (base + OFF_SCORE);
    int* count_part = (int*) (base + OFF_COUNT);
    float* part = (float*) (base + OFF_PART);
    cudaStream_t st = (cudaStream_t) stream;

    LutArg la;
    for (int i = 0; i < nlut; i++) la.v[i] = luts[i];
    fill_luts_kernel<<<1, 256, 0, st>>> (la, nlut, d_luts);
    PartLayout lay;
    lay.bx = lay.by = lay.bz = 1;
    lay.nbx = g.rdims[0]; lay.nby = g.rdims[1]; lay.nbz = g.rdims[2];
    lay.kx = lay.ky = lay.kz = 4;
    lay.slots = 64;
    if (cudaGetLastError () != cudaSuccess
        || launch_mse_fp32 (g, mse_grad, fixed_img, moving_img,
               need_mgrad ? moving_grad : nullptr, coeff, d_luts, part,
               score_part, count_part, st) != cudaSuccess
        || launch_reduce_score (score_part, count_part, g.ntiles, res, 0, st)
               != cudaSuccess
        || launch_gather_grad (g, lay, part, res, 0, grad, nullptr, score,
               nullptr, (long long*) num_vox, st) != cudaSuccess) {
        return static_fail (B200BSP_E_CUDA, "kernel launch failed");
    }
    return B200BSP_OK;
}
