// Pyramid resampling of a float image (the per-stage preprocessing of
// B-spline registration, Plastimatch src/register/bspline_stage.cxx:
// 193-205 via registration_resample_volume, src/register/
// registration_resample.cxx:12-59):
//   b200bsp_resample_geometry  the output grid of a resample type
//       (volume_subsample_vox, _legacy, volume_resample_spacing, _percent,
//       src/base/volume_resample.cxx:297-413)
//   b200bsp_resample           volume_resample_float_li (:70-136) onto any
//       output grid
// The reference's resampler is separable: output positions advance along
// each axis by the output spacing (direction cosines are not used), and the
// input index, its rounding, clamp and interpolation fractions depend on
// one axis each.  The host computes them per axis in the reference's float
// arithmetic; the kernel combines three table entries and forms the
// trilinear value with the reference's weight products and sum order, so
// the device result equals the reference's bit for bit.
#include <cmath>
#include <cstdio>
#include <vector>

#include "../../include/plastimatch_b200.h"
#include "kernels.cuh"

namespace b200 {

int static_fail (int code, const char* msg);   // runtime.cu

// Per output index along one axis: the input floor index (-1 when the
// rounded index lies outside the input) and the two fractions.
struct AxisTap {
    int f;
    float w1, w2;
};

static long long
round_long (double x)         // ROUND_PLM_LONG, src/sys/plm_math.h:53-54
{
    return (x >= 0) ? (long long) (x + 0.5) : (long long) (-(-x + 0.5));
}

// One axis of volume_resample_float_li: pos_n = origin + spacing added n
// times; ijk = (pos - in_origin) / in_spacing; out of range when the
// rounded ijk is; else li_clamp (src/base/interpolate.cxx:17-41).
static void
axis_taps (AxisTap* t, long long n, float oorigin, float ospacing,
    float iorigin, float ispacing, long long idim)
{
    float pos = oorigin;
    for (long long i = 0; i < n; i++, pos += ospacing) {
        volatile float ijk = (pos - iorigin) / ispacing;
        const long long r = round_long ((double) ijk);
        if (r < 0 || r >= idim) {
            t[i].f = -1;
            t[i].w1 = 1.f;
            t[i].w2 = 0.f;
            continue;
        }
        const long long dmax = idim - 1;
        long long f;
        float w2;
        if (ijk < 0.f) {
            f = 0; w2 = 0.f;
        } else if (ijk >= dmax) {
            f = dmax - 1; w2 = 1.f;
        } else {
            f = (long long) std::floor (ijk);
            w2 = ijk - (float) f;
        }
        t[i].f = (int) f;
        t[i].w2 = w2;
        t[i].w1 = 1.0f - w2;
    }
}

__global__ void
resample_li_kernel (int ox, int oy, int oz, int ix, int iy,
    const AxisTap* __restrict__ tx, const AxisTap* __restrict__ ty,
    const AxisTap* __restrict__ tz, const float* __restrict__ in,
    float* __restrict__ out)
{
    const long long n = (long long) ox * oy * oz;
    for (long long v = (long long) blockIdx.x * blockDim.x + threadIdx.x;
         v < n; v += (long long) gridDim.x * blockDim.x) {
        const int i = (int) (v % ox);
        const int j = (int) ((v / ox) % oy);
        const int k = (int) (v / ((long long) ox * oy));
        const AxisTap a = tx[i], b = ty[j], c = tz[k];
        if (a.f < 0 || b.f < 0 || c.f < 0) {
            out[v] = 0.f;
            continue;
        }
        const long long dx = ix, dxy = (long long) ix * iy;
        const float* p = in + a.f + dx * (b.f + (long long) iy * c.f);
        // LI_VALUE (src/base/interpolate_macros.h:23-38): ((wx wy) wz) m,
        // summed corner by corner
        float s = __fmul_rn (__fmul_rn (__fmul_rn (a.w1, b.w1), c.w1), p[0]);
        s = __fadd_rn (s, __fmul_rn (__fmul_rn (__fmul_rn (a.w2, b.w1), c.w1), p[1]));
        s = __fadd_rn (s, __fmul_rn (__fmul_rn (__fmul_rn (a.w1, b.w2), c.w1), p[dx]));
        s = __fadd_rn (s, __fmul_rn (__fmul_rn (__fmul_rn (a.w2, b.w2), c.w1), p[dx + 1]));
        s = __fadd_rn (s, __fmul_rn (__fmul_rn (__fmul_rn (a.w1, b.w1), c.w2), p[dxy]));
        s = __fadd_rn (s, __fmul_rn (__fmul_rn (__fmul_rn (a.w2, b.w1), c.w2), p[dxy + 1]));
        s = __fadd_rn (s, __fmul_rn (__fmul_rn (__fmul_rn (a.w1, b.w2), c.w2), p[dxy + dx]));
        s = __fadd_rn (s, __fmul_rn (__fmul_rn (__fmul_rn (a.w2, b.w2), c.w2), p[dxy + dx + 1]));
        out[v] = s;
    }
}

static bool
on_device (const void* p)
{
    cudaPointerAttributes a;
    if (!p || cudaPointerGetAttributes (&a, p) != cudaSuccess) {
        cudaGetLastError ();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

} // namespace b200

using namespace b200;

extern "C" int
b200bsp_resample_geometry (const b200bsp_volume* in, int type,
    const float rate[3], b200bsp_volume* out, int* is_copy)
{
    if (!in || !rate || !out) return static_fail (B200BSP_E_BADARG, "null argument");
    if (type < B200BSP_RESAMPLE_VOXEL || type > B200BSP_RESAMPLE_PERCENT) {
        return static_fail (B200BSP_E_BADARG, "unknown resample type");
    }
    for (int d = 0; d < 3; d++) {
        if (in->dim[d] < 1 || !(rate[d] > 0.f)) {
            return static_fail (B200BSP_E_BADARG,
                "need dim >= 1 and a positive rate on every axis");
        }
    }
    b200bsp_volume o = *in;
    const bool voxel = type == B200BSP_RESAMPLE_VOXEL
        || type == B200BSP_RESAMPLE_VOXEL_LEGACY;
    const bool copy = voxel && rate[0] == 1.0f && rate[1] == 1.0f
        && rate[2] == 1.0f;
    if (!copy) {
        for (int d = 0; d < 3; d++) {
            const int64_t dim = in->dim[d];
            const float sp = in->spacing[d];
            if (type == B200BSP_RESAMPLE_VOXEL) {
                const long long r = round_long ((double) rate[d]);
                o.dim[d] = (dim + r - 1) / r;
                o.origin[d] = in->origin[d];
                o.spacing[d] = sp * (float) r;
            } else if (type == B200BSP_RESAMPLE_VOXEL_LEGACY) {
                const float in_size = (float) dim * sp;
                o.dim[d] = dim / (int64_t) rate[d];
                if (o.dim[d] < 1) o.dim[d] = 1;
                o.spacing[d] = in_size / (float) o.dim[d];
                o.origin[d] = (float) (in->origin[d] - 0.5 * sp
                    + 0.5 * o.spacing[d]);
            } else if (type == B200BSP_RESAMPLE_MM) {
                const float in_size = (float) (dim - 1) * sp;
                o.dim[d] = 1 + round_long ((double) (in_size / rate[d]));
                o.origin[d] = in->origin[d];
                o.spacing[d] = rate[d];
            } else {
                const float in_size = (float) (dim - 1) * sp;
                o.dim[d] = 1 + round_long ((double) (rate[d] * (float) (dim - 1)));
                o.spacing[d] = o.dim[d] == 1 ? in_size
                    : in_size / (float) (o.dim[d] - 1);
                o.origin[d] = in->origin[d];
            }
        }
    }
    *out = o;
    if (is_copy) *is_copy = copy ? 1 : 0;
    return B200BSP_OK;
}

extern "C" int
b200bsp_resample (const b200bsp_volume* in, const float* in_img,
    const b200bsp_volume* out, float* out_img, int device)
{
    if (!in || !in_img || !out || !out_img) {
        return static_fail (B200BSP_E_BADARG, "null argument");
    }
    long long ni = 1, no = 1;
    for (int d = 0; d < 3; d++) {
        if (in->dim[d] < 1 || out->dim[d] < 1 || !(in->spacing[d] != 0.f)) {
            return static_fail (B200BSP_E_BADARG, "bad geometry");
        }
        ni *= in->dim[d];
        no *= out->dim[d];
    }
    if (ni >= (1LL << 31) || no >= (1LL << 31)) {
        return static_fail (B200BSP_E_UNSUPPORTED, "volumes must have < 2^31 voxels");
    }
    if (cudaSetDevice (device) != cudaSuccess) {
        cudaGetLastError ();
        return static_fail (B200BSP_E_CUDA, "no such device");
    }
    const long long nt = out->dim[0] + out->dim[1] + out->dim[2];
    std::vector<AxisTap> taps ((size_t) nt);
    AxisTap* t[3] = {taps.data (), taps.data () + out->dim[0],
        taps.data () + out->dim[0] + out->dim[1]};
    for (int d = 0; d < 3; d++) {
        axis_taps (t[d], out->dim[d], out->origin[d], out->spacing[d],
            in->origin[d], in->spacing[d], in->dim[d]);
    }
    const bool in_dev = on_device (in_img), out_dev = on_device (out_img);
    float *d_in = nullptr, *d_out = nullptr;
    AxisTap* d_taps = nullptr;
    int rc = B200BSP_OK;
    auto ck = [&](cudaError_t e) {
        if (e != cudaSuccess && rc == B200BSP_OK) {
            cudaGetLastError ();
            rc = static_fail (e == cudaErrorMemoryAllocation ? B200BSP_E_OOM
                : B200BSP_E_CUDA, cudaGetErrorString (e));
        }
    };
    ck (cudaMalloc (&d_taps, nt * sizeof (AxisTap)));
    if (!in_dev) ck (cudaMalloc (&d_in, ni * sizeof (float)));
    if (!out_dev) ck (cudaMalloc (&d_out, no * sizeof (float)));
    if (rc == B200BSP_OK) {
        ck (cudaMemcpy (d_taps, taps.data (), nt * sizeof (AxisTap),
            cudaMemcpyHostToDevice));
        if (!in_dev) {
            ck (cudaMemcpy (d_in, in_img, ni * sizeof (float),
                cudaMemcpyHostToDevice));
        }
    }
    if (rc == B200BSP_OK) {
        const long long blocks = std::min ((no + 255) / 256, 148LL * 16);
        resample_li_kernel<<<(unsigned) blocks, 256>>> ((int) out->dim[0],
            (int) out->dim[1], (int) out->dim[2], (int) in->dim[0],
            (int) in->dim[1], d_taps, d_taps + out->dim[0],
            d_taps + out->dim[0] + out->dim[1], in_dev ? in_img : d_in,
            out_dev ? out_img : d_out);
        ck (cudaGetLastError ());
        ck (cudaDeviceSynchronize ());
        if (!out_dev) {
            ck (cudaMemcpy (out_img, d_out, no * sizeof (float),
                cudaMemcpyDeviceToHost));
        }
    }
    cudaFree (d_taps); cudaFree (d_in); cudaFree (d_out);
    return rc;
}
