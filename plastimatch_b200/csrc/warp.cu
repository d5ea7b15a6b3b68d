// Dense displacement field and warped moving image on the fixed grid:
//   field   bspline_interpolate_vf (Plastimatch src/base/
//           bspline_interpolate.cxx:112-142) -- the B-spline displacement at
//           every ROI voxel, xyz interleaved, zero outside the ROI
//   warp    bspline_warp_dcos with linear interpolation on a float image
//           (src/base/bspline_warp.cxx:28-160) -- the moving image sampled
//           trilinearly (LI_VALUE, src/base/interpolate_macros.h:23-38) at
//           every displaced fixed voxel, default_value where the displaced
//           position falls outside the moving image
// One CTA per B-spline tile: the tile's 64 knots and the basis tables sit
// in shared memory, one thread per voxel.  Both outputs are written once
// per voxel, so the kernel is bound by the output stream (12 B/voxel field,
// 4 B/voxel warp) and the moving-image gather.
#include "bsp_common.cuh"
#include "kernels.cuh"

namespace b200 {

constexpr int FW_THREADS = 128;

// Trilinear moving value with the reference's weight products and sum
// order (LI_VALUE): products ((w_x w_y) w_z) m, added corner by corner.
__device__ __forceinline__ float
li_value_ref (const Sample& s, const float* __restrict__ m, int dx, int dxy)
{
    const float* a = s.w1;
    const float* b = s.w2;
    const float* p = m + s.mvf;
    float v = __fmul_rn (__fmul_rn (__fmul_rn (a[0], a[1]), a[2]), __ldg (p));
    v = __fadd_rn (v, __fmul_rn (__fmul_rn (__fmul_rn (b[0], a[1]), a[2]),
        __ldg (p + 1)));
    v = __fadd_rn (v, __fmul_rn (__fmul_rn (__fmul_rn (a[0], b[1]), a[2]),
        __ldg (p + dx)));
    v = __fadd_rn (v, __fmul_rn (__fmul_rn (__fmul_rn (b[0], b[1]), a[2]),
        __ldg (p + dx + 1)));
    v = __fadd_rn (v, __fmul_rn (__fmul_rn (__fmul_rn (a[0], a[1]), b[2]),
        __ldg (p + dxy)));
    v = __fadd_rn (v, __fmul_rn (__fmul_rn (__fmul_rn (b[0], a[1]), b[2]),
        __ldg (p + dxy + 1)));
    v = __fadd_rn (v, __fmul_rn (__fmul_rn (__fmul_rn (a[0], b[1]), b[2]),
        __ldg (p + dxy + dx)));
    v = __fadd_rn (v, __fmul_rn (__fmul_rn (__fmul_rn (b[0], b[1]), b[2]),
        __ldg (p + dxy + dx + 1)));
    return v;
}

template <bool WARP>
__global__ void __launch_bounds__ (FW_THREADS)
field_warp_kernel (BspGeom g, const float* __restrict__ coeff,
    const float* __restrict__ luts, const float* __restrict__ mimg,
    float default_value, float* __restrict__ vf, float* __restrict__ out)
{
    __shared__ float sC[192];
    __shared__ float slut[4 * 3 * 64];
    const int vx = g.vpr[0], vy = g.vpr[1], vz = g.vpr[2];
    const int V = vx * vy * vz;
    const int t = blockIdx.x;
    const int tx = t % g.rdims[0];
    const int ty = (t / g.rdims[0]) % g.rdims[1];
    const int tz = t / (g.rdims[0] * g.rdims[1]);
    for (int o = threadIdx.x; o < 192; o += FW_THREADS) {
        const int m = o / 3, c = o - 3 * m;
        const int i = m & 3, j = (m >> 2) & 3, k = m >> 4;
        sC[o] = coeff[3 * ((tz + k) * g.cdims[1] * g.cdims[0]
            + (ty + j) * g.cdims[0] + (tx + i)) + c];
    }
    for (int o = threadIdx.x; o < 4 * (vx + vy + vz); o += FW_THREADS) {
        slut[o] = luts[o];
    }
    __syncthreads ();
    const float* sbx = slut;
    const float* sby = slut + 4 * vx;
    const float* sbz = sby + 4 * vy;
    const int dx = g.mdim[0], dxy = g.mdim[0] * g.mdim[1];
    for (int v = threadIdx.x; v < V; v += FW_THREADS) {
        const int lx = v % vx, ly = (v / vx) % vy, lz = v / (vx * vy);
        const int fi = g.roi_off[0] + vx * tx + lx;
        const int fj = g.roi_off[1] + vy * ty + ly;
        const int fk = g.roi_off[2] + vz * tz + lz;
        if (fi >= g.roi_off[0] + g.roi_dim[0]
            || fj >= g.roi_off[1] + g.roi_dim[1]
            || fk >= g.roi_off[2] + g.roi_dim[2]) continue;
        float d[3] = {0.f, 0.f, 0.f};
        int m = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float C = sbz[lz * 4 + k];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const float B = sby[ly * 4 + j] * C;
#pragma unroll
                for (int i = 0; i < 4; i++, m++) {
                    const float A = sbx[lx * 4 + i] * B;
                    d[0] += A * sC[3 * m + 0];
                    d[1] += A * sC[3 * m + 1];
                    d[2] += A * sC[3 * m + 2];
                }
            }
        }
        const long long fidx = fi + (long long) g.fdim[0]
            * (fj + (long long) g.fdim[1] * fk);
        if (vf) {
            vf[3 * fidx + 0] = d[0];
            vf[3 * fidx + 1] = d[1];
            vf[3 * fidx + 2] = d[2];
        }
        if (WARP) {
            float fxyz[3];
            fixed_position (g, fi, fj, fk, fxyz);
            Sample s;
            out[fidx] = locate (g, fxyz, d, s)
                ? li_value_ref (s, mimg, dx, dxy) : default_value;
        }
    }
}

cudaError_t
launch_field_warp (const BspGeom& g, const float* coeff, const float* luts,
    const float* mimg, float default_value, float* vf, float* warped,
    cudaStream_t st)
{
    if (warped) {
        field_warp_kernel<true><<<g.ntiles, FW_THREADS, 0, st>>> (g, coeff,
            luts, mimg, default_value, vf, warped);
    } else {
        field_warp_kernel<false><<<g.ntiles, FW_THREADS, 0, st>>> (g, coeff,
            luts, mimg, default_value, vf, nullptr);
    }
    return cudaGetLastError ();
}

} // namespace b200
