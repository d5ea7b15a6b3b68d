// Device-side geometry and per-voxel steps of the B-spline cost function,
// shared by every kernel form.
//
// Each helper restates one step of the reference's voxel loop
// (Plastimatch src/register/bspline_mse.cxx:519-720, flavour g):
//   world position      POSITION_FROM_COORDS   src/base/volume_macros.h:78-94
//   correspondence      bspline_find_correspondence_dcos
//                                              src/util/bspline_correspond.cxx:80-107
//   inside test         Volume::is_inside      src/base/volume.cxx:900-906
//   clamp + fractions   li_clamp               src/base/interpolate.cxx:17-41
//   trilinear value     li_value               src/base/interpolate.cxx:135-158
//   trilinear gradient  li_value_dx/dy/dz      src/base/interpolate.cxx:161-257
// Linear voxel indices are 32-bit: volumes are limited to < 2^31 voxels
// (checked when a context is created).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace b200 {

// Geometry of one evaluation, passed by value to every kernel.
struct BspGeom {
    int fdim[3];          // fixed image dims (x fastest)
    float img_origin[3];  // B-spline grid's image origin (Bspline_xform::img_origin)
    float fstep[9];       // fixed step = dcos * spacing
    int mdim[3];          // moving image dims
    float morigin[3];
    float mproj[9];       // moving proj = inv(dcos) / spacing
    float minv_spacing[3];
    int roi_off[3];
    int roi_dim[3];
    int vpr[3];           // voxels per region (tile edge)
    int rdims[3];         // tiles per axis
    int cdims[3];         // knots per axis = rdims + 3
    int ntiles;
    int nknots;
    float m_hi[3];        // dim - 0.5: strict upper bound of the inside test
    float m_fmax[3];      // dim - 2: largest floor corner after clamping
    // Image ROIs (Bspline_state::fixed_roi / moving_roi; null: none).  The
    // fixed one as a byte per fixed voxel: bit 0 its ROI test at the
    // voxel's position (origin + step * ijk), bit 1 at the position the
    // reference's whole-image MI scan accumulates (LOOP_X).  The moving one
    // as its mask volume and geometry, tested at each moving position.
    const uint8_t* fmask;
    const uint8_t* mroi;
    int mroi_dim[3];
    float mroi_origin[3];
    float mroi_proj[9];
};

// The fixed ROI test of voxel fidx (bit 0, or bit 1 for the whole-image
// histogram scan).
__device__ __forceinline__ bool
roi_fixed_ok (const BspGeom& g, int fidx, int bit = 1)
{
    return !g.fmask || (__ldg (g.fmask + fidx) & bit);
}

// inside_roi (src/util/bspline_correspond.cxx:52-74): project the world
// position into the ROI volume in the reference's float order (PROJECT_X/
// Y/Z, no contraction), clamp each index to [0, dim - 1] (floor inside,
// float_to_plm_long_clamp :11-50), read the mask (nonzero: inside).
__device__ __forceinline__ bool
inside_roi_dev (const uint8_t* mask, const int dim[3], const float origin[3],
    const float proj[9], const float xyz[3])
{
    float tmp[3];
#pragma unroll
    for (int d = 0; d < 3; d++) tmp[d] = __fsub_rn (xyz[d], origin[d]);
    int p[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const float pf = __fadd_rn (__fadd_rn (__fmul_rn (tmp[0], proj[3 * d]),
            __fmul_rn (tmp[1], proj[3 * d + 1])), __fmul_rn (tmp[2], proj[3 * d + 2]));
        // pf >= dim (as float) -> dim - 1; pf < 0 (or NaN) -> 0
        p[d] = pf >= (float) dim[d] ? dim[d] - 1
            : (pf > 0.f ? (int) floorf (pf) : 0);
    }
    return __ldg (mask + p[0] + dim[0] * (p[1] + dim[1] * p[2])) != 0;
}

// The moving ROI test at the moving position mxyz = fxyz + dxyz
// (bspline_find_correspondence_dcos_roi, src/util/bspline_correspond.cxx:
// 112-145).
__device__ __forceinline__ bool
roi_moving_ok (const BspGeom& g, const float fxyz[3], const float dxyz[3])
{
    if (!g.mroi) return true;
    const float mxyz[3] = {__fadd_rn (fxyz[0], dxyz[0]),
        __fadd_rn (fxyz[1], dxyz[1]), __fadd_rn (fxyz[2], dxyz[2])};
    return inside_roi_dev (g.mroi, g.mroi_dim, g.mroi_origin, g.mroi_proj,
        mxyz);
}

// Where one fixed voxel lands in the moving image.
struct Sample {
    int mvf;        // linear index of the floor corner
    int mvr;        // linear index of the nearest ("round") voxel
    float w1[3];    // fraction for the lower corner, per axis
    float w2[3];    // fraction for the upper corner, per axis
    int clamp;      // bit d: li_clamp held the position at an end of axis d
};

// World position of fixed voxel (i, j, k): origin + step * ijk.
__device__ __forceinline__ void
fixed_position (const BspGeom& g, int i, int j, int k, float xyz[3])
{
#pragma unroll
    for (int d = 0; d < 3; d++) {
        xyz[d] = g.img_origin[d] + i * g.fstep[3*d+0] + j * g.fstep[3*d+1]
            + k * g.fstep[3*d+2];
    }
}

// Project the displaced position into the moving image, test that it lies
// strictly inside (-0.5, dim-0.5) on every axis and compute the clamped
// trilinear corner and fractions.  Returns false when outside.
__device__ __forceinline__ bool
locate (const BspGeom& g, const float fxyz[3], const float dxyz[3], Sample& s)
{
    float t0 = (fxyz[0] + dxyz[0]) - g.morigin[0];
    float t1 = (fxyz[1] + dxyz[1]) - g.morigin[1];
    float t2 = (fxyz[2] + dxyz[2]) - g.morigin[2];
    int f[3], r[3];
    s.clamp = 0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        float ma = t0 * g.mproj[3*d+0] + t1 * g.mproj[3*d+1]
            + t2 * g.mproj[3*d+2];
        if (!(ma > -0.5f && ma < (float) g.mdim[d] - 0.5f)) return false;
        int dmax = g.mdim[d] - 1;
        float w2;
        if (ma < 0.f || ma >= (float) dmax) s.clamp |= 1 << d;
        if (ma < 0.f) {
            f[d] = 0; r[d] = 0; w2 = 0.f;
        } else if (ma >= (float) dmax) {
            f[d] = dmax - 1; r[d] = dmax; w2 = 1.f;
        } else {
            float fl = floorf (ma);
            f[d] = (int) fl;
            w2 = ma - fl;                  // exact: ma and fl are close
            r[d] = f[d] + (w2 >= 0.5f);    // == (long)((double)ma + 0.5)
        }
        s.w2[d] = w2;
        s.w1[d] = 1.f - w2;
    }
    s.mvf = f[0] + g.mdim[0] * (f[1] + g.mdim[1] * f[2]);
    s.mvr = r[0] + g.mdim[0] * (r[1] + g.mdim[1] * r[2]);
    return true;
}

// Branch-free form of locate(): the same inside test, and the clamp of
// li_clamp written as floor -> clamp to [0, dim-2] -> fraction saturated to
// [0, 1], which reproduces all three of li_clamp's cases exactly
// (ma < 0: corner 0, fraction 0; ma >= dim-1: corner dim-2, fraction 1;
// otherwise floor and ma - floor).  Round index = corner + (fraction >= .5).
__device__ __forceinline__ bool
locate_fast (const BspGeom& g, const float fxyz[3], const float dxyz[3],
    int& mvf, int& mvr, float w2[3])
{
    float t0 = (fxyz[0] + dxyz[0]) - g.morigin[0];
    float t1 = (fxyz[1] + dxyz[1]) - g.morigin[1];
    float t2 = (fxyz[2] + dxyz[2]) - g.morigin[2];
    bool in = true;
    int f[3], r[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        float ma = t0 * g.mproj[3*d+0] + t1 * g.mproj[3*d+1]
            + t2 * g.mproj[3*d+2];
        in = in && (ma > -0.5f) && (ma < g.m_hi[d]);
        float fc = fminf (fmaxf (floorf (ma), 0.f), g.m_fmax[d]);
        float w = __saturatef (ma - fc);
        w2[d] = w;
        f[d] = (int) fc;
        r[d] = f[d] + (w >= 0.5f ? 1 : 0);
    }
    mvf = f[0] + g.mdim[0] * (f[1] + g.mdim[1] * f[2]);
    mvr = r[0] + g.mdim[0] * (r[1] + g.mdim[1] * r[2]);
    return in;
}

// locate_fast with the clamp flags: bit d set where li_clamp holds the
// position at an end of axis d (ma < 0 or ma >= dim - 1).
__device__ __forceinline__ bool
locate_fast_c (const BspGeom& g, const float fxyz[3], const float dxyz[3],
    int& mvf, int& mvr, float w2[3], int& clamp)
{
    float t0 = (fxyz[0] + dxyz[0]) - g.morigin[0];
    float t1 = (fxyz[1] + dxyz[1]) - g.morigin[1];
    float t2 = (fxyz[2] + dxyz[2]) - g.morigin[2];
    bool in = true;
    int f[3], r[3];
    clamp = 0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        float ma = t0 * g.mproj[3*d+0] + t1 * g.mproj[3*d+1]
            + t2 * g.mproj[3*d+2];
        in = in && (ma > -0.5f) && (ma < g.m_hi[d]);
        if (ma < 0.f || ma >= g.m_fmax[d] + 1.f) clamp |= 1 << d;
        float fc = fminf (fmaxf (floorf (ma), 0.f), g.m_fmax[d]);
        float w = __saturatef (ma - fc);
        w2[d] = w;
        f[d] = (int) fc;
        r[d] = f[d] + (w >= 0.5f ? 1 : 0);
    }
    mvf = f[0] + g.mdim[0] * (f[1] + g.mdim[1] * f[2]);
    mvr = r[0] + g.mdim[0] * (r[1] + g.mdim[1] * r[2]);
    return in;
}

// Conversion-free variants for the hot loops: the XU pipe (int <-> float,
// floor, float -> bf16) is narrow, so the per-sample path uses integer and
// FMA-pipe arithmetic instead.  The magic constant 2^23 = 8388608 puts an
// integer-valued float's value in the low mantissa bits.

// (float) i for 0 <= i < 2^23.
__device__ __forceinline__ float
i2f_small (int i)
{
    return __int_as_float (i + 0x4B000000) - 8388608.f;
}

// As locate_fast, without XU instructions: floor(max(ma, 0)) comes from an
// add with round-down to 2^23 (ma is first clamped to [0, 2^22]).  Same
// results as locate() / li_clamp for every input.
__device__ __forceinline__ bool
locate_nx (const BspGeom& g, const float fxyz[3], const float dxyz[3],
    int& mvf, int& mvr, float w2[3])
{
    float t0 = (fxyz[0] + dxyz[0]) - g.morigin[0];
    float t1 = (fxyz[1] + dxyz[1]) - g.morigin[1];
    float t2 = (fxyz[2] + dxyz[2]) - g.morigin[2];
    bool in = true;
    int f[3], r[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        float ma = t0 * g.mproj[3*d+0] + t1 * g.mproj[3*d+1]
            + t2 * g.mproj[3*d+2];
        in = in && (ma > -0.5f) && (ma < g.m_hi[d]);
        float mc = fminf (fmaxf (ma, 0.f), 4194304.f);
        float big = __fadd_rd (mc, 8388608.f);            // 2^23 + floor(mc)
        int fi = min (__float_as_int (big) - 0x4B000000, g.mdim[d] - 2);
        float fc = fminf (big - 8388608.f, g.m_fmax[d]);
        float w = __saturatef (ma - fc);
        w2[d] = w;
        f[d] = fi;
        r[d] = fi + (w >= 0.5f ? 1 : 0);
    }
    mvf = f[0] + g.mdim[0] * (f[1] + g.mdim[1] * f[2]);
    mvr = r[0] + g.mdim[0] * (r[1] + g.mdim[1] * r[2]);
    return in;
}

// Trilinear value as nested linear interpolation (x, then y, then z).
__device__ __forceinline__ float
trilinear_lerp (const float w2[3], const float m[8])
{
    float c00 = fmaf (w2[0], m[1] - m[0], m[0]);
    float c10 = fmaf (w2[0], m[3] - m[2], m[2]);
    float c01 = fmaf (w2[0], m[5] - m[4], m[4]);
    float c11 = fmaf (w2[0], m[7] - m[6], m[6]);
    float c0 = fmaf (w2[1], c10 - c00, c00);
    float c1 = fmaf (w2[1], c11 - c01, c01);
    return fmaf (w2[2], c1 - c0, c0);
}

// Gradient of the trilinear interpolant (index space, scaled by 1/spacing).
__device__ __forceinline__ void
trilinear_lerp_grad (const BspGeom& g, const float w2[3], const float m[8],
    float out[3])
{
    float c00 = fmaf (w2[0], m[1] - m[0], m[0]);
    float c10 = fmaf (w2[0], m[3] - m[2], m[2]);
    float c01 = fmaf (w2[0], m[5] - m[4], m[4]);
    float c11 = fmaf (w2[0], m[7] - m[6], m[6]);
    float c0 = fmaf (w2[1], c10 - c00, c00);
    float c1 = fmaf (w2[1], c11 - c01, c01);
    out[2] = g.minv_spacing[2] * (c1 - c0);
    float e0 = fmaf (w2[2], c01 - c00, c00);     // y = 0 face
    float e1 = fmaf (w2[2], c11 - c10, c10);     // y = 1 face
    out[1] = g.minv_spacing[1] * (e1 - e0);
    float a0 = fmaf (w2[1], m[2] - m[0], m[0]);  // x = 0 edge, z = 0
    float a1 = fmaf (w2[1], m[6] - m[4], m[4]);  // x = 0 edge, z = 1
    float b0 = fmaf (w2[1], m[3] - m[1], m[1]);  // x = 1 edge, z = 0
    float b1 = fmaf (w2[1], m[7] - m[5], m[5]);  // x = 1 edge, z = 1
    float x0 = fmaf (w2[2], a1 - a0, a0);
    float x1 = fmaf (w2[2], b1 - b0, b0);
    out[0] = g.minv_spacing[0] * (x1 - x0);
}

// Centred cubic B-spline and its derivative (the Parzen window of the
// Mattes MI variant).
__device__ __forceinline__ float
bspline3f (float t)
{
    const float a = fabsf (t);
    if (a < 1.f) return 2.f / 3.f - a * a + 0.5f * a * a * a;
    if (a < 2.f) return (2.f - a) * (2.f - a) * (2.f - a) * (1.f / 6.f);
    return 0.f;
}

__device__ __forceinline__ float
bspline3f_d (float t)
{
    const float a = fabsf (t);
    if (a < 1.f) return -2.f * t + 1.5f * t * a;
    if (a < 2.f) return (t < 0.f ? 0.5f : -0.5f) * (2.f - a) * (2.f - a);
    return 0.f;
}

// Index-space gradient of the trilinear interpolant (w2: upper-corner
// fractions, m: corners in li_value's order); an axis in `clamp` (bit d)
// gets 0, since li_clamp holds the value constant there.
__device__ __forceinline__ void
trilinear_igrad (const float w2[3], const float m[8], int clamp, float out[3])
{
    const float w1[3] = {1.f - w2[0], 1.f - w2[1], 1.f - w2[2]};
    out[0] = w1[1] * w1[2] * (m[1] - m[0]) + w2[1] * w1[2] * (m[3] - m[2])
        + w1[1] * w2[2] * (m[5] - m[4]) + w2[1] * w2[2] * (m[7] - m[6]);
    out[1] = w1[0] * w1[2] * (m[2] - m[0]) + w2[0] * w1[2] * (m[3] - m[1])
        + w1[0] * w2[2] * (m[6] - m[4]) + w2[0] * w2[2] * (m[7] - m[5]);
    out[2] = w1[0] * w1[1] * (m[4] - m[0]) + w2[0] * w1[1] * (m[5] - m[1])
        + w1[0] * w2[1] * (m[6] - m[2]) + w2[0] * w2[1] * (m[7] - m[3]);
#pragma unroll
    for (int d = 0; d < 3; d++) {
        if (clamp & (1 << d)) out[d] = 0.f;
    }
}

// Mattes MI with cubic B-spline Parzen windows: the fixed voxel's bin is
// precomputed; the moving value's window centre in bins, the first of its
// four bins (clamped so the four stay inside [1, bins - 1]).
__device__ __forceinline__ float
parzen_centre (float v, float m_min, float m_delta)
{
    return __fdiv_rn (v - m_min, m_delta) + 2.f;
}

__device__ __forceinline__ int
parzen_first_bin (float u, int bins)
{
    return min (max ((int) floorf (u), 1), bins - 3) - 1;
}

// The eight corner values of a trilinear cell, in li_value's order.
struct Corners { float m[8]; };

__device__ __forceinline__ Corners
load_corners (const float* __restrict__ img, int mvf, int dx, int dxy)
{
    Corners c;
    c.m[0] = __ldg (img + mvf);
    c.m[1] = __ldg (img + mvf + 1);
    c.m[2] = __ldg (img + mvf + dx);
    c.m[3] = __ldg (img + mvf + dx + 1);
    c.m[4] = __ldg (img + mvf + dxy);
    c.m[5] = __ldg (img + mvf + dxy + 1);
    c.m[6] = __ldg (img + mvf + dxy + dx);
    c.m[7] = __ldg (img + mvf + dxy + dx + 1);
    return c;
}

__device__ __forceinline__ float
trilinear (const Sample& s, const Corners& c)
{
    const float* f1 = s.w1;
    const float* f2 = s.w2;
    return f1[0] * f1[1] * f1[2] * c.m[0] + f2[0] * f1[1] * f1[2] * c.m[1]
        + f1[0] * f2[1] * f1[2] * c.m[2] + f2[0] * f2[1] * f1[2] * c.m[3]
        + f1[0] * f1[1] * f2[2] * c.m[4] + f2[0] * f1[1] * f2[2] * c.m[5]
        + f1[0] * f2[1] * f2[2] * c.m[6] + f2[0] * f2[1] * f2[2] * c.m[7];
}

// Derivative of the trilinear interpolant along each index axis, scaled by
// 1/spacing (li_value_dx/dy/dz; no rotation by the direction cosines).
__device__ __forceinline__ void
trilinear_grad (const BspGeom& g, const Sample& s, const Corners& c,
    float out[3])
{
    const float* f1 = s.w1;
    const float* f2 = s.w2;
    float rx = g.minv_spacing[0], ry = g.minv_spacing[1];
    float rz = g.minv_spacing[2];
    out[0] = rx * (f1[1] * f1[2] * (c.m[1] - c.m[0])
        + f2[1] * f1[2] * (c.m[3] - c.m[2])
        + f1[1] * f2[2] * (c.m[5] - c.m[4])
        + f2[1] * f2[2] * (c.m[7] - c.m[6]));
    out[1] = ry * (f1[0] * f1[2] * (c.m[2] - c.m[0])
        + f2[0] * f1[2] * (c.m[3] - c.m[1])
        + f1[0] * f2[2] * (c.m[6] - c.m[4])
        + f2[0] * f2[2] * (c.m[7] - c.m[5]));
    out[2] = rz * (f1[0] * f1[1] * (c.m[4] - c.m[0])
        + f2[0] * f1[1] * (c.m[5] - c.m[1])
        + f1[0] * f2[1] * (c.m[6] - c.m[2])
        + f2[0] * f2[1] * (c.m[7] - c.m[3]));
}

// Deterministic block-wide sum of a double and an int (fixed tree order).
template <int NT>
__device__ __forceinline__ void
block_sum (double& v, int& n, double* sh_v, int* sh_n)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v += __shfl_down_sync (0xffffffffu, v, o);
        n += __shfl_down_sync (0xffffffffu, n, o);
    }
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { sh_v[w] = v; sh_n[w] = n; }
    __syncthreads ();
    if (w == 0) {
        v = (l < NT / 32) ? sh_v[l] : 0.0;
        n = (l < NT / 32) ? sh_n[l] : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            v += __shfl_down_sync (0xffffffffu, v, o);
            n += __shfl_down_sync (0xffffffffu, n, o);
        }
    }
}

} // namespace b200
