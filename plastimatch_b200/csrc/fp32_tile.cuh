// Plain FP32 SIMT tile kernel shared by the metrics: one CTA per B-spline
// tile, the 64-tap field evaluated directly per voxel, a metric functor
// turning each voxel's sample into dc/dv, and the per-tile adjoint condense
// (bspline_update_sets_b, Plastimatch src/register/bspline.cxx:347-374).
//
// Functor interface:
//   __device__ bool voxel (const BspGeom&, int fidx, const Sample&,
//       const Corners&, float dc[3], double& score) const
// returns whether the voxel counts (num_vox) and fills dc/dv.
#pragma once

#include "bsp_common.cuh"
#include "kernels.cuh"

namespace b200 {

constexpr int FP32_THREADS = 128;

template <class F>
__global__ void __launch_bounds__ (FP32_THREADS)
fp32_tile_kernel (BspGeom g, F fn, const float* __restrict__ mimg,
    const float* __restrict__ coeff, const float* __restrict__ luts,
    float* __restrict__ part, double* __restrict__ score_part,
    int* __restrict__ count_part)
{
    extern __shared__ float sm[];
    const int vx = g.vpr[0], vy = g.vpr[1], vz = g.vpr[2];
    const int V = vx * vy * vz;
    float* sC = sm;                    // 64 knots x 3
    float* sbx = sC + 192;             // 4*vx
    float* sby = sbx + 4 * vx;         // 4*vy
    float* sbz = sby + 4 * vy;         // 4*vz
    float* sdc = sbz + 4 * vz;         // V x 3 dc/dv
    __shared__ double sh_v[FP32_THREADS / 32];
    __shared__ int sh_n[FP32_THREADS / 32];

    const int t = blockIdx.x;
    const int tx = t % g.rdims[0];
    const int ty = (t / g.rdims[0]) % g.rdims[1];
    const int tz = t / (g.rdims[0] * g.rdims[1]);

    for (int o = threadIdx.x; o < 192; o += FP32_THREADS) {
        int m = o / 3, c = o - 3 * m;
        int i = m & 3, j = (m >> 2) & 3, k = m >> 4;
        int knot = (tz + k) * g.cdims[1] * g.cdims[0]
            + (ty + j) * g.cdims[0] + (tx + i);
        sC[o] = coeff[3 * knot + c];
    }
    for (int o = threadIdx.x; o < 4 * (vx + vy + vz); o += FP32_THREADS) {
        sbx[o] = luts[o];
    }
    __syncthreads ();

    const int dx = g.mdim[0], dxy = g.mdim[0] * g.mdim[1];
    double sc = 0.0;
    int cnt = 0;
    for (int v = threadIdx.x; v < V; v += FP32_THREADS) {
        int lx = v % vx, ly = (v / vx) % vy, lz = v / (vx * vy);
        int fi = g.roi_off[0] + vx * tx + lx;
        int fj = g.roi_off[1] + vy * ty + ly;
        int fk = g.roi_off[2] + vz * tz + lz;
        float dc[3] = {0.f, 0.f, 0.f};
        const int fidx = fi + g.fdim[0] * (fj + g.fdim[1] * fk);
        if (fi < g.roi_off[0] + g.roi_dim[0] && fj < g.roi_off[1] + g.roi_dim[1]
            && fk < g.roi_off[2] + g.roi_dim[2] && roi_fixed_ok (g, fidx)) {
            float fxyz[3], d[3] = {0.f, 0.f, 0.f};
            fixed_position (g, fi, fj, fk, fxyz);
            int m = 0;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                float C = sbz[lz * 4 + k];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    float B = sby[ly * 4 + j] * C;
#pragma unroll
                    for (int i = 0; i < 4; i++, m++) {
                        float A = sbx[lx * 4 + i] * B;
                        d[0] += A * sC[3 * m + 0];
                        d[1] += A * sC[3 * m + 1];
                        d[2] += A * sC[3 * m + 2];
                    }
                }
            }
            Sample s;
            if (locate (g, fxyz, d, s) && roi_moving_ok (g, fxyz, d)) {
                Corners cr = F::kNeedCorners
                    ? load_corners (mimg, s.mvf, dx, dxy) : Corners ();
                if (fn.voxel (g, fidx, s, cr, dc, sc)) cnt++;
            }
        }
        sdc[3 * v + 0] = dc[0];
        sdc[3 * v + 1] = dc[1];
        sdc[3 * v + 2] = dc[2];
    }
    __syncthreads ();

    // Adjoint: slot m, component c sums basis weight x dc/dv over the tile
    // in the reference's voxel order (z, y, x).
    for (int o = threadIdx.x; o < 192; o += FP32_THREADS) {
        int m = o / 3, c = o - 3 * m;
        int i = m & 3, j = (m >> 2) & 3, k = m >> 4;
        float s = 0.f;
        int v = 0;
        for (int lz = 0; lz < vz; lz++) {
            float C = sbz[lz * 4 + k];
            for (int ly = 0; ly < vy; ly++) {
                float B = sby[ly * 4 + j] * C;
                for (int lx = 0; lx < vx; lx++, v++) {
                    float A = sbx[lx * 4 + i] * B;
                    s += sdc[3 * v + c] * A;
                }
            }
        }
        part[((size_t) m * g.ntiles + t) * 3 + c] = s;
    }

    block_sum<FP32_THREADS> (sc, cnt, sh_v, sh_n);
    if (threadIdx.x == 0) {
        score_part[t] = sc;
        count_part[t] = cnt;
    }
}

inline size_t
fp32_tile_smem_bytes (const BspGeom& g)
{
    size_t V = (size_t) g.vpr[0] * g.vpr[1] * g.vpr[2];
    return sizeof (float) * (192 + 4 * (g.vpr[0] + g.vpr[1] + g.vpr[2])
        + 3 * V);
}

template <class F>
cudaError_t
launch_fp32_tile (const BspGeom& g, const F& fn, const float* mimg,
    const float* coeff, const float* luts, float* part, double* score_part,
    int* count_part, cudaStream_t st)
{
    size_t smem = fp32_tile_smem_bytes (g);
    auto k = fp32_tile_kernel<F>;
    if (smem > 48 * 1024) {
        cudaError_t e = set_max_dynamic_smem ((const void*) k, (int) smem);
        if (e != cudaSuccess) return e;
    }
    k<<<g.ntiles, FP32_THREADS, smem, st>>> (g, fn, mimg, coeff, luts, part,
        score_part, count_part);
    return cudaGetLastError ();
}

} // namespace b200
