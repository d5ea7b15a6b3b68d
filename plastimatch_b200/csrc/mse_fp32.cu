// Plain FP32 SIMT form of the MSE score + gradient: the straightforward GPU
// mapping of the reference's tile loop (Plastimatch src/register/
// bspline_mse.cxx:519-720, flavour g) and the baseline the tensor-core form
// is measured against.  The tile machinery is fp32_tile.cuh; this file
// holds the MSE voxel functor.
#include "fp32_tile.cuh"
#include "kernels.cuh"

namespace b200 {

// diff = trilinear(moving) - fixed; score += diff^2; dc/dv = diff * gradient
// (nearest-voxel moving gradient, or the trilinear derivative).
template <int GRAD_MODE>
struct MseVoxel {
    static constexpr bool kNeedCorners = true;
    const float* fimg;
    const float* mgrad;
    __device__ __forceinline__ bool
    voxel (const BspGeom& g, int fidx, const Sample& s, const Corners& cr,
        float dc[3], double& sc) const
    {
        float diff = trilinear (s, cr) - __ldg (fimg + fidx);
        sc += (double) (diff * diff);
        if (GRAD_MODE == 0) {
            dc[0] = diff * __ldg (mgrad + 3 * s.mvr + 0);
            dc[1] = diff * __ldg (mgrad + 3 * s.mvr + 1);
            dc[2] = diff * __ldg (mgrad + 3 * s.mvr + 2);
        } else {
            float gr[3];
            trilinear_grad (g, s, cr, gr);
            dc[0] = diff * gr[0];
            dc[1] = diff * gr[1];
            dc[2] = diff * gr[2];
        }
        return true;
    }
};

size_t
mse_fp32_smem_bytes (const BspGeom& g)
{
    return fp32_tile_smem_bytes (g);
}

cudaError_t
launch_mse_fp32 (const BspGeom& g, int grad_mode, const float* fimg,
    const float* mimg, const float* mgrad, const float* coeff,
    const float* luts, float* part, double* score_part, int* count_part,
    cudaStream_t st)
{
    if (grad_mode == 0) {
        MseVoxel<0> f{fimg, mgrad};
        return launch_fp32_tile (g, f, mimg, coeff, luts, part, score_part,
            count_part, st);
    }
    MseVoxel<1> f{fimg, mgrad};
    return launch_fp32_tile (g, f, mimg, coeff, luts, part, score_part,
        count_part, st);
}

} // namespace b200
