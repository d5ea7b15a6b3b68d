// Launch wrappers shared between the runtime and the kernel files.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "bsp_common.cuh"

namespace b200 {

// Result block written on the device by the final reduction.
struct DevResult {
    double score;        // normalised score (double)
    double raw;          // raw sum (MSE: sum diff^2)
    long long num_vox;
    float score_f;       // the float score the reference reports
    int error;           // non-zero when a bounded wait gave up
};

// How the per-tile-batch partial gradients are laid out (see gather).
struct PartLayout {
    int bx, by, bz;      // tiles per batch along x, y, z
    int nbx, nby, nbz;   // batches along x, y, z
    int kx, ky, kz;      // knots per batch footprint = b? + 3
    int slots;           // 1: footprint layout part[batch][c][knot];
                         // 64: per-tile slot layout part[slot][tile][3]
};

cudaError_t launch_mse_fp32 (const BspGeom& g, int grad_mode,
    const float* fimg, const float* mimg, const float* mgrad,
    const float* coeff, const float* luts, float* part, double* score_part,
    int* count_part, cudaStream_t st);
size_t mse_fp32_smem_bytes (const BspGeom& g);

// Tensor-core form (mse_tc.cu).
struct TcPlan {
    int bx;              // tiles per CTA batch along x
    int nbatches;
    int n_mma;           // N of the forward MMA = 3 * bx rounded up
    int mblk;            // 128-row M blocks covering one tile's voxels
    size_t smem;         // dynamic shared memory per CTA
    int tmem_cols;
    int threads;
    int grid;
};
// extra_row_batches: split each row of tiles into that many more batches
// than the fewest (the autotuner's knob); false when unsupported.
bool tc_plan (const BspGeom& g, TcPlan* plan, int ctas_per_sm, int sm_count,
    int extra_row_batches = 0);
constexpr int TC_TUNE_MAX_EXTRA = 2;      // autotuner candidates: 0 .. this
int tc_build_tables (const BspGeom& g, const TcPlan& plan, void** d_qlut);
cudaError_t launch_mse_tc (const BspGeom& g, const TcPlan& plan,
    int grad_mode, const float* fimg, const float* mimg, const float* mgrad,
    const float4* mgrad4, const float* coeff, const void* qlut_bf16,
    float* part, double* score_part, int* count_part, int* err_flag,
    unsigned wait_limit, cudaStream_t st);

// cudaFuncAttributeMaxDynamicSharedMemorySize for a kernel on the current
// device, set once per (kernel, device) and size: the attribute call is a
// host round trip that would otherwise precede every launch.
cudaError_t set_max_dynamic_smem (const void* kernel, int bytes);

// Tensor-core form, x-lane kernel (mse_xl.cu): one batch is a row of T
// tiles along x with TMEM lane = voxel x; rows of the batch in chunks of
// whole z planes (at most 32 rows).  Supports 3 <= vox_per_rgn[1] <= 10.
struct XlPlan {
    int T;               // tiles per batch along x
    int nbx;             // batches per row of tiles
    int nbatches;
    int nlz, nch;        // z planes per chunk, chunks per batch
    size_t smem;
    int threads;
    int grid;
    int score_parts;     // one per batch
};
// extra_row_batches: more batches per row of tiles than the fewest (the
// autotuner's knob).  The basis table of the fewest serves every split.
bool xl_plan (const BspGeom& g, XlPlan* plan, int sm_count,
    int extra_row_batches = 0);
int xl_build_table (const BspGeom& g, const XlPlan& plan, const float* bx_lut,
    void** d_tab);
// Polls before a device-side wait gives up (between polls the waiting
// thread sleeps up to about 1 us).
constexpr unsigned XL_DEFAULT_WAIT_LIMIT = 1u << 22;
cudaError_t launch_mse_xl (const BspGeom& g, const XlPlan& plan,
    int grad_mode, const float* fimg, const float* mimg, const float* mgrad,
    const float* coeff, const void* tab, const float* luts, float* part,
    double* score_part, int* count_part, int* err, unsigned wait_limit,
    int withhold, cudaStream_t st);

// Mattes MI on the tensor-core kernel (axis-aligned geometry, tiles of at
// most 128 voxels, histograms that fit the adjoint operand's area): pass 1
// (hist_pass: PVI-8 or Parzen histograms into mi.hist, integer 2^-24 units,
// count last) or pass 2 (dc/dv from the factor table -> per-batch
// partials).
struct TcMiArgs {
    const uint8_t* fbin;
    const uint8_t* mbin;
    int bins;
    const float* lut;            // [fixed bin][moving bin] pass-2 factors
    const float* nvf;            // voxel count as float (Parzen: [1] the
                                 // pass-2 scale 1 / (N delta_m))
    unsigned long long* hist;    // f[B], m[B], j[B*B], count
    bool parzen;                 // cubic B-spline Parzen windows
    const float* mimg;           // Parzen: the moving image
    float m_min, m_delta;        // Parzen: moving value -> window centre
};
bool tc_mi_supported (const BspGeom& g, const TcPlan& p, int bins);
// The same passes on the x-lane kernel (mse_xl.cu): pass 1 into mi.hist,
// pass 2's partial gradients into part (the x-lane batch layout).
bool xl_mi_supported (int bins);
cudaError_t launch_mi_xl (const BspGeom& g, const XlPlan& p, bool hist_pass,
    const TcMiArgs& mi, const float* coeff, const void* tab,
    const float* luts, float* part, int* err, unsigned wait_limit,
    cudaStream_t st);
cudaError_t launch_mi_tc (const BspGeom& g, const TcPlan& p, bool hist_pass,
    const TcMiArgs& mi, const float* coeff, const void* qimg, float* part,
    double* score_part, int* count_part, int* err, cudaStream_t st);
// Moving gradient xyz-interleaved -> float4 (w = 0), for 16-byte loads.
cudaError_t launch_pad_grad4 (const float* grad3, float4* grad4, long long n,
    cudaStream_t st);

// Dense field (vf, may be NULL) and/or warped moving image (warped, may be
// NULL) over the ROI's voxels (warp.cu).
cudaError_t launch_field_warp (const BspGeom& g, const float* coeff,
    const float* luts, const float* mimg, float default_value, float* vf,
    float* warped, cudaStream_t st);

// bspline_score's combination done by the finish kernel (all device
// pointers; total_score null: plain metric output): total score = lambda *
// score + reg score, gradient = lambda * metric gradient + reg gradient.
struct FinishCombine {
    float lambda = 1.f;
    const double* reg_grad = nullptr;    // [num_coeff] or null
    const double* reg_score = nullptr;   // or null
    float* total_score = nullptr;
};

// Score reduction + per-knot gradient gather, MSE normalisation, one
// launch.  err (may be null): the tile kernel's error flag, copied into the
// result block; res_host (may be null): a second copy of the result block,
// e.g. mapped host memory.  Any output may be mapped host memory.
cudaError_t launch_finish_mse (const BspGeom& g, const PartLayout& lay,
    const float* part, const double* score_part, const int* count_part,
    int nparts, const int* err, DevResult* res, DevResult* res_host,
    float* grad_out, double* grad64_out, float* score_out,
    double* score64_out, long long* nvox_out, cudaStream_t st,
    unsigned* clear = nullptr, int nclear = 0,
    const FinishCombine& combine = FinishCombine ());

cudaError_t launch_reduce_score (const double* score_part,
    const int* count_part, int n, DevResult* res, int mode,
    cudaStream_t st);
cudaError_t launch_gather_grad (const BspGeom& g, const PartLayout& lay,
    const float* part, const DevResult* res, int mode, float* grad_out,
    double* grad64_out, float* score_out, double* score64_out,
    long long* nvox_out, cudaStream_t st);
cudaError_t launch_volume_grad (const int dim[3], const float spacing[3],
    const float inv_dc[9], const float* img, float* grad, cudaStream_t st);

// Geometry of an image or ROI volume for the ROI tests: dims, origin,
// step (dcos * spacing) and proj (inv(dcos) / spacing), row-major.
struct RoiGeom {
    int dim[3];
    float origin[3];
    float step[9];
    float proj[9];
};
// Fixed ROI test of every fixed voxel into out[fdim] (bit 0 at the
// voxel's position, bit 1 at the whole-image scan's accumulated position).
cudaError_t launch_fixed_roi_mask (const int fdim[3], const RoiGeom& fixed,
    const RoiGeom& roi_geom, const uint8_t* roi, uint8_t* out,
    cudaStream_t st);

// Landmark term (landmarks.cu): n landmarks with tiles p[3n], q_lut rows
// w[64n], fixed/moving xyz fm[6n]; scratch dc[4n]; ADDS the gradient into
// grad and writes lmetric (device float).
cudaError_t launch_landmarks (const BspGeom& g, int n, const int* p,
    const float* w, const float* fm, const float* coeff, float grad_coeff,
    float* dc, float* grad, float* lmetric, cudaStream_t st);

} // namespace b200
