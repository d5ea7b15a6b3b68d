// Mattes mutual information on the device (PVI-8, the reference's binning,
// or cubic B-spline Parzen windows): state and entry points.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace b200 {

constexpr int MI_MAX_BINS = 64;

struct MiResult {
    float score_f;
    double score;
    long long num_vox;
};

constexpr int MI_VOPT_KEYS = 1000;            // VOPT_RES, src/register/histogram.h:12

struct MiState {
    int bins = 0;
    int window = 0;                           // B200BSP_MI_PVI8 / _PARZEN
    int hist = 0;                             // B200BSP_MI_HIST_EQSP / _VOPT
    // V-optimal bins: offset/delta span the fine keys, key -> bin tables
    int* d_fkey = nullptr;
    int* d_mkey = nullptr;
    bool ready = false;
    // Parzen: fixed bin = floor((v - pz_fmin) / pz_fdelta) + 2; moving
    // window centre (v - pz_mmin) / pz_mdelta + 2
    float pz_fmin = 0.f, pz_fdelta = 1.f, pz_mmin = 0.f, pz_mdelta = 1.f;
    float f_offset = 0.f, f_delta = 1.f, m_offset = 0.f, m_delta = 1.f;
    uint8_t* d_fbin = nullptr;                // fixed-image bin per voxel
    uint8_t* d_mbin = nullptr;                // moving-image bin per voxel
    unsigned long long* d_hist = nullptr;     // f[B], m[B], j[B*B], N (fixed point)
    double* d_histd = nullptr;                // f, m, j as doubles
    float* d_lut = nullptr;                   // dS/dP per joint bin (0 = skip)
    float* d_nvf = nullptr;                   // num_vox as float; Parzen:
                                              // [1] = 1 / (num_vox delta_m)
    float* d_minmax = nullptr;                // per-block min/max scratch
    float* d_part = nullptr;                  // pass-2 tile partials, 64 slots
    double* d_score_part = nullptr;
    int* d_count_part = nullptr;
    double* h_histd = nullptr;
    DevResult* h_res = nullptr;
};

int mi_alloc (MiState* s, const BspGeom& g, int bins, int window,
    int hist = 0);
void mi_free (MiState* s);
int mi_set_images (MiState* s, const BspGeom& g, const float* d_fixed,
    const float* d_moving, size_t nf, size_t nm, cudaStream_t st);
// passes: MI_PASS_HIST (histograms into d_hist), MI_PASS_GRAD (score and
// gradient from the histograms in d_hist), or both
constexpr int MI_PASS_HIST = 1;
constexpr int MI_PASS_GRAD = 2;
int mi_run (MiState* s, const BspGeom& g, const float* d_coeff,
    const float* d_moving, const float* d_luts, DevResult* d_res,
    float* grad_out, double* grad64_out, cudaStream_t st, int* launches,
    int passes = MI_PASS_HIST | MI_PASS_GRAD);
int mi_run_tc (MiState* s, const BspGeom& g, const TcPlan& plan,
    const PartLayout& lay, const void* qlut, float* part, double* score_part,
    int* count_part, int* err, const float* d_coeff, const float* d_moving,
    DevResult* d_res, float* grad_out, double* grad64_out, cudaStream_t st,
    int* launches, int passes = MI_PASS_HIST | MI_PASS_GRAD);
int mi_run_xl (MiState* s, const BspGeom& g, const XlPlan& plan,
    const PartLayout& lay, const void* tab, const float* luts, float* part,
    int* err, unsigned wait_limit, const float* d_coeff,
    const float* d_moving, DevResult* d_res, float* grad_out,
    double* grad64_out, cudaStream_t st, int* launches,
    int passes = MI_PASS_HIST | MI_PASS_GRAD);
int mi_fetch (MiState* s, const DevResult* d_res, double* f_hist,
    double* m_hist, double* j_hist, cudaStream_t st);
void mi_finish (MiState* s, MiResult* r);

} // namespace b200
