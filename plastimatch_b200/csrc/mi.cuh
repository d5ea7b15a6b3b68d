// Mattes mutual information (PVI-8) on the device: state and entry points.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace b200 {

constexpr int MI_MAX_BINS = 64;

struct MiResult {
    float score_f;
    double score;
    long long num_vox;
};

struct MiState {
    int bins = 0;
    bool ready = false;
    float f_offset = 0.f, f_delta = 1.f, m_offset = 0.f, m_delta = 1.f;
    unsigned long long* d_hist = nullptr;   // fixed-point histograms
    double* d_histd = nullptr;              // f, m, j histograms (double)
    float* d_lut = nullptr;                 // dS/dP per joint bin
    double* d_scal = nullptr;               // score, N
    double* h_scal = nullptr;
    double* h_hist = nullptr;
    float* d_minmax = nullptr;
};

int mi_alloc (MiState* s, const BspGeom& g, int bins, int form,
    const TcPlan& plan, const PartLayout& lay, int nparts);
void mi_free (MiState* s);
int mi_set_images (MiState* s, const BspGeom& g, const float* d_fixed,
    const float* d_moving, size_t nf, size_t nm, cudaStream_t st);
int mi_run (MiState* s, const BspGeom& g, int form, const TcPlan& plan,
    const PartLayout& lay, const float* d_fixed, const float* d_moving,
    const float* d_coeff, const float* d_luts, const void* d_qlut,
    float* d_part, double* d_score_part, int* d_count_part, int* d_err,
    float* grad_out, double* grad64_out, cudaStream_t st, int* launches);
int mi_fetch (MiState* s, MiResult* r, double* f_hist, double* m_hist,
    double* j_hist, cudaStream_t st);
void mi_finish (MiState* s, MiResult* r);

} // namespace b200
