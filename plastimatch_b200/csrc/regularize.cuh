// Analytic B-spline regulariser on the device: state and entry points.
#pragma once

#include <cuda_runtime.h>

#include "../../include/plastimatch_b200.h"
#include "bsp_common.cuh"

namespace b200 {

struct RegState {
    double* d_bands = nullptr;     // per-axis banded 1-D operators
    double* d_score = nullptr;
    double* h_score = nullptr;
    float* d_tmp = nullptr;
    int nterms = 0;
};

int reg_alloc (RegState* s, const BspGeom& g);
void reg_free (RegState* s);
int reg_run (RegState* s, const BspGeom& g, const b200bsp_reg_parms* p,
    const float* d_coeff, float* d_grad, cudaStream_t st);
int reg_fetch (RegState* s, double* score, cudaStream_t st);

} // namespace b200
