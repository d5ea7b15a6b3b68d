// Analytic B-spline regulariser on the device: state and entry points.
#pragma once

#include <vector>
#include <cuda_runtime.h>

#include "../../include/plastimatch_b200.h"
#include "bsp_common.cuh"

namespace b200 {

constexpr int REG_T1_MAX = 18;     // 3 components x 6 x-axis factors
constexpr int REG_T2_MAX = 48;     // 3 components x 16 (y, x) factor pairs
constexpr int REG_E_MAX = 64;      // z-axis entries of the final pass

// Which partial products each pass forms (built on the host from the
// weights; terms with zero weight are dropped).
struct RegPlan {
    int n1;                         // pass 1: x-axis filters
    unsigned char t1_c[REG_T1_MAX], t1_xf[REG_T1_MAX];
    int n2;                         // pass 2: y-axis filters of pass-1 fields
    unsigned char t2_src[REG_T2_MAX], t2_yf[REG_T2_MAX];
    int ne;                         // pass 3: z-axis bands into outputs
    unsigned char e_src[REG_E_MAX], e_out[REG_E_MAX];
    // pass 3's entries grouped by output (stable, so each output sums its
    // entries in the order they were formed): output o takes entries
    // e_off[o] .. e_off[o + 1] - 1 of the nine
    unsigned char e_off[10];
};

struct RegState {
    int cdims[3] = {0, 0, 0};
    int nknots = 0;
    double gs[3] = {0, 0, 0};       // grid spacing per axis
    double* d_gx = nullptr;         // [6][cdims0][7] knot-x bands
    double* d_gy = nullptr;         // [6][cdims1][7] knot-y bands
    double* d_hz = nullptr;         // [REG_E_MAX][cdims2][7] weighted z bands
    double* d_t1 = nullptr;         // [REG_T1_MAX][nknots]
    double* d_t2 = nullptr;         // [REG_T2_MAX][nknots]
    double* d_part = nullptr;       // per-block score partials
    unsigned* d_arrive = nullptr;   // blocks of pass 3 done (zero between runs)
    double* d_score = nullptr;
    double* h_score = nullptr;
    int nblocks = 0;
    RegPlan plan;
    bool have_parms = false;
    b200bsp_reg_parms parms;
    std::vector<double> gz_host;    // [6][cdims2][7] unweighted z bands
};

int reg_alloc (RegState* s, const BspGeom& g, const float grid_spac[3]);
void reg_free (RegState* s);
// d_grad: the gradient is added into it (float, one double rounding per
// entry); d_grad64 (instead): stored there in double.  The score goes to
// s->d_score (double).
int reg_run (RegState* s, const BspGeom& g, const b200bsp_reg_parms* p,
    const float* d_coeff, float* d_grad, cudaStream_t st,
    double* d_grad64 = nullptr);
int reg_fetch (RegState* s, double* score, cudaStream_t st);

} // namespace b200
