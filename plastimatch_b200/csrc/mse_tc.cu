#include "kernels.cuh"
#include "../../include/plastimatch_b200.h"

namespace b200 {
bool tc_plan (const BspGeom&, TcPlan*, int, int) { return false; }
int tc_build_tables (const BspGeom&, const TcPlan&, void**) { return B200BSP_E_UNSUPPORTED; }
cudaError_t launch_mse_tc (const BspGeom&, const TcPlan&, int, const float*,
    const float*, const float*, const float*, const void*, float*, double*,
    int*, int*, cudaStream_t) { return cudaErrorNotSupported; }
}
