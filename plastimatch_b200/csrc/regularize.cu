#include "regularize.cuh"

namespace b200 {
int reg_alloc (RegState*, const BspGeom&) { return 0; }
void reg_free (RegState*) {}
int reg_run (RegState*, const BspGeom&, const b200bsp_reg_parms*,
    const float*, float*, cudaStream_t) { return B200BSP_E_UNSUPPORTED; }
int reg_fetch (RegState*, double*, cudaStream_t) { return B200BSP_E_UNSUPPORTED; }
}
