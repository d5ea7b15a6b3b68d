#include "mi.cuh"
#include "../../include/plastimatch_b200.h"

namespace b200 {
int mi_alloc (MiState* s, const BspGeom&, int bins, int, const TcPlan&,
    const PartLayout&, int) { s->bins = bins; return 0; }
void mi_free (MiState*) {}
int mi_set_images (MiState*, const BspGeom&, const float*, const float*,
    size_t, size_t, cudaStream_t) { return 0; }
int mi_run (MiState*, const BspGeom&, int, const TcPlan&, const PartLayout&,
    const float*, const float*, const float*, const float*, const void*,
    float*, double*, int*, int*, float*, double*, cudaStream_t, int*)
{ return B200BSP_E_UNSUPPORTED; }
int mi_fetch (MiState*, MiResult*, double*, double*, double*, cudaStream_t)
{ return B200BSP_E_UNSUPPORTED; }
void mi_finish (MiState*, MiResult*) {}
}
