// The graph-resident L-BFGS controller kernels (lbfgs_graph.cu).
#pragma once

#include <cuda_runtime.h>

#include "../../include/plastimatch_b200.h"
#include "lbfgs_logic.cuh"

namespace b200 {

// Start of a line search (after the correction pair, the two-loop
// recursion and gp.d): the search's state and its first trial step; ends
// the run (h_while) when the step or the direction is unusable.  dginit is
// the sum of slot LP_DG0 of part (nparts partials per slot), or, with part
// NULL, already in s.  Launched with one warp.
__global__ void lb_begin_search_kernel (LbDev* s,
    cudaGraphConditionalHandle h_while, const double* part, int nparts);

// After an evaluation: g.d, x.x and g.g from slots LP_GD, LP_XX and LP_GG
// of part, then the progress rule, the line search's tests, and either the
// next trial step, a new line search (h_new) or the end of the run
// (h_while).  Launched with one warp.
__global__ void lb_after_eval_kernel (LbDev* s,
    cudaGraphConditionalHandle h_while, cudaGraphConditionalHandle h_new,
    const double* part, int nparts);

}  // namespace b200
