// The controller of the graph-resident L-BFGS (optimize.cu builds the
// graph): single-thread kernels that run the line-search and iteration
// logic of the host-driven loop on the device, between the vector kernels
// and the evaluations, and steer the graph's conditional nodes -- the
// while loop over trial points and the branch that starts a new line
// search (correction pair, two-loop recursion, dginit).  No scalar leaves
// the device until the run ends.
//
// This file is compiled without floating-point contraction, so the
// controller rounds exactly as the host-driven loop (host code) does.
#include "lbfgs_graph.cuh"

namespace b200 {

namespace {

// The step's bracket and the safeguarded trial step (the top of each
// iteration of the Moré-Thuente loop).
__device__ void
pre_trial (LbDev* s)
{
    if (s->brackt) {
        s->stmin = lb_min (s->stx, s->sty);
        s->stmax = lb_max (s->stx, s->sty);
    } else {
        s->stmin = s->stx;
        s->stmax = s->stp + 4.0 * (s->stp - s->stx);
    }
    s->stp = lb_max (s->min_step, lb_min (s->max_step, s->stp));
    if ((s->brackt && ((s->stp <= s->stmin || s->stmax <= s->stp)
             || s->max_linesearch <= s->count + 1 || s->uinfo != 0))
        || (s->brackt && (s->stmax - s->stmin <= s->xtol * s->stmax))) {
        s->stp = s->stx;
    }
}

__device__ void
finish_run (LbDev* s, int status, cudaGraphConditionalHandle h_while)
{
    s->status = status;
    s->done = 1;
    cudaGraphSetConditional (h_while, 0);
}

}  // namespace

__global__ void
lb_begin_search_kernel (LbDev* s, cudaGraphConditionalHandle h_while,
    const double* part, int nparts)
{
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    if (part) {
        const double dg0 = lb_warp_sum (part + (size_t) LP_DG0 * nparts, nparts);
        if (threadIdx.x == 0) s->dginit = dg0;
    }
    if (threadIdx.x != 0 || s->done) return;
    s->first = 0;
    s->finit = s->f;
    if (s->stp <= 0.0) {
        finish_run (s, LS_BADSTEP, h_while);
        return;
    }
    if (0.0 < s->dginit) {
        finish_run (s, LS_INCREASE, h_while);
        return;
    }
    s->brackt = 0;
    s->stage1 = 1;
    s->uinfo = 0;
    s->count = 0;
    s->dgtest = s->ftol * s->dginit;
    s->width = s->max_step - s->min_step;
    s->prev_width = 2.0 * s->width;
    s->stx = 0.0;
    s->fx = s->finit;
    s->dgx = s->dginit;
    s->sty = 0.0;
    s->fy = s->finit;
    s->dgy = s->dginit;
    pre_trial (s);
}

__global__ void
lb_after_eval_kernel (LbDev* s, cudaGraphConditionalHandle h_while,
    cudaGraphConditionalHandle h_new, const double* part, int nparts)
{
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    {
        const double dg = lb_warp_sum (part + (size_t) LP_GD * nparts, nparts);
        const double xx = lb_warp_sum (part + (size_t) LP_XX * nparts, nparts);
        const double gg = lb_warp_sum (part + (size_t) LP_GG * nparts, nparts);
        if (threadIdx.x == 0) {
            s->dg = dg;
            s->xx = xx;
            s->gg = gg;
        }
    }
    if (threadIdx.x != 0) return;
    cudaGraphSetConditional (h_new, 0);
    if (s->done) {
        cudaGraphSetConditional (h_while, 0);
        return;
    }
    // Bspline_score's total (float) as the objective
    s->f = (double) s->total;
    s->last = s->total;
    s->fevals++;
    if (lb_stop_rule (s->max_its, s->max_feval, s->k, s->fevals)) {
        finish_run (s, LS_STOPPED, h_while);
        return;
    }
    const double f = s->f, dg = s->dg;
    const double ftest1 = s->finit + s->stp * s->dgtest;
    ++s->count;
    if (s->brackt && ((s->stp <= s->stmin || s->stmax <= s->stp)
            || s->uinfo != 0)) {
        finish_run (s, LS_ROUNDING, h_while);
        return;
    }
    if (s->stp == s->max_step && f <= ftest1 && dg <= s->dgtest) {
        finish_run (s, LS_MAXSTEP, h_while);
        return;
    }
    if (s->stp == s->min_step && (ftest1 < f || s->dgtest <= dg)) {
        finish_run (s, LS_MINSTEP, h_while);
        return;
    }
    if (s->brackt && (s->stmax - s->stmin) <= s->xtol * s->stmax) {
        finish_run (s, LS_WIDTH, h_while);
        return;
    }
    if (s->max_linesearch <= s->count) {
        finish_run (s, LS_MAXLS, h_while);
        return;
    }
    if (f <= ftest1 && fabs (dg) <= s->gtol * (-s->dginit)) {
        // the line search is done: the iteration's tests, then a new pair
        s->iterations = s->k;
        double xnorm = sqrt (s->xx), gnorm = sqrt (s->gg);
        if (lb_stop_rule (s->max_its, s->max_feval, s->k, s->fevals)) {
            finish_run (s, B200BSP_LBFGS_STOPPED, h_while);
            return;
        }
        if (xnorm < 1.0) xnorm = 1.0;
        if (gnorm / xnorm <= s->epsilon) {
            finish_run (s, B200BSP_LBFGS_CONVERGED, h_while);
            return;
        }
        s->newest = s->end;
        s->bound = s->m < s->k ? s->m : s->k;
        ++s->k;
        s->end = (s->end + 1) % s->m;
        s->stp = 1.0;
        s->newiter = 1;
        cudaGraphSetConditional (h_new, 1);
        return;
    }
    if (s->stage1 && f <= ftest1
        && lb_min (s->ftol, s->gtol) * s->dginit <= dg) {
        s->stage1 = 0;
    }
    if (s->stage1 && ftest1 < f && f <= s->fx) {
        // first stage: work on the modified function f - stp * dgtest
        const double fm = f - s->stp * s->dgtest;
        double fxm = s->fx - s->stx * s->dgtest, fym = s->fy - s->sty * s->dgtest;
        const double dgm = dg - s->dgtest;
        double dgxm = s->dgx - s->dgtest, dgym = s->dgy - s->dgtest;
        s->uinfo = lb_update_interval (&s->stx, &fxm, &dgxm, &s->sty, &fym,
            &dgym, &s->stp, fm, dgm, s->stmin, s->stmax, &s->brackt);
        s->fx = fxm + s->stx * s->dgtest;
        s->fy = fym + s->sty * s->dgtest;
        s->dgx = dgxm + s->dgtest;
        s->dgy = dgym + s->dgtest;
    } else {
        s->uinfo = lb_update_interval (&s->stx, &s->fx, &s->dgx, &s->sty,
            &s->fy, &s->dgy, &s->stp, f, dg, s->stmin, s->stmax, &s->brackt);
    }
    if (s->brackt) {
        if (0.66 * s->prev_width <= fabs (s->sty - s->stx)) {
            s->stp = s->stx + 0.5 * (s->sty - s->stx);
        }
        s->prev_width = s->width;
        s->width = fabs (s->sty - s->stx);
    }
    s->newiter = 0;
    pre_trial (s);
}

}  // namespace b200
