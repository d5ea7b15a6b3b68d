// The scalar logic of the device L-BFGS, shared by the host-driven loop
// (optimize.cu) and the graph-resident controller (lbfgs_graph.cu, built
// without floating-point contraction so both round alike): the
// Moré-Thuente trial-interval update, the progress rule, the line-search
// status codes and the controller's state.
#pragma once

#include <cmath>

#include <cuda_runtime.h>

namespace b200 {

enum {
    LS_ROUNDING = -1001, LS_MAXSTEP = -1002, LS_MINSTEP = -1003,
    LS_WIDTH = -1004, LS_MAXLS = -1005, LS_INCREASE = -1006, LS_BADSTEP = -1007,
    LS_STOPPED = -1100      // the progress rule stopped the run mid-search
};

__host__ __device__ inline double lb_min (double a, double b) { return a < b ? a : b; }
__host__ __device__ inline double lb_max (double a, double b) { return a < b ? b : a; }

// Moré-Thuente trial-interval update (the cstep of MINPACK): x = best
// step so far (fx, dx), y = other end of the interval (fy, dy), t = trial
// step (ft, dt).  Returns 0, or an error code when the inputs are
// inconsistent (rounding errors).
__host__ __device__ inline double
lb_cubic (double u, double fu, double du, double v, double fv, double dv,
    bool clamp_zero, double* gamma_out)
{
    // minimiser of the cubic interpolating (u, fu, du) and (v, fv, dv),
    // written from u's side: returns r with minimiser u + r (v - u), and
    // gamma (zero when the cubic has no minimiser there and clamp_zero)
    const double theta = 3.0 * (fu - fv) / (v - u) + du + dv;
    const double s = lb_max (fabs (theta), lb_max (fabs (du), fabs (dv)));
    const double a = theta / s;
    double gamma2 = a * a - (du / s) * (dv / s);
    if (clamp_zero && gamma2 < 0) gamma2 = 0;
    double gamma = s * sqrt (gamma2);
    if (v < u) gamma = -gamma;
    const double p = (gamma - du) + theta;
    const double q = ((gamma - du) + gamma) + dv;
    if (gamma_out) *gamma_out = gamma;
    return p / q;
}

__host__ __device__ inline int
lb_update_interval (double* x, double* fx, double* dx, double* y, double* fy,
    double* dy, double* t, double ft, double dt, double tmin, double tmax,
    int* brackt)
{
    if (*brackt) {
        if (*t <= lb_min (*x, *y) || lb_max (*x, *y) <= *t) return 1;
        if (0.0 <= *dx * (*t - *x)) return 2;
        if (tmax < tmin) return 3;
    }
    // the derivatives differ in sign (dt * sign(dx) < 0)
    const bool dsign = dt * (*dx / fabs (*dx)) < 0.0;
    bool bound;
    double newt;
    if (*fx < ft) {
        // case 1: higher function value; the minimum is bracketed
        *brackt = 1;
        bound = true;
        const double mc = *x + lb_cubic (*x, *fx, *dx, *t, ft, dt, false,
            nullptr) * (*t - *x);
        const double mq = *x + (*dx / ((*fx - ft) / (*t - *x) + *dx)) / 2.0
            * (*t - *x);
        if (fabs (mc - *x) < fabs (mq - *x)) newt = mc;
        else newt = mc + 0.5 * (mq - mc);
    } else if (dsign) {
        // case 2: lower value, derivatives of opposite sign; bracketed
        *brackt = 1;
        bound = false;
        const double mc = *t + lb_cubic (*t, ft, dt, *x, *fx, *dx, false,
            nullptr) * (*x - *t);
        const double mq = *t + (dt / (dt - *dx)) * (*x - *t);
        if (fabs (mc - *t) > fabs (mq - *t)) newt = mc;
        else newt = mq;
    } else if (fabs (dt) < fabs (*dx)) {
        // case 3: lower value, same sign, smaller derivative magnitude
        bound = true;
        double gamma;
        const double r = lb_cubic (*t, ft, dt, *x, *fx, *dx, true, &gamma);
        double mc;
        // the cubic may have no minimiser beyond t
        if (r < 0.0 && gamma != 0.0) mc = *t + r * (*x - *t);
        else if (*x < *t) mc = tmax;
        else mc = tmin;
        const double mq = *t + (dt / (dt - *dx)) * (*x - *t);
        if (*brackt) {
            newt = fabs (*t - mc) < fabs (*t - mq) ? mc : mq;
        } else {
            newt = fabs (*t - mc) > fabs (*t - mq) ? mc : mq;
        }
    } else {
        // case 4: lower value, same sign, derivative does not decrease
        bound = false;
        if (*brackt) {
            newt = *t + lb_cubic (*t, ft, dt, *y, *fy, *dy, false, nullptr)
                * (*y - *t);
        } else if (*x < *t) {
            newt = tmax;
        } else {
            newt = tmin;
        }
    }
    // update the interval
    if (*fx < ft) {
        *y = *t; *fy = ft; *dy = dt;
    } else {
        if (dsign) {
            *y = *x; *fy = *fx; *dy = *dx;
        }
        *x = *t; *fx = ft; *dx = dt;
    }
    newt = lb_min (tmax, newt);
    newt = lb_max (tmin, newt);
    if (*brackt && bound) {
        const double mq = *x + 0.66 * (*y - *x);
        if (*x < *y) newt = lb_min (mq, newt);
        else newt = lb_max (mq, newt);
    }
    *t = newt;
    return 0;
}

// Plastimatch's progress rule (src/register/bspline_optimize_liblbfgs.cxx:
// 53-79): stop once the iteration number exceeds max_its or the function
// evaluations exceed max_feval.  The liblbfgs it links consults the rule
// after every evaluation inside a line search (with the current iteration
// number) and once more after each completed line search.
__host__ __device__ inline bool
lb_stop_rule (int max_its, int max_feval, int k, int fevals)
{
    return k > max_its || fevals > max_feval;
}

// Slots of the graph-resident run's partial sums (one block's partial per
// slot entry; each slot holds one dot product's partials): the correction
// pair's y.s and y.y, gp.d of a new line search, the evaluated point's g.d,
// x.x and g.g, then the two-loop recursion's dot products (the first loop's
// s_j.d at LP_REC + i, the second loop's y_j.d at LP_REC + m + i).
enum { LP_YS, LP_YY, LP_DG0, LP_GD, LP_XX, LP_GG, LP_REC };

#ifdef __CUDACC__
// The sum of n partials by one whole warp: lane-strided sums, then a
// butterfly, so every lane returns the same value.
__device__ __forceinline__ double
lb_warp_sum (const double* part, int n)
{
    double s = 0.0;
    for (int k = threadIdx.x & 31; k < n; k += 32) s += part[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync (0xffffffffu, s, o);
    return s;
}
#endif

// The graph-resident optimiser's state (device memory).  The host writes
// it before the launch (parameters, the prologue's evaluation and first
// step) and reads the outcome after.
struct LbDev {
    // parameters (b200bsp_lbfgs_parms)
    int m, max_its, max_feval, max_linesearch;
    double epsilon, min_step, max_step, ftol, gtol, xtol;
    // progress: iteration k, the history's next slot `end`, the slot of the
    // newest pair and the pairs in use; evaluations so far
    int k, end, newest, bound, fevals;
    int first;        // no correction pair yet (the first line search)
    int newiter;      // the next graph iteration starts a line search
    int done, status;
    int iterations;   // line searches completed (b200bsp_lbfgs_result)
    double f, finit, stp, dginit, dgtest;
    float total;      // the evaluation's total score (the finish kernel's)
    float last;       // the last evaluation's total
    // line search (Moré-Thuente)
    int brackt, stage1, uinfo, count;
    double stx, fx, dgx, sty, fy, dgy, stmin, stmax, width, prev_width;
    // dot products of the evaluated point: g.d, x.x, g.g
    double dg, xx, gg;
};

}  // namespace b200
