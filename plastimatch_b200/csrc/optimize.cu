// Limited-memory BFGS on the device: the optimiser Plastimatch runs around
// the cost function with implementation "liblbfgs"
// (src/register/bspline_optimize_liblbfgs.cxx:20-117, library
// libs/liblbfgs-1.9, default parameters), restated from the published
// methods rather than from that library's code:
//   direction   the two-loop recursion of Nocedal (1980) / Liu & Nocedal
//               (1989) over the last m (s, y) pairs, scaled by y's/y'y
//   line search Moré & Thuente (1994): strong Wolfe conditions, the
//               safeguarded trial-interval update of MINPACK's cstep
//               (cubic/quadratic/secant steps, four cases), the modified
//               function in the first stage and bisection when the
//               interval does not shrink by 2/3
//   stopping    ||g|| / max(1, ||x||) <= epsilon, a line-search failure, or
//               Plastimatch's progress rule (see stop_rule), checked after
//               every evaluation of a line search and after each one;
//               stopping inside a line search returns to the last accepted
//               point
// All vectors (x, g, d, history) live in device memory in double precision
// (liblbfgs' lbfgsfloatval_t); dot products are reduced in a fixed order
// and only scalars (dots, the score) come back to the host, where the
// line-search logic runs.
#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/plastimatch_b200.h"
#include "kernels.cuh"

namespace b200 {

int static_fail (int code, const char* msg);   // runtime.cu
cudaStream_t ctx_stream (const b200bsp_ctx* c); // runtime.cu
void* ctx_opt_ws (const b200bsp_ctx* c);
int ctx_landmarks (const b200bsp_ctx* c, float* stiffness);
void ctx_set_opt_ws (b200bsp_ctx* c, void* ws, void (*release) (void*));

constexpr int OPT_THREADS = 256;
constexpr int OPT_BLOCKS = 296;

__global__ void __launch_bounds__ (OPT_THREADS)
dot_partial_kernel (const double* __restrict__ a, const double* __restrict__ b,
    long long n, double* __restrict__ part)
{
    __shared__ double sh[OPT_THREADS];
    double s = 0.0;
    for (long long i = (long long) blockIdx.x * OPT_THREADS + threadIdx.x;
         i < n; i += (long long) gridDim.x * OPT_THREADS) {
        s += a[i] * b[i];
    }
    sh[threadIdx.x] = s;
    __syncthreads ();
    for (int o = OPT_THREADS / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads ();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void
dot_final_kernel (const double* __restrict__ part, int n, double* out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < n; i++) s += part[i];
        *out = s;
    }
}

// *out = sum of part (dot_final_kernel's order), divided by *den if given
__global__ void
dot_final_div_kernel (const double* __restrict__ part, int n,
    const double* __restrict__ den, double* out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < n; i++) s += part[i];
        *out = den ? s / *den : s;
    }
}

// y = (sign * *a) * x + b * y, the coefficient read on the device
__global__ void
axpby_dev_kernel (const double* __restrict__ a, double sign,
    const double* __restrict__ x, double b, double* __restrict__ y,
    long long n)
{
    const double av = sign * *a;
    for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x) {
        y[i] = av * x[i] + b * y[i];
    }
}

// y = (*a - *c) * x + 1 * y
__global__ void
axpy_diff_kernel (const double* __restrict__ a, const double* __restrict__ c,
    const double* __restrict__ x, double* __restrict__ y, long long n)
{
    const double av = *a - *c;
    for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x) {
        y[i] = av * x[i] + 1.0 * y[i];
    }
}

// y = 0 * y + (*num / *den) * y
__global__ void
scale_ratio_kernel (const double* __restrict__ num,
    const double* __restrict__ den, double* __restrict__ y, long long n)
{
    const double bv = *num / *den;
    for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x) {
        y[i] = 0.0 * y[i] + bv * y[i];
    }
}

// y = a * x + b * y
__global__ void
axpby_kernel (double a, const double* __restrict__ x, double b,
    double* __restrict__ y, long long n)
{
    for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x) {
        y[i] = a * x[i] + b * y[i];
    }
}

// z = x + a * y
__global__ void
xpay_kernel (const double* __restrict__ x, double a,
    const double* __restrict__ y, double* __restrict__ z, long long n)
{
    for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x) {
        z[i] = x[i] + a * y[i];
    }
}

__global__ void
sub_kernel (const double* __restrict__ a, const double* __restrict__ b,
    double* __restrict__ out, long long n)
{
    for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x) {
        out[i] = a[i] - b[i];
    }
}

__global__ void
to_float_kernel (const double* __restrict__ a, float* __restrict__ out,
    long long n)
{
    for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x) {
        out[i] = (float) a[i];
    }
}

__global__ void
to_double_kernel (const float* __restrict__ a, double* __restrict__ out,
    long long n)
{
    for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x) {
        out[i] = (double) a[i];
    }
}

__global__ void
scale_float_kernel (float* __restrict__ a, float s, long long n)
{
    for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x) {
        a[i] = 0.f + s * a[i];
    }
}

// Device workspace of one run.
struct Lbfgs {
    long long n = 0;
    int m = 0;
    double *x = nullptr, *g = nullptr, *d = nullptr, *xp = nullptr,
        *gp = nullptr, *s = nullptr, *y = nullptr, *part = nullptr,
        *scalar = nullptr;
    // device scalars of the two-loop recursion: ys[m], alpha[m], beta, yy
    double* dsc = nullptr;
    double* h_scalar = nullptr;
    cudaStream_t st = nullptr;
    int err = 0;

    int alloc (long long n_, int m_)
    {
        n = n_;
        m = m_;
        auto a = [&](double** p, size_t cnt) {
            if (!err && cudaMalloc (p, cnt * sizeof (double)) != cudaSuccess) {
                cudaGetLastError ();
                err = B200BSP_E_OOM;
            }
        };
        a (&x, n); a (&g, n); a (&d, n); a (&xp, n); a (&gp, n);
        a (&s, (size_t) m * n); a (&y, (size_t) m * n);
        a (&part, OPT_BLOCKS); a (&scalar, 2); a (&dsc, 2 * (size_t) m + 2);
        if (!err && cudaMallocHost (&h_scalar, 2 * sizeof (double)) != cudaSuccess) {
            cudaGetLastError ();
            err = B200BSP_E_OOM;
        }
        return err;
    }
    ~Lbfgs ()
    {
        cudaFree (x); cudaFree (g); cudaFree (d); cudaFree (xp); cudaFree (gp);
        cudaFree (s); cudaFree (y); cudaFree (part); cudaFree (scalar);
        cudaFree (dsc);
        cudaFreeHost (h_scalar);
    }
    unsigned grid () const
    {
        return (unsigned) std::min<long long> ((n + 255) / 256, 148 * 8);
    }
    // dot product into a device scalar (*den divides it when given); no
    // synchronisation
    void dot_dev (const double* a, const double* b, double* out,
        const double* den = nullptr)
    {
        dot_partial_kernel<<<OPT_BLOCKS, OPT_THREADS, 0, st>>> (a, b, n, part);
        dot_final_div_kernel<<<1, 32, 0, st>>> (part, OPT_BLOCKS, den, out);
    }
    // |a|^2 and |b|^2 with one synchronisation
    void norms2 (const double* a, const double* b, double* na, double* nb)
    {
        dot_dev (a, a, scalar);
        dot_dev (b, b, scalar + 1);
        if (cudaMemcpyAsync (h_scalar, scalar, 2 * sizeof (double),
                cudaMemcpyDeviceToHost, st) != cudaSuccess
            || cudaStreamSynchronize (st) != cudaSuccess) {
            cudaGetLastError ();
            err = B200BSP_E_CUDA;
            *na = *nb = 0.0;
            return;
        }
        *na = h_scalar[0];
        *nb = h_scalar[1];
    }
    double dot (const double* a, const double* b)
    {
        dot_partial_kernel<<<OPT_BLOCKS, OPT_THREADS, 0, st>>> (a, b, n, part);
        dot_final_kernel<<<1, 32, 0, st>>> (part, OPT_BLOCKS, scalar);
        if (cudaMemcpyAsync (h_scalar, scalar, sizeof (double),
                cudaMemcpyDeviceToHost, st) != cudaSuccess
            || cudaStreamSynchronize (st) != cudaSuccess) {
            cudaGetLastError ();
            err = B200BSP_E_CUDA;
            return 0.0;
        }
        return *h_scalar;
    }
    void axpby (double a, const double* xv, double b, double* yv)
    {
        axpby_kernel<<<grid (), 256, 0, st>>> (a, xv, b, yv, n);
    }
    void xpay (const double* xv, double a, const double* yv, double* z)
    {
        xpay_kernel<<<grid (), 256, 0, st>>> (xv, a, yv, z, n);
    }
    void copy (double* dst, const double* src)
    {
        if (cudaMemcpyAsync (dst, src, n * sizeof (double),
                cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
            cudaGetLastError ();
            err = B200BSP_E_CUDA;
        }
    }
    double* sv (int j) { return s + (size_t) j * n; }
    double* yv (int j) { return y + (size_t) j * n; }
};

// The objective: f(x) with its gradient written to the device vector g.
struct Objective {
    virtual ~Objective () {}
    // returns a status code; f receives the value
    virtual int eval (const double* x, double* g, double* f) = 0;
    int fevals = 0;
};

// Moré-Thuente trial-interval update (the cstep of MINPACK): x = best
// step so far (fx, dx), y = other end of the interval (fy, dy), t = trial
// step (ft, dt).  Returns 0, or an error code when the inputs are
// inconsistent (rounding errors).
static int
update_interval (double* x, double* fx, double* dx, double* y, double* fy,
    double* dy, double* t, double ft, double dt, double tmin, double tmax,
    int* brackt)
{
    if (*brackt) {
        if (*t <= std::min (*x, *y) || std::max (*x, *y) <= *t) return 1;
        if (0.0 <= *dx * (*t - *x)) return 2;
        if (tmax < tmin) return 3;
    }
    // the derivatives differ in sign (dt * sign(dx) < 0)
    const bool dsign = dt * (*dx / std::fabs (*dx)) < 0.0;
    bool bound;
    double newt;
    // Minimiser of the cubic interpolating (u, fu, du) and (v, fv, dv),
    // written from u's side: returns r with minimiser u + r (v - u), and
    // gamma (zero when the cubic has no minimiser there and clamp_zero).
    auto cubic = [](double u, double fu, double du, double v, double fv,
                     double dv, bool clamp_zero, double* gamma_out) {
        const double theta = 3.0 * (fu - fv) / (v - u) + du + dv;
        const double s = std::max (std::fabs (theta),
            std::max (std::fabs (du), std::fabs (dv)));
        const double a = theta / s;
        double gamma2 = a * a - (du / s) * (dv / s);
        if (clamp_zero && gamma2 < 0) gamma2 = 0;
        double gamma = s * std::sqrt (gamma2);
        if (v < u) gamma = -gamma;
        const double p = (gamma - du) + theta;
        const double q = ((gamma - du) + gamma) + dv;
        if (gamma_out) *gamma_out = gamma;
        return p / q;
    };
    if (*fx < ft) {
        // case 1: higher function value; the minimum is bracketed
        *brackt = 1;
        bound = true;
        const double mc = *x + cubic (*x, *fx, *dx, *t, ft, dt, false,
            nullptr) * (*t - *x);
        const double mq = *x + (*dx / ((*fx - ft) / (*t - *x) + *dx)) / 2.0
            * (*t - *x);
        if (std::fabs (mc - *x) < std::fabs (mq - *x)) newt = mc;
        else newt = mc + 0.5 * (mq - mc);
    } else if (dsign) {
        // case 2: lower value, derivatives of opposite sign; bracketed
        *brackt = 1;
        bound = false;
        const double mc = *t + cubic (*t, ft, dt, *x, *fx, *dx, false,
            nullptr) * (*x - *t);
        const double mq = *t + (dt / (dt - *dx)) * (*x - *t);
        if (std::fabs (mc - *t) > std::fabs (mq - *t)) newt = mc;
        else newt = mq;
    } else if (std::fabs (dt) < std::fabs (*dx)) {
        // case 3: lower value, same sign, smaller derivative magnitude
        bound = true;
        double gamma;
        const double r = cubic (*t, ft, dt, *x, *fx, *dx, true, &gamma);
        double mc;
        // the cubic may have no minimiser beyond t
        if (r < 0.0 && gamma != 0.0) mc = *t + r * (*x - *t);
        else if (*x < *t) mc = tmax;
        else mc = tmin;
        const double mq = *t + (dt / (dt - *dx)) * (*x - *t);
        if (*brackt) {
            newt = std::fabs (*t - mc) < std::fabs (*t - mq) ? mc : mq;
        } else {
            newt = std::fabs (*t - mc) > std::fabs (*t - mq) ? mc : mq;
        }
    } else {
        // case 4: lower value, same sign, derivative does not decrease
        bound = false;
        if (*brackt) {
            newt = *t + cubic (*t, ft, dt, *y, *fy, *dy, false, nullptr)
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
    newt = std::min (tmax, newt);
    newt = std::max (tmin, newt);
    if (*brackt && bound) {
        const double mq = *x + 0.66 * (*y - *x);
        if (*x < *y) newt = std::min (mq, newt);
        else newt = std::max (mq, newt);
    }
    *t = newt;
    return 0;
}

enum {
    LS_ROUNDING = -1001, LS_MAXSTEP = -1002, LS_MINSTEP = -1003,
    LS_WIDTH = -1004, LS_MAXLS = -1005, LS_INCREASE = -1006, LS_BADSTEP = -1007,
    LS_STOPPED = -1100      // the progress rule stopped the run mid-search
};

// Plastimatch's progress rule (src/register/bspline_optimize_liblbfgs.cxx:
// 53-79): stop once the iteration number exceeds max_its or the function
// evaluations exceed max_feval.  The liblbfgs it links consults the rule
// after every evaluation inside a line search (with the current iteration
// number) and once more after each completed line search.
static bool
stop_rule (const b200bsp_lbfgs_parms& p, int k, int fevals)
{
    return k > p.max_its || fevals > p.max_feval;
}

// Moré-Thuente line search from xp along d; on return x, f, g are the last
// trial.  Returns the evaluation count (> 0) on success, a negative code
// on failure (LS_* or a library status).
static int
line_search (Lbfgs& w, Objective& obj, const b200bsp_lbfgs_parms& p,
    double* f, double* stp, double finit, int k)
{
    if (*stp <= 0.0) return LS_BADSTEP;
    const double dginit = w.dot (w.gp, w.d);
    if (w.err) return w.err;
    if (0.0 < dginit) return LS_INCREASE;
    int brackt = 0, stage1 = 1, uinfo = 0, count = 0;
    const double dgtest = p.ftol * dginit;
    double width = p.max_step - p.min_step;
    double prev_width = 2.0 * width;
    double stx = 0.0, fx = finit, dgx = dginit;
    double sty = 0.0, fy = finit, dgy = dginit;
    double stmin, stmax;
    while (true) {
        if (brackt) {
            stmin = std::min (stx, sty);
            stmax = std::max (stx, sty);
        } else {
            stmin = stx;
            stmax = *stp + 4.0 * (*stp - stx);
        }
        *stp = std::max (p.min_step, std::min (p.max_step, *stp));
        if ((brackt && ((*stp <= stmin || stmax <= *stp)
                 || p.max_linesearch <= count + 1 || uinfo != 0))
            || (brackt && (stmax - stmin <= p.xtol * stmax))) {
            *stp = stx;
        }
        w.xpay (w.xp, *stp, w.d, w.x);
        int rc = obj.eval (w.x, w.g, f);
        if (rc) return rc;
        if (stop_rule (p, k, obj.fevals)) return LS_STOPPED;
        const double dg = w.dot (w.g, w.d);
        if (w.err) return w.err;
        const double ftest1 = finit + *stp * dgtest;
        ++count;
        if (brackt && ((*stp <= stmin || stmax <= *stp) || uinfo != 0)) {
            return LS_ROUNDING;
        }
        if (*stp == p.max_step && *f <= ftest1 && dg <= dgtest) return LS_MAXSTEP;
        if (*stp == p.min_step && (ftest1 < *f || dgtest <= dg)) return LS_MINSTEP;
        if (brackt && (stmax - stmin) <= p.xtol * stmax) return LS_WIDTH;
        if (p.max_linesearch <= count) return LS_MAXLS;
        if (*f <= ftest1 && std::fabs (dg) <= p.gtol * (-dginit)) return count;
        if (stage1 && *f <= ftest1 && std::min (p.ftol, p.gtol) * dginit <= dg) {
            stage1 = 0;
        }
        if (stage1 && ftest1 < *f && *f <= fx) {
            // first stage: work on the modified function f - stp * dgtest
            double fm = *f - *stp * dgtest;
            double fxm = fx - stx * dgtest, fym = fy - sty * dgtest;
            double dgm = dg - dgtest;
            double dgxm = dgx - dgtest, dgym = dgy - dgtest;
            uinfo = update_interval (&stx, &fxm, &dgxm, &sty, &fym, &dgym, stp,
                fm, dgm, stmin, stmax, &brackt);
            fx = fxm + stx * dgtest;
            fy = fym + sty * dgtest;
            dgx = dgxm + dgtest;
            dgy = dgym + dgtest;
        } else {
            uinfo = update_interval (&stx, &fx, &dgx, &sty, &fy, &dgy, stp, *f,
                dg, stmin, stmax, &brackt);
        }
        if (brackt) {
            if (0.66 * prev_width <= std::fabs (sty - stx)) {
                *stp = stx + 0.5 * (sty - stx);
            }
            prev_width = width;
            width = std::fabs (sty - stx);
        }
    }
}

static int
lbfgs_run (Lbfgs& w, Objective& obj, const b200bsp_lbfgs_parms& p,
    b200bsp_lbfgs_result* res)
{
    const int m = p.m;
    double f = 0.0;
    int rc = obj.eval (w.x, w.g, &f);
    if (rc) return rc;
    res->score = f;
    res->iterations = 0;
    double xnorm, gnorm;
    w.norms2 (w.x, w.g, &xnorm, &gnorm);
    xnorm = std::sqrt (xnorm);
    gnorm = std::sqrt (gnorm);
    if (w.err) return w.err;
    if (xnorm < 1.0) xnorm = 1.0;
    if (gnorm / xnorm <= p.epsilon) {
        res->status = B200BSP_LBFGS_ALREADY_MINIMIZED;
        return B200BSP_OK;
    }
    w.axpby (-1.0, w.g, 0.0, w.d);                // d = -g
    double step = 1.0 / std::sqrt (w.dot (w.d, w.d));
    int k = 1, end = 0;
    while (true) {
        w.copy (w.xp, w.x);
        w.copy (w.gp, w.g);
        const double finit = f;
        int ls = line_search (w, obj, p, &f, &step, finit, k);
        if (ls < 0) {
            // return to the last accepted point
            w.copy (w.x, w.xp);
            w.copy (w.g, w.gp);
            f = finit;
            res->score = f;
            res->status = ls == LS_STOPPED ? B200BSP_LBFGS_STOPPED : ls;
            return w.err ? w.err : B200BSP_OK;
        }
        res->score = f;
        res->iterations = k;
        w.norms2 (w.x, w.g, &xnorm, &gnorm);
        xnorm = std::sqrt (xnorm);
        gnorm = std::sqrt (gnorm);
        if (w.err) return w.err;
        if (stop_rule (p, k, obj.fevals)) {
            res->status = B200BSP_LBFGS_STOPPED;
            return B200BSP_OK;
        }
        if (xnorm < 1.0) xnorm = 1.0;
        if (gnorm / xnorm <= p.epsilon) {
            res->status = B200BSP_LBFGS_CONVERGED;
            return B200BSP_OK;
        }
        // new correction pair; the two-loop recursion runs on the device
        // with its scalars in device memory (no synchronisation until the
        // next line search)
        double* ys_d = w.dsc;                 // [m]
        double* alpha_d = w.dsc + m;          // [m]
        double* beta_d = w.dsc + 2 * m;
        double* yy_d = w.dsc + 2 * m + 1;
        sub_kernel<<<w.grid (), 256, 0, w.st>>> (w.x, w.xp, w.sv (end), w.n);
        sub_kernel<<<w.grid (), 256, 0, w.st>>> (w.g, w.gp, w.yv (end), w.n);
        w.dot_dev (w.yv (end), w.sv (end), ys_d + end);
        w.dot_dev (w.yv (end), w.yv (end), yy_d);
        const int newest = end;
        const int bound = std::min (m, k);
        ++k;
        end = (end + 1) % m;
        w.axpby (-1.0, w.g, 0.0, w.d);
        int j = end;
        for (int i = 0; i < bound; i++) {
            j = (j + m - 1) % m;
            w.dot_dev (w.sv (j), w.d, alpha_d + j, ys_d + j);
            axpby_dev_kernel<<<w.grid (), 256, 0, w.st>>> (alpha_d + j, -1.0,
                w.yv (j), 1.0, w.d, w.n);
        }
        scale_ratio_kernel<<<w.grid (), 256, 0, w.st>>> (ys_d + newest, yy_d,
            w.d, w.n);
        for (int i = 0; i < bound; i++) {
            w.dot_dev (w.yv (j), w.d, beta_d, ys_d + j);
            axpy_diff_kernel<<<w.grid (), 256, 0, w.st>>> (alpha_d + j, beta_d,
                w.sv (j), w.d, w.n);
            j = (j + 1) % m;
        }
        if (cudaGetLastError () != cudaSuccess) return B200BSP_E_CUDA;
        if (w.err) return w.err;
        step = 1.0;
    }
}

// ---- objectives -----------------------------------------------------------

// bspline_score() on the context: lambda * metric (+ regulariser, +
// landmarks when the context has them), values and gradients in float as
// the reference's Bspline_score holds them.
struct ContextObjective : Objective {
    b200bsp_ctx* ctx;
    int metric;
    float lambda;
    const b200bsp_reg_parms* reg;
    float* coeff_f;
    float* grad_f;
    long long n;
    cudaStream_t st;
    // batched evaluation (a registration of a batch): the score and the
    // gradient come from the batch's graph launch instead
    void* member = nullptr;
    int (*batch_eval) (void*, int, const float*, float*, float*) = nullptr;
    int eval (const double* x, double* g, double* f) override
    {
        const unsigned grid = (unsigned) std::min<long long> ((n + 255) / 256,
            148 * 8);
        to_float_kernel<<<grid, 256, 0, st>>> (x, coeff_f, n);
        float s = 0.f;
        int64_t nv = 0;
        int rc;
        if (batch_eval) {
            rc = cudaStreamSynchronize (st) == cudaSuccess
                ? batch_eval (member, 0, coeff_f, grad_f, &s) : B200BSP_E_CUDA;
        } else {
            rc = metric == 0
                ? b200bsp_score_mse (ctx, coeff_f, &s, grad_f, &nv)
                : b200bsp_score_mi (ctx, coeff_f, &s, grad_f, &nv, nullptr,
                    nullptr, nullptr);
        }
        if (rc) return rc;
        // Bspline_score::accumulate: total = lambda * smetric, total_grad =
        // lambda * smetric_grad (src/register/bspline_score.cxx:63-74)
        float total = 0.f;
        total += lambda * s;
        scale_float_kernel<<<grid, 256, 0, st>>> (grad_f, lambda, n);
        if (reg) {
            float r = 0.f;
            rc = b200bsp_regularize (ctx, coeff_f, reg, &r, grad_f);
            if (rc) return rc;
            total += r;
        }
        float stiffness = 0.f;
        if (ctx_landmarks (ctx, &stiffness) > 0) {
            // src/register/bspline.cxx:624-628
            float lm = 0.f;
            rc = b200bsp_landmarks_score (ctx, coeff_f, &lm, grad_f);
            if (rc) return rc;
            total += stiffness * lm;
        }
        to_double_kernel<<<grid, 256, 0, st>>> (grad_f, g, n);
        if (cudaGetLastError () != cudaSuccess) return B200BSP_E_CUDA;
        *f = (double) total;
        last = total;
        fevals++;
        return B200BSP_OK;
    }
    float last = 0.f;     // score of the last evaluation
};

// A caller's function on host copies of x and g.
struct HostObjective : Objective {
    b200bsp_eval_fn fn;
    void* user;
    long long n;
    cudaStream_t st;
    std::vector<double> hx, hg;
    int eval (const double* x, double* g, double* f) override
    {
        hx.resize (n);
        hg.resize (n);
        if (cudaMemcpyAsync (hx.data (), x, n * sizeof (double),
                cudaMemcpyDeviceToHost, st) != cudaSuccess
            || cudaStreamSynchronize (st) != cudaSuccess) {
            cudaGetLastError ();
            return B200BSP_E_CUDA;
        }
        *f = fn (user, hx.data (), hg.data (), n);
        if (cudaMemcpyAsync (g, hg.data (), n * sizeof (double),
                cudaMemcpyHostToDevice, st) != cudaSuccess
            || cudaStreamSynchronize (st) != cudaSuccess) {
            cudaGetLastError ();
            return B200BSP_E_CUDA;
        }
        fevals++;
        return B200BSP_OK;
    }
};

static int
check_parms (const b200bsp_lbfgs_parms* p)
{
    if (p->m < 1 || p->m > 64 || !(p->epsilon >= 0) || p->max_linesearch < 1
        || !(p->min_step > 0) || !(p->max_step > p->min_step)
        || !(p->ftol > 0 && p->ftol < 0.5) || !(p->gtol > p->ftol && p->gtol < 1)
        || !(p->xtol >= 0)) {
        return static_fail (B200BSP_E_BADARG, "bad L-BFGS parameters");
    }
    return B200BSP_OK;
}

static bool
device_mem (const void* p)
{
    cudaPointerAttributes a;
    if (!p || cudaPointerGetAttributes (&a, p) != cudaSuccess) {
        cudaGetLastError ();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

__global__ void
f2d_kernel (const float* __restrict__ a, double* __restrict__ out, long long n)
{
    for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x) {
        out[i] = (double) a[i];
    }
}

// A context's optimiser workspace: the L-BFGS vectors and the float
// coefficient / gradient buffers, allocated on the first run and kept by
// the context (reallocated only when the history length changes), so a
// registration allocates nothing after its first run.
struct OptWorkspace {
    Lbfgs w;
    float* buf = nullptr;
    ~OptWorkspace () { cudaFree (buf); }
};

static void
release_ws (void* p)
{
    delete (OptWorkspace*) p;
}

static OptWorkspace*
context_workspace (b200bsp_ctx* ctx, int64_t nc, int m)
{
    auto* ws = (OptWorkspace*) ctx_opt_ws (ctx);
    if (ws && ws->w.n == nc && ws->w.m == m) return ws;
    ws = new OptWorkspace ();
    if (ws->w.alloc (nc, m)
        || cudaMalloc (&ws->buf, 2 * nc * sizeof (float)) != cudaSuccess) {
        cudaGetLastError ();
        delete ws;
        return nullptr;
    }
    ctx_set_opt_ws (ctx, ws, release_ws);
    return ws;
}

// L-BFGS over a context's coefficients (host or device floats, updated in
// place with the last evaluated point), evaluations by `obj`.
static int
optimize_on_context (b200bsp_ctx* ctx, const b200bsp_lbfgs_parms& p,
    int64_t nc, float* coeff, b200bsp_lbfgs_result* res,
    ContextObjective& obj)
{
    int rc = B200BSP_OK;
    OptWorkspace* ws = context_workspace (ctx, nc, p.m);
    if (!ws) return static_fail (B200BSP_E_OOM, "optimiser buffers");
    Lbfgs& w = ws->w;
    w.err = 0;
    float* buf = ws->buf;
    obj.coeff_f = buf; obj.grad_f = buf + nc; obj.n = nc;
    // the context's stream orders every kernel of the run
    cudaStream_t st = ctx_stream (ctx);
    w.st = st;
    obj.st = st;
    const bool dev = device_mem (coeff);
    if (cudaMemcpyAsync (buf, coeff, nc * sizeof (float),
            dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st)
        != cudaSuccess) {
        cudaGetLastError ();
        return static_fail (B200BSP_E_CUDA, "coefficient upload");
    }
    f2d_kernel<<<w.grid (), 256, 0, st>>> (buf, w.x, nc);
    res->status = 0;
    res->fevals = 0;
    rc = lbfgs_run (w, obj, p, res);
    res->fevals = obj.fevals;
    if (!rc) {
        // Plastimatch's evaluate callback copies every trial point into the
        // transform, so the registration ends with the last evaluated
        // coefficients and score (bspline_optimize_liblbfgs.cxx:20-51); the
        // buffer already holds them.
        res->score = obj.last;
        if (cudaMemcpyAsync (coeff, buf, nc * sizeof (float),
                dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st)
                != cudaSuccess
            || cudaStreamSynchronize (st) != cudaSuccess) {
            cudaGetLastError ();
            rc = static_fail (B200BSP_E_CUDA, "coefficient download");
        }
    }
    return rc;
}

// One registration of a batch (batch.cu): MSE, no regulariser, each
// evaluation through `eval` (the batch's barrier and graph launch).
int
lbfgs_optimize_batched (b200bsp_ctx* ctx, float lambda,
    const b200bsp_lbfgs_parms* parms, float* coeff, b200bsp_lbfgs_result* res,
    void* member, int (*eval) (void*, int, const float*, float*, float*))
{
    b200bsp_lbfgs_parms p;
    if (parms) p = *parms; else b200bsp_lbfgs_default_parms (&p);
    int rc = check_parms (&p);
    if (rc) return rc;
    int64_t nc = 0;
    rc = b200bsp_grid_info (ctx, nullptr, nullptr, &nc);
    if (rc) return rc;
    ContextObjective obj;
    obj.ctx = ctx; obj.metric = 0; obj.lambda = lambda; obj.reg = nullptr;
    obj.member = member;
    obj.batch_eval = eval;
    return optimize_on_context (ctx, p, nc, coeff, res, obj);
}

} // namespace b200

using namespace b200;

extern "C" void
b200bsp_lbfgs_default_parms (b200bsp_lbfgs_parms* p)
{
    p->m = 6;
    p->epsilon = 1e-5;
    p->max_its = 10;            // Bspline_parms defaults (bspline_parms.cxx:16-17)
    p->max_feval = 10;
    p->max_linesearch = 40;
    p->min_step = 1e-20;
    p->max_step = 1e20;
    p->ftol = 1e-4;
    p->gtol = 0.9;
    p->xtol = 1e-16;
}

extern "C" int
b200bsp_optimize_lbfgs (b200bsp_ctx* ctx, int metric_type, float lambda,
    const b200bsp_reg_parms* reg, const b200bsp_lbfgs_parms* parms,
    float* coeff, b200bsp_lbfgs_result* res)
{
    if (!ctx || !coeff || !res) return static_fail (B200BSP_E_BADARG, "null argument");
    b200bsp_lbfgs_parms p;
    if (parms) p = *parms; else b200bsp_lbfgs_default_parms (&p);
    int rc = check_parms (&p);
    if (rc) return rc;
    int64_t nc = 0;
    rc = b200bsp_grid_info (ctx, nullptr, nullptr, &nc);
    if (rc) return rc;
    ContextObjective obj;
    obj.ctx = ctx; obj.metric = metric_type; obj.lambda = lambda; obj.reg = reg;
    return optimize_on_context (ctx, p, nc, coeff, res, obj);
}

extern "C" int
b200bsp_lbfgs_minimize (int64_t n, double* x, b200bsp_eval_fn fn, void* user,
    const b200bsp_lbfgs_parms* parms, b200bsp_lbfgs_result* res, int device)
{
    if (n < 1 || !x || !fn || !res) return static_fail (B200BSP_E_BADARG, "bad argument");
    b200bsp_lbfgs_parms p;
    if (parms) p = *parms; else b200bsp_lbfgs_default_parms (&p);
    int rc = check_parms (&p);
    if (rc) return rc;
    if (cudaSetDevice (device) != cudaSuccess) {
        cudaGetLastError ();
        return static_fail (B200BSP_E_CUDA, "no such device");
    }
    Lbfgs w;
    if (w.alloc (n, p.m)) return static_fail (B200BSP_E_OOM, "optimiser buffers");
    HostObjective obj;
    obj.fn = fn; obj.user = user; obj.n = n; obj.st = nullptr;
    if (cudaMemcpy (w.x, x, n * sizeof (double), cudaMemcpyHostToDevice)
        != cudaSuccess) {
        cudaGetLastError ();
        return static_fail (B200BSP_E_CUDA, "upload");
    }
    res->status = 0;
    rc = lbfgs_run (w, obj, p, res);
    res->fevals = obj.fevals;
    if (!rc && cudaMemcpy (x, w.x, n * sizeof (double), cudaMemcpyDeviceToHost)
        != cudaSuccess) {
        cudaGetLastError ();
        rc = static_fail (B200BSP_E_CUDA, "download");
    }
    return rc;
}
