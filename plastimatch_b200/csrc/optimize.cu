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
#include <cstring>
#include <vector>

#include "../../include/plastimatch_b200.h"
#include "kernels.cuh"
#include "lbfgs_graph.cuh"
#include "lbfgs_logic.cuh"

namespace b200 {

int static_fail (int code, const char* msg);   // runtime.cu
cudaStream_t ctx_stream (const b200bsp_ctx* c); // runtime.cu
void* ctx_opt_ws (const b200bsp_ctx* c);
int ctx_landmarks (const b200bsp_ctx* c, float* stiffness);
void ctx_set_opt_ws (b200bsp_ctx* c, void* ws, void (*release) (void*));
unsigned ctx_generation (const b200bsp_ctx* c);                // runtime.cu
int* ctx_err_flag (b200bsp_ctx* c);
int ctx_report_device_error (b200bsp_ctx* c, int e);

constexpr int OPT_THREADS = 256;
constexpr int OPT_BLOCKS = 296;

// one block's partial sum of a . b (blocks stride the vector)
__device__ __forceinline__ void
dot_partial_body (const double* __restrict__ a, const double* __restrict__ b,
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

__global__ void __launch_bounds__ (OPT_THREADS)
dot_partial_kernel (const double* __restrict__ a, const double* __restrict__ b,
    long long n, double* __restrict__ part)
{
    dot_partial_body (a, b, n, part);
}

// *out = the sum of the block partials (one warp, lb_warp_sum's order: the
// partials' loads all go out at once)
__global__ void
dot_final_kernel (const double* __restrict__ part, int n, double* out)
{
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    const double s = lb_warp_sum (part, n);
    if (threadIdx.x == 0) *out = s;
}

// *out = the sum of part (dot_final_kernel's order), divided by *den if
// given
__global__ void
dot_final_div_kernel (const double* __restrict__ part, int n,
    const double* __restrict__ den, double* out)
{
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    const double s = lb_warp_sum (part, n);
    if (threadIdx.x == 0) *out = den ? s / *den : s;
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
        // partial sums: one slot for the host-driven loop's dot products,
        // LP_REC + 2 m slots for the graph-resident run's
        a (&part, (size_t) OPT_BLOCKS * (LP_REC + 2 * m));
        a (&scalar, 2); a (&dsc, 2 * (size_t) m + 2);
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

static int
update_interval (double* x, double* fx, double* dx, double* y, double* fy,
    double* dy, double* t, double ft, double dt, double tmin, double tmax,
    int* brackt)
{
    return lb_update_interval (x, fx, dx, y, fy, dy, t, ft, dt, tmin, tmax,
        brackt);
}

static bool
stop_rule (const b200bsp_lbfgs_parms& p, int k, int fevals)
{
    return lb_stop_rule (p.max_its, p.max_feval, k, fevals);
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

// The start of a run: the objective at x0, the gradient test, d = -g and
// the first step 1/|d|.  Returns a status; *more is false when the run is
// already over (res holds its outcome).
static int
lbfgs_prologue (Lbfgs& w, Objective& obj, const b200bsp_lbfgs_parms& p,
    b200bsp_lbfgs_result* res, double* f, double* step, bool* more)
{
    *more = false;
    int rc = obj.eval (w.x, w.g, f);
    if (rc) return rc;
    res->score = *f;
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
    *step = 1.0 / std::sqrt (w.dot (w.d, w.d));
    if (w.err) return w.err;
    *more = true;
    return B200BSP_OK;
}

// The iterations after the prologue, driven from the host.
static int
lbfgs_loop (Lbfgs& w, Objective& obj, const b200bsp_lbfgs_parms& p,
    b200bsp_lbfgs_result* res, double f, double step)
{
    const int m = p.m;
    double xnorm, gnorm;
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

static int
lbfgs_run (Lbfgs& w, Objective& obj, const b200bsp_lbfgs_parms& p,
    b200bsp_lbfgs_result* res)
{
    double f = 0.0, step = 0.0;
    bool more = false;
    int rc = lbfgs_prologue (w, obj, p, res, &f, &step, &more);
    if (rc || !more) return rc;
    return lbfgs_loop (w, obj, p, res, f, step);
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
    int eval (const double* x, double* g, double* f) override
    {
        const unsigned grid = (unsigned) std::min<long long> ((n + 255) / 256,
            148 * 8);
        to_float_kernel<<<grid, 256, 0, st>>> (x, coeff_f, n);
        float s = 0.f;
        int64_t nv = 0;
        int rc;
        rc = metric == 0
            ? b200bsp_score_mse (ctx, coeff_f, &s, grad_f, &nv)
            : b200bsp_score_mi (ctx, coeff_f, &s, grad_f, &nv, nullptr,
                nullptr, nullptr);
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

// ---- the graph-resident run --------------------------------------------------
//
// For MSE or MI on a context (with or without the regulariser, no
// landmarks) the iterations after the prologue run as one CUDA graph: a
// while node over trial points whose body is [new line search?] -> x = xp +
// stp d -> evaluation (MSE: the context's MSE kernel and finish kernel, the
// regulariser beside them; MI: both passes, the regulariser, the combine
// kernel) -> g.d, x.x, g.g -> the controller (lbfgs_graph.cu).  The
// "new line search" branch (an if node) forms the correction pair, runs the
// two-loop recursion with its indices read on the device, copies xp, gp and
// takes dginit.  Only the outcome comes back to the host.

namespace {

__device__ __forceinline__ bool
lb_skip (const LbDev* s, int i)
{
    return s->first || i >= s->bound;
}

// the i-th pair of the first loop (newest first) and of the second
__device__ __forceinline__ int
lb_j1 (const LbDev* s, int i)
{
    return (s->end - 1 - i + 2 * s->m) % s->m;
}

__device__ __forceinline__ int
lb_j2 (const LbDev* s, int i)
{
    return (s->end - s->bound + i + 2 * s->m) % s->m;
}

// The whole new-line-search branch in one block, for vectors of at most
// LB_FUSED_MAX entries: correction pair, the two-loop recursion, xp = x,
// gp = g and dginit = gp.d, each dot product a block reduction in a fixed
// order (one launch instead of some fifty for small registrations).
constexpr long long LB_FUSED_MAX = 1 << 17;
constexpr int LB_FUSED_THREADS = 1024;

__device__ double
lb_block_dot (const double* __restrict__ a, const double* __restrict__ b,
    long long n, double* red)
{
    double s = 0.0;
    for (long long i = threadIdx.x; i < n; i += LB_FUSED_THREADS) s += a[i] * b[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync (0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads ();
    if (threadIdx.x < 32) {
        double v = red[threadIdx.x];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync (0xffffffffu, v, o);
        if (threadIdx.x == 0) red[32] = v;
    }
    __syncthreads ();
    const double r = red[32];
    __syncthreads ();
    return r;
}

__global__ void __launch_bounds__ (LB_FUSED_THREADS)
lb_branch_fused_kernel (const LbDev* __restrict__ st, double* __restrict__ S,
    double* __restrict__ Y, const double* __restrict__ x,
    double* __restrict__ xp, const double* __restrict__ g,
    double* __restrict__ gp, double* __restrict__ d,
    double* __restrict__ dsc, double* __restrict__ dginit, long long n)
{
    __shared__ double red[33];
    const int m = st->m;
    const bool first = st->first;
    const int t = threadIdx.x;
    if (!first) {
        double* sn = S + (size_t) st->newest * n;
        double* yn = Y + (size_t) st->newest * n;
        for (long long i = t; i < n; i += LB_FUSED_THREADS) {
            sn[i] = x[i] - xp[i];
            yn[i] = g[i] - gp[i];
        }
        __syncthreads ();
        const double ys = lb_block_dot (yn, sn, n, red);
        const double yy = lb_block_dot (yn, yn, n, red);
        if (t == 0) {
            dsc[st->newest] = ys;
            dsc[2 * m + 1] = yy;
        }
    }
    for (long long i = t; i < n; i += LB_FUSED_THREADS) d[i] = -1.0 * g[i] + 0.0 * d[i];
    __syncthreads ();
    if (!first) {
        const int bound = st->bound;
        int j = st->end;
        for (int k = 0; k < bound; k++) {
            j = (j + m - 1) % m;
            const double* sj = S + (size_t) j * n;
            const double* yj = Y + (size_t) j * n;
            const double alpha = lb_block_dot (sj, d, n, red) / dsc[j];
            if (t == 0) dsc[m + j] = alpha;
            for (long long i = t; i < n; i += LB_FUSED_THREADS) {
                d[i] = (-1.0 * alpha) * yj[i] + 1.0 * d[i];
            }
            __syncthreads ();
        }
        const double bv = dsc[st->newest] / dsc[2 * m + 1];
        for (long long i = t; i < n; i += LB_FUSED_THREADS) d[i] = 0.0 * d[i] + bv * d[i];
        __syncthreads ();
        for (int k = 0; k < bound; k++) {
            const double* sj = S + (size_t) j * n;
            const double* yj = Y + (size_t) j * n;
            const double beta = lb_block_dot (yj, d, n, red) / dsc[j];
            const double av = dsc[m + j] - beta;
            for (long long i = t; i < n; i += LB_FUSED_THREADS) {
                d[i] = av * sj[i] + 1.0 * d[i];
            }
            __syncthreads ();
            j = (j + 1) % m;
        }
    }
    for (long long i = t; i < n; i += LB_FUSED_THREADS) {
        xp[i] = x[i];
        gp[i] = g[i];
    }
    __syncthreads ();
    const double dg0 = lb_block_dot (gp, d, n, red);
    if (t == 0) *dginit = dg0;
}

// x = xp + stp d (the trial point) and its float copy, the evaluation's
// coefficients; both stay when the run is over (the float copy already
// holds x then)
__global__ void
lb_trial_kernel (const LbDev* __restrict__ st, const double* __restrict__ xp,
    const double* __restrict__ d, double* __restrict__ x,
    float* __restrict__ xf, long long n)
{
    if (st->done) return;
    const double a = st->stp;
    for (long long k = (long long) blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (long long) gridDim.x * blockDim.x) {
        const double v = xp[k] + a * d[k];
        x[k] = v;
        xf[k] = (float) v;
    }
}

// ---- the recursion and the evaluation's dot products, fused ----------------
//
// Each kernel below runs on OPT_BLOCKS blocks of OPT_THREADS threads and
// writes one block partial per dot product it forms (a thread sums its
// indices in the order of dot_partial_body, then the block's tree); the
// next kernel of the chain sums the partials it needs in every block (one
// warp, lb_warp_sum) instead of waiting for a separate reduction launch.
// Early returns depend on the run's state only, so whole blocks take them.

// the block's partials of K dot products into slots out[k]
template <int K>
__device__ __forceinline__ void
block_partials (const double (&v)[K], double* const (&out)[K])
{
    __shared__ double sh[K][OPT_THREADS];
#pragma unroll
    for (int k = 0; k < K; k++) sh[k][threadIdx.x] = v[k];
    __syncthreads ();
    for (int o = OPT_THREADS / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
#pragma unroll
            for (int k = 0; k < K; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + o];
        }
        __syncthreads ();
    }
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) out[k][blockIdx.x] = sh[k][0];
    }
}

// the sum of slot `slot`'s partials, in every thread of the block
__device__ __forceinline__ double
block_final (const double* __restrict__ part, int slot)
{
    __shared__ double r;
    if (threadIdx.x < 32) {
        const double v = lb_warp_sum (part + (size_t) slot * OPT_BLOCKS,
            OPT_BLOCKS);
        if (threadIdx.x == 0) r = v;
    }
    __syncthreads ();
    const double v = r;
    __syncthreads ();
    return v;
}

__device__ __forceinline__ double*
slot_of (double* part, int slot)
{
    return part + (size_t) slot * OPT_BLOCKS;
}

// After an evaluation: g = (double) grad, and the partials of g.d, x.x and
// g.g (slots LP_GD, LP_XX, LP_GG).
__global__ void __launch_bounds__ (OPT_THREADS)
lb_eval_dots_kernel (const float* __restrict__ grad, double* __restrict__ g,
    const double* __restrict__ d, const double* __restrict__ x, long long n,
    double* __restrict__ part)
{
    double gd = 0.0, xx = 0.0, gg = 0.0;
    for (long long i = (long long) blockIdx.x * OPT_THREADS + threadIdx.x;
         i < n; i += (long long) gridDim.x * OPT_THREADS) {
        const double gi = (double) grad[i];
        const double xi = x[i];
        g[i] = gi;
        gd += gi * d[i];
        xx += xi * xi;
        gg += gi * gi;
    }
    block_partials<3> ({gd, xx, gg}, {slot_of (part, LP_GD),
        slot_of (part, LP_XX), slot_of (part, LP_GG)});
}

// Start of the new-line-search branch: d = -g and, with a correction pair
// to form, s_new = x - xp, y_new = g - gp with the partials of y.s, y.y and
// the first loop's first s_j.d; without one (the first line search), xp =
// x, gp = g and the partials of gp.d.
__global__ void __launch_bounds__ (OPT_THREADS)
lb_rec_start_kernel (const LbDev* __restrict__ st, double* __restrict__ S,
    double* __restrict__ Y, const double* __restrict__ x,
    double* __restrict__ xp, const double* __restrict__ g,
    double* __restrict__ gp, double* __restrict__ d, long long n,
    double* __restrict__ part)
{
    const long long i0 = (long long) blockIdx.x * OPT_THREADS + threadIdx.x;
    const long long step = (long long) gridDim.x * OPT_THREADS;
    if (st->first) {
        double dg = 0.0;
        for (long long i = i0; i < n; i += step) {
            const double gi = g[i];
            const double di = -1.0 * gi + 0.0 * d[i];
            d[i] = di;
            xp[i] = x[i];
            gp[i] = gi;
            dg += gi * di;
        }
        block_partials<1> ({dg}, {slot_of (part, LP_DG0)});
        return;
    }
    double* sn = S + (size_t) st->newest * n;
    double* yn = Y + (size_t) st->newest * n;
    // the first loop starts at the newest pair (the one formed here)
    const bool a0 = !lb_skip (st, 0);
    const bool s0_new = lb_j1 (st, 0) == st->newest;
    const double* s0 = S + (size_t) lb_j1 (st, 0) * n;
    double ys = 0.0, yy = 0.0, sd = 0.0;
    for (long long i = i0; i < n; i += step) {
        const double si = x[i] - xp[i];
        const double yi = g[i] - gp[i];
        sn[i] = si;
        yn[i] = yi;
        ys += yi * si;
        yy += yi * yi;
        const double di = -1.0 * g[i] + 0.0 * d[i];
        d[i] = di;
        if (a0) sd += (s0_new ? si : s0[i]) * di;
    }
    block_partials<3> ({ys, yy, sd}, {slot_of (part, LP_YS),
        slot_of (part, LP_YY), slot_of (part, LP_REC)});
}

// Step i of the first loop: alpha_j = s_j.d / ys_j, d -= alpha_j y_j, and
// the partials of the next step's s_j.d.
__global__ void __launch_bounds__ (OPT_THREADS)
lb_rec_alpha_kernel (const LbDev* __restrict__ st, int i,
    const double* __restrict__ S, const double* __restrict__ Y,
    double* __restrict__ d, double* __restrict__ dsc, long long n,
    double* __restrict__ part)
{
    if (lb_skip (st, i)) return;
    const int m = st->m;
    const int j = lb_j1 (st, i);
    // ys of the newest pair is formed here; the older ones are stored
    const double ysj = i == 0 ? block_final (part, LP_YS) : dsc[j];
    const double alpha = block_final (part, LP_REC + i) / ysj;
    if (blockIdx.x == 0 && threadIdx.x == 0) dsc[m + j] = alpha;
    const bool next = i + 1 < m && !lb_skip (st, i + 1);
    const double* sn = S + (size_t) lb_j1 (st, next ? i + 1 : i) * n;
    const double* yj = Y + (size_t) j * n;
    const double av = -1.0 * alpha;
    double sd = 0.0;
    for (long long k = (long long) blockIdx.x * OPT_THREADS + threadIdx.x;
         k < n; k += (long long) gridDim.x * OPT_THREADS) {
        const double dk = av * yj[k] + 1.0 * d[k];
        d[k] = dk;
        if (next) sd += sn[k] * dk;
    }
    if (next) block_partials<1> ({sd}, {slot_of (part, LP_REC + i + 1)});
}

// Between the loops: d *= ys / yy of the newest pair (both stored for the
// pairs to come), and the partials of the second loop's first y_j.d.
__global__ void __launch_bounds__ (OPT_THREADS)
lb_rec_scale_kernel (const LbDev* __restrict__ st, const double* __restrict__ Y,
    double* __restrict__ d, double* __restrict__ dsc, long long n,
    double* __restrict__ part)
{
    if (st->first) return;
    const int m = st->m;
    const double ys = block_final (part, LP_YS);
    const double yy = block_final (part, LP_YY);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        dsc[st->newest] = ys;
        dsc[2 * m + 1] = yy;
    }
    const double bv = ys / yy;
    const bool next = !lb_skip (st, 0);
    const double* yn = Y + (size_t) lb_j2 (st, 0) * n;
    double yd = 0.0;
    for (long long k = (long long) blockIdx.x * OPT_THREADS + threadIdx.x;
         k < n; k += (long long) gridDim.x * OPT_THREADS) {
        const double dk = 0.0 * d[k] + bv * d[k];
        d[k] = dk;
        if (next) yd += yn[k] * dk;
    }
    if (next) block_partials<1> ({yd}, {slot_of (part, LP_REC + m)});
}

// Step i of the second loop: beta = y_j.d / ys_j, d += (alpha_j - beta)
// s_j, then the partials of the next step's y_j.d, or after the last step
// xp = x, gp = g and the partials of gp.d.
__global__ void __launch_bounds__ (OPT_THREADS)
lb_rec_beta_kernel (const LbDev* __restrict__ st, int i,
    const double* __restrict__ S, const double* __restrict__ Y,
    const double* __restrict__ x, double* __restrict__ xp,
    const double* __restrict__ g, double* __restrict__ gp,
    double* __restrict__ d, const double* __restrict__ dsc, long long n,
    double* __restrict__ part)
{
    if (lb_skip (st, i)) return;
    const int m = st->m;
    const int j = lb_j2 (st, i);
    const double beta = block_final (part, LP_REC + m + i) / dsc[j];
    const double av = dsc[m + j] - beta;
    const bool last = i + 1 >= m || lb_skip (st, i + 1);
    const double* yn = Y + (size_t) lb_j2 (st, last ? i : i + 1) * n;
    const double* sj = S + (size_t) j * n;
    double acc = 0.0;
    const long long i0 = (long long) blockIdx.x * OPT_THREADS + threadIdx.x;
    const long long step = (long long) gridDim.x * OPT_THREADS;
    if (!last) {
        for (long long k = i0; k < n; k += step) {
            const double dk = av * sj[k] + 1.0 * d[k];
            d[k] = dk;
            acc += yn[k] * dk;
        }
        block_partials<1> ({acc}, {slot_of (part, LP_REC + m + i + 1)});
        return;
    }
    for (long long k = i0; k < n; k += step) {
        const double dk = av * sj[k] + 1.0 * d[k];
        const double gk = g[k];
        d[k] = dk;
        xp[k] = x[k];
        gp[k] = gk;
        acc += gk * dk;
    }
    block_partials<1> ({acc}, {slot_of (part, LP_DG0)});
}

}  // namespace

// Record the graph of the run's iterations on the context's stream (which
// must be idle); false when a step of the construction is refused.
static bool
build_lbfgs_graph (b200bsp_ctx* ctx, Lbfgs& w, LbDev* dst, int metric,
    float lambda, const b200bsp_reg_parms* reg, float* coeff_f,
    float* grad_f, cudaGraphExec_t* exec)
{
    cudaStream_t st = w.st;
    const long long n = w.n;
    const unsigned grid = w.grid ();
    cudaGraph_t graph = nullptr, out = nullptr;
    bool ok = cudaGraphCreate (&graph, 0) == cudaSuccess;
    cudaGraphConditionalHandle h_while = 0, h_new = 0;
    ok = ok && cudaGraphConditionalHandleCreate (&h_while, graph, 1,
        cudaGraphCondAssignDefault) == cudaSuccess;
    ok = ok && cudaGraphConditionalHandleCreate (&h_new, graph, 1,
        cudaGraphCondAssignDefault) == cudaSuccess;
    cudaGraphNode_t wnode = nullptr, inode = nullptr;
    cudaGraph_t body = nullptr, branch = nullptr;
    if (ok) {
        cudaGraphNodeParams wp = {};
        wp.type = cudaGraphNodeTypeConditional;
        wp.conditional.handle = h_while;
        wp.conditional.type = cudaGraphCondTypeWhile;
        wp.conditional.size = 1;
        ok = cudaGraphAddNode (&wnode, graph, nullptr, 0, &wp) == cudaSuccess;
        body = wp.conditional.phGraph_out[0];
    }
    if (ok) {
        cudaGraphNodeParams ip = {};
        ip.type = cudaGraphNodeTypeConditional;
        ip.conditional.handle = h_new;
        ip.conditional.type = cudaGraphCondTypeIf;
        ip.conditional.size = 1;
        ok = cudaGraphAddNode (&inode, body, nullptr, 0, &ip) == cudaSuccess;
        branch = ip.conditional.phGraph_out[0];
    }
    const int m = w.m;
    double* ys_d = w.dsc;
    // the new-line-search branch
    if (ok && n <= LB_FUSED_MAX && cudaStreamBeginCaptureToGraph (st, branch,
            nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) == cudaSuccess) {
        lb_branch_fused_kernel<<<1, LB_FUSED_THREADS, 0, st>>> (dst, w.s, w.y,
            w.x, w.xp, w.g, w.gp, w.d, ys_d, &dst->dginit, n);
        lb_begin_search_kernel<<<1, 32, 0, st>>> (dst, h_while, nullptr, 0);
        ok = cudaStreamEndCapture (st, &out) == cudaSuccess && out == branch;
    } else if (ok && cudaStreamBeginCaptureToGraph (st, branch, nullptr,
            nullptr, 0, cudaStreamCaptureModeRelaxed) == cudaSuccess) {
        // the correction pair, the two-loop recursion, xp, gp and gp.d:
        // 2 m + 2 launches, each reducing the partials of the one before
        lb_rec_start_kernel<<<OPT_BLOCKS, OPT_THREADS, 0, st>>> (dst, w.s,
            w.y, w.x, w.xp, w.g, w.gp, w.d, n, w.part);
        for (int i = 0; i < m; i++) {
            lb_rec_alpha_kernel<<<OPT_BLOCKS, OPT_THREADS, 0, st>>> (dst, i,
                w.s, w.y, w.d, ys_d, n, w.part);
        }
        lb_rec_scale_kernel<<<OPT_BLOCKS, OPT_THREADS, 0, st>>> (dst, w.y, w.d,
            ys_d, n, w.part);
        for (int i = 0; i < m; i++) {
            lb_rec_beta_kernel<<<OPT_BLOCKS, OPT_THREADS, 0, st>>> (dst, i,
                w.s, w.y, w.x, w.xp, w.g, w.gp, w.d, ys_d, n, w.part);
        }
        lb_begin_search_kernel<<<1, 32, 0, st>>> (dst, h_while, w.part,
            OPT_BLOCKS);
        ok = cudaStreamEndCapture (st, &out) == cudaSuccess && out == branch;
    } else {
        ok = false;
    }
    // the trial: after the branch, every iteration of the loop
    if (ok && cudaStreamBeginCaptureToGraph (st, body, &inode, nullptr, 1,
            cudaStreamCaptureModeRelaxed) == cudaSuccess) {
        lb_trial_kernel<<<grid, 256, 0, st>>> (dst, w.xp, w.d, w.x, coeff_f,
            n);
        // bspline_score with device outputs: lambda * metric (+
        // regulariser)
        const int rc = b200bsp_score (ctx, coeff_f, metric, lambda, reg,
            &dst->total, grad_f, nullptr, nullptr);
        lb_eval_dots_kernel<<<OPT_BLOCKS, OPT_THREADS, 0, st>>> (grad_f, w.g,
            w.d, w.x, n, w.part);
        lb_after_eval_kernel<<<1, 32, 0, st>>> (dst, h_while, h_new, w.part,
            OPT_BLOCKS);
        ok = cudaStreamEndCapture (st, &out) == cudaSuccess && out == body
            && rc == B200BSP_OK;
    } else {
        ok = false;
    }
    ok = ok && cudaGraphInstantiate (exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy (graph);
    if (!ok) cudaGetLastError ();
    return ok;
}

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
    LbDev* lbdev = nullptr;          // the graph-resident run's state
    // the recorded graph of the iterations, and what it was recorded for
    cudaGraphExec_t exec = nullptr;
    unsigned gen = 0;
    int metric = 0;
    float lambda = 0.f;
    bool has_reg = false;
    b200bsp_reg_parms reg = {};
    ~OptWorkspace ()
    {
        if (exec) cudaGraphExecDestroy (exec);
        cudaFree (buf);
        cudaFree (lbdev);
    }
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
        || cudaMalloc (&ws->buf, 2 * nc * sizeof (float)) != cudaSuccess
        || cudaMalloc (&ws->lbdev, sizeof (LbDev)) != cudaSuccess) {
        cudaGetLastError ();
        delete ws;
        return nullptr;
    }
    ctx_set_opt_ws (ctx, ws, release_ws);
    return ws;
}

// The iterations after the prologue as one graph launch (MSE or MI on a
// context); the host-driven loop when the graph cannot be built.
static int
lbfgs_graph_run (b200bsp_ctx* ctx, Lbfgs& w, ContextObjective& obj,
    const b200bsp_lbfgs_parms& p, b200bsp_lbfgs_result* res, double f,
    double step, OptWorkspace* ws)
{
    LbDev* dst = ws->lbdev;
    LbDev h;
    memset (&h, 0, sizeof h);
    h.m = p.m;
    h.max_its = p.max_its;
    h.max_feval = p.max_feval;
    h.max_linesearch = p.max_linesearch;
    h.epsilon = p.epsilon;
    h.min_step = p.min_step;
    h.max_step = p.max_step;
    h.ftol = p.ftol;
    h.gtol = p.gtol;
    h.xtol = p.xtol;
    h.k = 1;
    h.fevals = obj.fevals;
    h.first = 1;
    h.newiter = 1;
    h.f = f;
    h.stp = step;
    h.last = obj.last;
    if (cudaMemcpyAsync (dst, &h, sizeof h, cudaMemcpyHostToDevice, w.st)
            != cudaSuccess
        || cudaStreamSynchronize (w.st) != cudaSuccess) {
        cudaGetLastError ();
        return B200BSP_E_CUDA;
    }
    // record the graph once per (context state, lambda, regulariser); the
    // history length and the buffers are the workspace's own
    const bool fresh = ws->exec && ws->gen == ctx_generation (ctx)
        && ws->metric == obj.metric && ws->lambda == obj.lambda && ws->has_reg == (obj.reg != nullptr)
        && (!obj.reg || memcmp (&ws->reg, obj.reg, sizeof ws->reg) == 0);
    if (!fresh) {
        if (ws->exec) cudaGraphExecDestroy (ws->exec);
        ws->exec = nullptr;
        if (!build_lbfgs_graph (ctx, w, dst, obj.metric, obj.lambda, obj.reg,
                obj.coeff_f, obj.grad_f, &ws->exec)) {
            ws->exec = nullptr;
            return lbfgs_loop (w, obj, p, res, f, step);
        }
        ws->gen = ctx_generation (ctx);
        ws->metric = obj.metric;
        ws->lambda = obj.lambda;
        ws->has_reg = obj.reg != nullptr;
        if (obj.reg) ws->reg = *obj.reg;
    }
    const bool ran = cudaGraphLaunch (ws->exec, w.st) == cudaSuccess
        && cudaMemcpyAsync (&h, dst, sizeof h, cudaMemcpyDeviceToHost, w.st)
            == cudaSuccess
        && cudaStreamSynchronize (w.st) == cudaSuccess;
    if (!ran) {
        cudaGetLastError ();
        return B200BSP_E_CUDA;
    }
    // a bounded device-side wait that gave up inside the run (the
    // tensor-core kernels' error flag, read once per run): its evaluations
    // are not to be trusted
    if (int* flag = ctx_err_flag (ctx)) {
        int e = 0;
        if (cudaMemcpy (&e, flag, sizeof e, cudaMemcpyDeviceToHost)
                != cudaSuccess) {
            cudaGetLastError ();
            return B200BSP_E_CUDA;
        }
        if (e) return ctx_report_device_error (ctx, e);
    }
    obj.fevals = h.fevals;
    obj.last = h.last;
    res->iterations = h.iterations;
    res->status = h.status == LS_STOPPED ? B200BSP_LBFGS_STOPPED : h.status;
    return B200BSP_OK;
}

// b200bsp_debug_host_lbfgs: this thread's runs stay on the host-driven loop
static thread_local int g_host_lbfgs = 0;

// L-BFGS over a context's coefficients (host or device floats, updated in
// place with the last evaluated point), evaluations by `obj`: MSE or MI
// without landmarks runs its iterations as one graph launch
// (lbfgs_graph_run), the rest from the host.
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
    float stiffness = 0.f;
    if ((obj.metric == 0 || obj.metric == 1)
        && ctx_landmarks (ctx, &stiffness) == 0 && !g_host_lbfgs) {
        double f = 0.0, step = 0.0;
        bool more = false;
        rc = lbfgs_prologue (w, obj, p, res, &f, &step, &more);
        if (!rc && more) {
            rc = lbfgs_graph_run (ctx, w, obj, p, res, f, step, ws);
        }
    } else {
        rc = lbfgs_run (w, obj, p, res);
    }
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

} // namespace b200

using namespace b200;

extern "C" void
b200bsp_debug_host_lbfgs (int on)
{
    g_host_lbfgs = on ? 1 : 0;
}

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
