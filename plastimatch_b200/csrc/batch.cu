// Batched registrations: many contexts (uneven volume sizes, one device)
// evaluated together.
//
// One batch evaluation is one CUDA graph launch: the graph forks from the
// batch's stream into every context's stream, runs that context's tile pass
// and finish kernel there, gathers the contexts' device error flags and
// joins.  Graphs are captured once per set of participating contexts and
// replayed.
//
// The batched L-BFGS runs every registration's graph-resident optimiser
// (b200bsp_optimize_lbfgs, optimize.cu) at once, each on its context's
// stream, and no trial point waits for the host.  Each registration's
// trial sequence is that of b200bsp_optimize_lbfgs.
//
// Every context's persistent kernel keeps its full grid: the kernels of
// different registrations take SMs as they free up (no CTA of these
// kernels waits for another CTA, so none needs the others resident), and
// the optimisers' small kernels fill the gaps.  A fixed split of the SMs
// in proportion to each registration's voxels measured 2.6x slower on the
// 16-registration workload: registrations that finish early leave their
// share idle while the others run on theirs.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "kernels.cuh"
#include "../../include/plastimatch_b200.h"

namespace b200 {
cudaStream_t ctx_stream (const b200bsp_ctx* c);                 // runtime.cu
int ctx_device (const b200bsp_ctx* c);
int* ctx_err_flag (b200bsp_ctx* c);
int ctx_report_device_error (b200bsp_ctx* c, int e);

// Largest error flag over the participating contexts.
__global__ void
batch_err_kernel (int* const* flags, int n, int* out)
{
    int e = 0;
    for (int i = threadIdx.x; i < n; i += 32) {
        if (flags[i]) e = max (e, *flags[i]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e = max (e, __shfl_down_sync (0xffffffffu, e, o));
    if (threadIdx.x == 0) *out = e;
}
} // namespace b200

using namespace b200;

struct b200bsp_batch {
    std::vector<b200bsp_ctx*> ctx;
    int device = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    int** d_flags = nullptr;            // per context: its error flag
    int* d_err = nullptr;
    int* h_err = nullptr;
    struct Graph {
        std::vector<const void*> key;
        cudaGraphExec_t exec;
    };
    std::vector<Graph> graphs;
    std::string err;

    std::mutex mu;                      // one batch evaluation at a time
    float* d_scores = nullptr;
    float* h_scores = nullptr;
};

static int
bfail (b200bsp_batch* b, int code, const char* msg)
{
    if (b) b->err = msg;
    return code;
}

#define BCK(b, x)                                                           \
    do {                                                                    \
        cudaError_t e_ = (x);                                               \
        if (e_ != cudaSuccess) {                                            \
            cudaGetLastError ();                                            \
            return bfail (b, B200BSP_E_CUDA, cudaGetErrorString (e_));      \
        }                                                                   \
    } while (0)

// Capture (or find) the graph evaluating contexts `sel` with the given
// device buffers, and launch it on the batch stream.  The graph ends with
// the copy of the error flag (and, for the batch's own score buffer, of the
// scores) into page-locked host memory, so one synchronisation ends it.
static int
launch_eval (b200bsp_batch* b, const std::vector<int>& sel,
    const float* const* coeffs, float* const* grads, float* scores,
    int64_t* nvox)
{
    const bool own_scores = scores == b->d_scores;
    std::vector<const void*> key;
    for (int i : sel) {
        key.push_back ((const void*) (intptr_t) i);
        key.push_back (coeffs[i]);
        key.push_back (grads[i]);
    }
    key.push_back (scores);
    key.push_back (nvox);
    cudaGraphExec_t exec = nullptr;
    for (auto& gph : b->graphs) {
        if (gph.key == key) exec = gph.exec;
    }
    if (!exec) {
        cudaGraph_t graph = nullptr;
        BCK (b, cudaStreamBeginCapture (b->st, cudaStreamCaptureModeRelaxed));
        int rc = 0;
        if (cudaEventRecord (b->fork, b->st) != cudaSuccess) rc = B200BSP_E_CUDA;
        for (size_t k = 0; k < sel.size () && !rc; k++) {
            const int i = sel[k];
            cudaStream_t s = ctx_stream (b->ctx[i]);
            if (cudaStreamWaitEvent (s, b->fork, 0) != cudaSuccess) {
                rc = B200BSP_E_CUDA;
                break;
            }
            rc = b200bsp_score_mse (b->ctx[i], coeffs[i], scores + i, grads[i],
                nvox ? nvox + i : nullptr);
            if (!rc && (cudaEventRecord (b->join[i], s) != cudaSuccess
                    || cudaStreamWaitEvent (b->st, b->join[i], 0) != cudaSuccess)) {
                rc = B200BSP_E_CUDA;
            }
        }
        if (!rc) {
            batch_err_kernel<<<1, 32, 0, b->st>>> (b->d_flags, (int) b->ctx.size (),
                b->d_err);
            if (cudaMemcpyAsync (b->h_err, b->d_err, sizeof (int),
                    cudaMemcpyDeviceToHost, b->st) != cudaSuccess
                || (own_scores && cudaMemcpyAsync (b->h_scores, b->d_scores,
                    b->ctx.size () * sizeof (float), cudaMemcpyDeviceToHost,
                    b->st) != cudaSuccess)) {
                rc = B200BSP_E_CUDA;
            }
        }
        cudaError_t ce = cudaStreamEndCapture (b->st, &graph);
        if (rc || ce != cudaSuccess) {
            cudaGetLastError ();
            if (graph) cudaGraphDestroy (graph);
            return bfail (b, rc ? rc : B200BSP_E_CUDA,
                "capturing the batch evaluation failed");
        }
        ce = cudaGraphInstantiate (&exec, graph, 0);
        cudaGraphDestroy (graph);
        if (ce != cudaSuccess) {
            cudaGetLastError ();
            return bfail (b, B200BSP_E_CUDA, "graph instantiation failed");
        }
        b->graphs.push_back ({key, exec});
    }
    BCK (b, cudaGraphLaunch (exec, b->st));
    BCK (b, cudaStreamSynchronize (b->st));
    if (*b->h_err) {
        for (int i : sel) ctx_report_device_error (b->ctx[i], *b->h_err);
        return bfail (b, B200BSP_E_TIMEOUT,
            "a bounded device-side wait gave up in a batch evaluation");
    }
    return B200BSP_OK;
}

extern "C" int
b200bsp_batch_create (b200bsp_ctx* const* ctxs, int n, b200bsp_batch** out)
{
    if (!ctxs || n < 1 || !out) return B200BSP_E_BADARG;
    *out = nullptr;
    const int dev = ctx_device (ctxs[0]);
    for (int i = 0; i < n; i++) {
        if (!ctxs[i] || ctx_device (ctxs[i]) != dev) return B200BSP_E_BADARG;
        for (int j = 0; j < i; j++) {
            if (ctxs[j] == ctxs[i]) return B200BSP_E_BADARG;
        }
    }
    auto* b = new b200bsp_batch ();
    b->ctx.assign (ctxs, ctxs + n);
    b->device = dev;
    b->join.assign (n, nullptr);
    int rc = B200BSP_OK;
    if (cudaSetDevice (dev) != cudaSuccess
        || cudaStreamCreateWithFlags (&b->st, cudaStreamNonBlocking) != cudaSuccess
        || cudaEventCreateWithFlags (&b->fork, cudaEventDisableTiming) != cudaSuccess
        || cudaMalloc (&b->d_flags, n * sizeof (int*)) != cudaSuccess
        || cudaMalloc (&b->d_err, sizeof (int)) != cudaSuccess
        || cudaMallocHost (&b->h_err, sizeof (int)) != cudaSuccess
        || cudaMalloc (&b->d_scores, n * sizeof (float)) != cudaSuccess
        || cudaMallocHost (&b->h_scores, n * sizeof (float)) != cudaSuccess) {
        rc = B200BSP_E_OOM;
    }
    for (int i = 0; i < n && !rc; i++) {
        if (cudaEventCreateWithFlags (&b->join[i], cudaEventDisableTiming)
            != cudaSuccess) {
            rc = B200BSP_E_CUDA;
        }
    }
    if (!rc) {
        std::vector<int*> flags (n);
        for (int i = 0; i < n; i++) flags[i] = ctx_err_flag (ctxs[i]);
        if (cudaMemcpy (b->d_flags, flags.data (), n * sizeof (int*),
                cudaMemcpyHostToDevice) != cudaSuccess) {
            rc = B200BSP_E_CUDA;
        }
    }
    if (rc) {
        cudaGetLastError ();
        b200bsp_batch_destroy (b);
        return rc;
    }
    *out = b;
    return B200BSP_OK;
}

extern "C" void
b200bsp_batch_destroy (b200bsp_batch* b)
{
    if (!b) return;
    cudaSetDevice (b->device);
    if (b->st) cudaStreamSynchronize (b->st);
    for (auto& g : b->graphs) cudaGraphExecDestroy (g.exec);
    for (auto e : b->join) if (e) cudaEventDestroy (e);
    if (b->fork) cudaEventDestroy (b->fork);
    if (b->st) cudaStreamDestroy (b->st);
    cudaFree (b->d_flags);
    cudaFree (b->d_err);
    cudaFreeHost (b->h_err);
    cudaFree (b->d_scores);
    cudaFreeHost (b->h_scores);
    delete b;
}

extern "C" const char*
b200bsp_batch_last_error (const b200bsp_batch* b)
{
    return b ? b->err.c_str () : "null batch";
}

extern "C" int
b200bsp_batch_score_mse (b200bsp_batch* b, const float* const* coeffs,
    float* const* grads, float* scores, int64_t* num_vox)
{
    if (!b || !coeffs || !grads || !scores) {
        return bfail (b, B200BSP_E_BADARG, "null argument");
    }
    const int n = (int) b->ctx.size ();
    for (int i = 0; i < n; i++) {
        if (!coeffs[i] || !grads[i]) return bfail (b, B200BSP_E_BADARG, "null buffer");
        cudaPointerAttributes a1, a2;
        if (cudaPointerGetAttributes (&a1, coeffs[i]) != cudaSuccess
            || cudaPointerGetAttributes (&a2, grads[i]) != cudaSuccess
            || a1.type != cudaMemoryTypeDevice || a2.type != cudaMemoryTypeDevice) {
            cudaGetLastError ();
            return bfail (b, B200BSP_E_BADARG,
                "batch buffers must be device memory");
        }
    }
    BCK (b, cudaSetDevice (b->device));
    std::vector<int> sel (n);
    for (int i = 0; i < n; i++) sel[i] = i;
    std::lock_guard<std::mutex> lk (b->mu);
    return launch_eval (b, sel, coeffs, grads, scores, num_vox);
}

// ---- batched L-BFGS ---------------------------------------------------------
//
// Every registration runs the graph-resident optimiser on its own context
// and stream, all at once from one host thread each: no trial waits for
// the host, and the kernels of different registrations take the SMs as
// they free up.

extern "C" int
b200bsp_batch_optimize_lbfgs (b200bsp_batch* b, float lambda,
    const b200bsp_lbfgs_parms* parms, float* const* coeffs,
    b200bsp_lbfgs_result* results)
{
    if (!b || !coeffs || !results) return bfail (b, B200BSP_E_BADARG, "null argument");
    const int n = (int) b->ctx.size ();
    for (int i = 0; i < n; i++) {
        if (!coeffs[i]) return bfail (b, B200BSP_E_BADARG, "null coefficients");
    }
    std::vector<int> rcs (n, B200BSP_OK);
    std::vector<std::thread> th;
    th.reserve (n);
    for (int i = 0; i < n; i++) {
        th.emplace_back ([&, i] {
            cudaSetDevice (b->device);
            rcs[i] = b200bsp_optimize_lbfgs (b->ctx[i], 0, lambda, nullptr,
                parms, coeffs[i], &results[i]);
        });
    }
    for (auto& t : th) t.join ();
    for (int i = 0; i < n; i++) {
        if (rcs[i]) {
            char msg[96];
            snprintf (msg, sizeof msg, "registration %d failed (status %d)", i,
                rcs[i]);
            return bfail (b, rcs[i], msg);
        }
    }
    return B200BSP_OK;
}
