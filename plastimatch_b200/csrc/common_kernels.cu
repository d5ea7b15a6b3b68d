// Reductions shared by all forms:
//   reduce_score  -- sum of the per-CTA score/count partials (fixed order)
//   gather_grad   -- per-knot sum of the partial gradients written by the
//                    tile kernels, normalised as bspline_score_normalize
//                    (Plastimatch src/register/bspline_mse.cxx:43-72);
//                    replaces the reference's serial condense
//                    (bspline_condense_smetric_grad, src/register/bspline.cxx:
//                    400-413) with one thread per knot, each summing its
//                    contributions in a fixed order in double precision, so
//                    the result is deterministic without atomics.
//   volume_grad   -- volume_calc_grad (src/base/volume_grad.cxx:9-76)
#include <cfloat>
#include <map>
#include <mutex>
#include <utility>

#include "kernels.cuh"

namespace b200 {

constexpr int RED_THREADS = 1024;

__global__ void __launch_bounds__ (RED_THREADS)
reduce_score_kernel (const double* __restrict__ sp, const int* __restrict__ cp,
    int n, DevResult* __restrict__ res, int mode)
{
    __shared__ double sh_v[RED_THREADS / 32];
    __shared__ int sh_n[RED_THREADS / 32];
    double v = 0.0;
    long long nn = 0;
    for (int i = threadIdx.x; i < n; i += RED_THREADS) {
        v += sp[i];
        nn += cp[i];
    }
    int n32 = (int) nn;   // per-thread counts stay far below 2^31
    block_sum<RED_THREADS> (v, n32, sh_v, sh_n);
    if (threadIdx.x == 0) {
        res->raw = v;
        res->num_vox = n32;
        res->error = 0;
        if (mode == 0) {
            if (n32 < 1) {
                res->score = FLT_MAX;
                res->score_f = FLT_MAX;
            } else {
                res->score = v / (double) n32;
                res->score_f = (float) res->score;
            }
        }
    }
}

cudaError_t
launch_reduce_score (const double* score_part, const int* count_part, int n,
    DevResult* res, int mode, cudaStream_t st)
{
    reduce_score_kernel<<<1, RED_THREADS, 0, st>>> (score_part, count_part, n,
        res, mode);
    return cudaGetLastError ();
}

// One thread per knot.  mode 0: MSE normalisation grad = 2*sum/N;
// mode 1: no normalisation (MI pass-2 dc/dv already carries 1/N).
__global__ void
gather_grad_kernel (BspGeom g, PartLayout lay, const float* __restrict__ part,
    const DevResult* __restrict__ res, int mode, float* __restrict__ grad_out,
    double* __restrict__ grad64_out, float* __restrict__ score_out,
    double* __restrict__ score64_out, long long* __restrict__ nvox_out)
{
    int knot = blockIdx.x * blockDim.x + threadIdx.x;
    long long N = res->num_vox;
    if (knot == 0) {
        if (score_out) *score_out = res->score_f;
        if (score64_out) *score64_out = res->score;
        if (nvox_out) *nvox_out = N;
    }
    if (knot >= g.nknots) return;
    const int cx = g.cdims[0], cy = g.cdims[1];
    const int kx = knot % cx, ky = (knot / cx) % cy, kz = knot / (cx * cy);
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    if (lay.slots == 64) {
        // Slot m = i + 4j + 16k of tile (kx-i, ky-j, kz-k), in slot order
        // as the reference's condense sums them.
        for (int k = 0; k < 4; k++) {
            int tz = kz - k;
            if (tz < 0 || tz >= g.rdims[2]) continue;
            for (int j = 0; j < 4; j++) {
                int ty = ky - j;
                if (ty < 0 || ty >= g.rdims[1]) continue;
                for (int i = 0; i < 4; i++) {
                    int tx = kx - i;
                    if (tx < 0 || tx >= g.rdims[0]) continue;
                    int t = tx + g.rdims[0] * (ty + g.rdims[1] * tz);
                    int m = i + 4 * j + 16 * k;
                    const float* p = part + ((size_t) m * g.ntiles + t) * 3;
                    s0 += p[0]; s1 += p[1]; s2 += p[2];
                }
            }
        }
    } else {
        // Batch footprints: batch (bi, bj, bk) covers knots
        // [bi*bx, bi*bx + bx + 3) along x, likewise y and z.
        int bi0 = max (0, (kx - lay.bx - 2 + lay.bx - 1) / lay.bx);
        if (kx - lay.bx - 2 < 0) bi0 = 0;
        int bi1 = min (lay.nbx - 1, kx / lay.bx);
        int bj0 = (ky - lay.by - 2 < 0) ? 0 : (ky - lay.by - 2 + lay.by - 1) / lay.by;
        int bj1 = min (lay.nby - 1, ky / lay.by);
        int bk0 = (kz - lay.bz - 2 < 0) ? 0 : (kz - lay.bz - 2 + lay.bz - 1) / lay.bz;
        int bk1 = min (lay.nbz - 1, kz / lay.bz);
        const int KF = lay.kx * lay.ky * lay.kz;
        for (int bk = bk0; bk <= bk1; bk++) {
            int lz = kz - bk * lay.bz;
            for (int bj = bj0; bj <= bj1; bj++) {
                int ly = ky - bj * lay.by;
                for (int bi = bi0; bi <= bi1; bi++) {
                    int lx = kx - bi * lay.bx;
                    int b = bi + lay.nbx * (bj + lay.nby * bk);
                    int kk = lx + lay.kx * (ly + lay.ky * lz);
                    const float* p = part + (size_t) b * 3 * KF + kk;
                    s0 += p[0]; s1 += p[KF]; s2 += p[2 * KF];
                }
            }
        }
    }
    if (mode == 0) {
        if (N < 1) {
            s0 = s1 = s2 = 0.0;
        } else {
            double sc = 2.0 / (double) N;
            s0 *= sc; s1 *= sc; s2 *= sc;
        }
    }
    if (grad_out) {
        grad_out[3 * knot + 0] = (float) s0;
        grad_out[3 * knot + 1] = (float) s1;
        grad_out[3 * knot + 2] = (float) s2;
    }
    if (grad64_out) {
        grad64_out[3 * knot + 0] = s0;
        grad64_out[3 * knot + 1] = s1;
        grad64_out[3 * knot + 2] = s2;
    }
}

cudaError_t
launch_gather_grad (const BspGeom& g, const PartLayout& lay, const float* part,
    const DevResult* res, int mode, float* grad_out, double* grad64_out,
    float* score_out, double* score64_out, long long* nvox_out,
    cudaStream_t st)
{
    int threads = 256;
    int blocks = (g.nknots + threads - 1) / threads;
    gather_grad_kernel<<<blocks, threads, 0, st>>> (g, lay, part, res, mode,
        grad_out, grad64_out, score_out, score64_out, nvox_out);
    return cudaGetLastError ();
}

// Score reduction and gradient gather in one launch (MSE): every block sums
// the per-CTA voxel counts in the same fixed order (it needs N to
// normalise), block 0 also sums the scores and writes the result block
// (with the tile kernel's error flag); then one thread per knot, x fastest
// so that a warp's loads of one component run along a footprint row,
// gathers each component's partials in the same order as
// gather_grad_kernel and normalises by 2 / N.  The block's gradient goes
// out through shared memory as one contiguous run (16-byte stores), which
// also suits an output in mapped host memory.
constexpr int FIN_THREADS = 256;
constexpr int FIN_UNROLL = 8;

template <typename T>
__device__ __forceinline__ void
store_run (T* __restrict__ dst, const double* __restrict__ src, int n)
{
    constexpr int V = 16 / sizeof (T);
    if (((uintptr_t) dst & 15) == 0) {
        for (int i = threadIdx.x; i < n / V; i += FIN_THREADS) {
            __align__ (16) T v[V];
#pragma unroll
            for (int e = 0; e < V; e++) v[e] = (T) src[V * i + e];
            *(uint4*) (dst + V * i) = *(const uint4*) v;
        }
        for (int i = (n / V) * V + threadIdx.x; i < n; i += FIN_THREADS) {
            dst[i] = (T) src[i];
        }
    } else {
        for (int i = threadIdx.x; i < n; i += FIN_THREADS) dst[i] = (T) src[i];
    }
}

cudaError_t
set_max_dynamic_smem (const void* kernel, int bytes)
{
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> done;   // -> bytes set
    int dev = 0;
    cudaError_t e = cudaGetDevice (&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock (mu);
    const auto key = std::make_pair (kernel, dev);
    const auto it = done.find (key);
    if (it != done.end () && it->second >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute (kernel,
        cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) done[key] = bytes;
    return e;
}

__global__ void __launch_bounds__ (FIN_THREADS)
finish_mse_kernel (BspGeom g, PartLayout lay, const float* __restrict__ part,
    const double* __restrict__ sp, const int* __restrict__ cp, int nparts,
    const int* __restrict__ err, DevResult* __restrict__ res,
    DevResult* __restrict__ res_host, float* __restrict__ grad_out,
    double* __restrict__ grad64_out, float* __restrict__ score_out,
    double* __restrict__ score64_out, long long* __restrict__ nvox_out,
    unsigned* __restrict__ clear, int nclear, FinishCombine cb)
{
    // the tile kernel's per-batch arrival counters start the next
    // evaluation at zero, also after a tile kernel that gave up early
    for (int i = blockIdx.x * FIN_THREADS + threadIdx.x; i < nclear;
         i += gridDim.x * FIN_THREADS) {
        clear[i] = 0u;
    }
    __shared__ double sh_v[FIN_THREADS / 32];
    __shared__ int sh_n[FIN_THREADS / 32];
    __shared__ long long s_n;
    __shared__ __align__ (16) double s_g[3 * FIN_THREADS];
    const bool first = blockIdx.x == 0;
    // the counts (and on block 0 the scores), FIN_UNROLL independent loads
    // at a time, each thread in ascending index order, then the fixed-order
    // block sum
    double v = 0.0;
    int n32 = 0;
    for (int i0 = threadIdx.x; i0 < nparts; i0 += FIN_UNROLL * FIN_THREADS) {
        int c8[FIN_UNROLL];
        double s8[FIN_UNROLL];
#pragma unroll
        for (int u = 0; u < FIN_UNROLL; u++) {
            const int i = i0 + u * FIN_THREADS;
            c8[u] = i < nparts ? __ldg (cp + i) : 0;
            s8[u] = first && i < nparts ? __ldg (sp + i) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < FIN_UNROLL; u++) {
            n32 += c8[u];
            v += s8[u];
        }
    }
    block_sum<FIN_THREADS> (v, n32, sh_v, sh_n);
    if (threadIdx.x == 0) {
        s_n = n32;
        if (first) {
            DevResult r;
            r.raw = v;
            r.num_vox = n32;
            r.error = err ? *err : 0;
            if (n32 < 1) {
                r.score = FLT_MAX;
                r.score_f = FLT_MAX;
            } else {
                r.score = v / (double) n32;
                r.score_f = (float) r.score;
            }
            *res = r;
            if (res_host) *res_host = r;
            if (cb.total_score) {
                // Bspline_score::accumulate then the regulariser's score
                // (src/register/bspline.cxx:595-622), in float
                float total = 0.f;
                total += cb.lambda * r.score_f;
                if (cb.reg_score) total += (float) *cb.reg_score;
                *cb.total_score = total;
            }
            if (score_out) *score_out = r.score_f;
            if (score64_out) *score64_out = r.score;
            if (nvox_out) *nvox_out = r.num_vox;
        }
    }
    __syncthreads ();
    const long long N = s_n;
    const int knot0 = blockIdx.x * FIN_THREADS;
    const int knot = knot0 + threadIdx.x;
    const double scale = N < 1 ? 0.0 : 2.0 / (double) N;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    if (knot < g.nknots) {
        const int cx = g.cdims[0], cy = g.cdims[1];
        const int kx = knot % cx, ky = (knot / cx) % cy, kz = knot / (cx * cy);
        if (lay.slots == 64) {
            // slot m = i + 4j + 16k of tile (kx-i, ky-j, kz-k), ascending
            // m; the loads of 8 slots x 3 components go out together
#pragma unroll 1
            for (int m0 = 0; m0 < 64; m0 += 8) {
                const int k = m0 >> 4, tz = kz - k;
                const bool okz = tz >= 0 && tz < g.rdims[2];
                float val[8][3];
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    const int i = q & 3, j = ((m0 + q) >> 2) & 3;
                    const int tx = kx - i, ty = ky - j;
                    const bool ok = okz && tx >= 0 && tx < g.rdims[0]
                        && ty >= 0 && ty < g.rdims[1];
                    const int t = tx + g.rdims[0] * (ty + g.rdims[1] * tz);
                    const float* p = part + ((size_t) (m0 + q) * g.ntiles
                        + (ok ? t : 0)) * 3;
                    val[q][0] = ok ? __ldg (p) : 0.f;
                    val[q][1] = ok ? __ldg (p + 1) : 0.f;
                    val[q][2] = ok ? __ldg (p + 2) : 0.f;
                }
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    s0 += val[q][0]; s1 += val[q][1]; s2 += val[q][2];
                }
            }
        } else {
            // batches (bi, bj, bk) whose footprint holds the knot: bk and
            // bj from kz - 3 .. kz and ky - 3 .. ky (the tensor-core layout
            // has one tile per batch along y and z), bi one of two (a row
            // split into several batches gives each at least 3 tiles, so a
            // footprint of bx + 3 knots meets at most two batches); per bk
            // the 8 x 3 loads first, then the sums in ascending batch order
            const int KF = lay.kx * lay.ky * lay.kz;
            const int bi1 = min (lay.nbx - 1, kx / lay.bx);
            // all 4 x 8 x 3 loads in flight (the sums stay in ascending
            // batch order)
#pragma unroll
            for (int dk = 0; dk < 4; dk++) {
                const int bk = kz - 3 + dk, lz = kz - bk * lay.bz;
                const bool okz = bk >= 0 && bk < lay.nbz && lz < lay.kz;
                float val[8][3];
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    const int dj = q >> 1, di = q & 1;
                    const int bj = ky - 3 + dj, bi = bi1 - 1 + di;
                    const int ly = ky - bj * lay.by, lx = kx - bi * lay.bx;
                    const bool ok = okz && bj >= 0 && bj < lay.nby && bi >= 0
                        && lx < lay.kx && lx >= 0 && ly < lay.ky;
                    const int b = bi + lay.nbx * (bj + lay.nby * bk);
                    const int kk = lx + lay.kx * (ly + lay.ky * lz);
                    const float* p = part + (ok ? (size_t) b * 3 * KF + kk : 0);
                    val[q][0] = ok ? __ldg (p) : 0.f;
                    val[q][1] = ok ? __ldg (p + KF) : 0.f;
                    val[q][2] = ok ? __ldg (p + 2 * KF) : 0.f;
                }
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    s0 += val[q][0]; s1 += val[q][1]; s2 += val[q][2];
                }
            }
        }
    }
    s_g[3 * threadIdx.x] = s0 * scale;
    s_g[3 * threadIdx.x + 1] = s1 * scale;
    s_g[3 * threadIdx.x + 2] = s2 * scale;
    if (cb.total_score && knot < g.nknots) {
        // total_grad = 0 + lambda * smetric_grad (float), then the
        // regulariser's double gradient added with one rounding, as the
        // separate calls would leave it
#pragma unroll
        for (int c = 0; c < 3; c++) {
            float t = 0.f + cb.lambda * (float) s_g[3 * threadIdx.x + c];
            s_g[3 * threadIdx.x + c] = cb.reg_grad
                ? (double) (float) ((double) t + cb.reg_grad[3 * (size_t) knot + c])
                : (double) t;
        }
    }
    __syncthreads ();
    const int n = 3 * min (FIN_THREADS, g.nknots - knot0);
    if (grad_out) store_run<float> (grad_out + 3 * (size_t) knot0, s_g, n);
    if (grad64_out) store_run<double> (grad64_out + 3 * (size_t) knot0, s_g, n);
}

cudaError_t
launch_finish_mse (const BspGeom& g, const PartLayout& lay, const float* part,
    const double* score_part, const int* count_part, int nparts,
    const int* err, DevResult* res, DevResult* res_host, float* grad_out,
    double* grad64_out, float* score_out, double* score64_out,
    long long* nvox_out, cudaStream_t st, unsigned* clear, int nclear,
    const FinishCombine& cb)
{
    const int blocks = std::max (1, (g.nknots + FIN_THREADS - 1) / FIN_THREADS);
    finish_mse_kernel<<<blocks, FIN_THREADS, 0, st>>> (g, lay, part,
        score_part, count_part, nparts, err, res, res_host, grad_out,
        grad64_out, score_out, score64_out, nvox_out, clear, nclear, cb);
    return cudaGetLastError ();
}

// Central differences with replicated borders, divided by 2*spacing and
// rotated by the inverse direction cosines; xyz interleaved.
__global__ void
volume_grad_kernel (int nx, int ny, int nz, float sx, float sy, float sz,
    const float* __restrict__ inv_dc9, const float* __restrict__ img,
    float* __restrict__ out)
{
    long long n = (long long) nx * ny * nz;
    long long v = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    int i = (int) (v % nx), j = (int) ((v / nx) % ny), k = (int) (v / ((long long) nx * ny));
    int ip = i > 0 ? i - 1 : 0, in = i < nx - 1 ? i + 1 : nx - 1;
    int jp = j > 0 ? j - 1 : 0, jn = j < ny - 1 ? j + 1 : ny - 1;
    int kp = k > 0 ? k - 1 : 0, kn = k < nz - 1 ? k + 1 : nz - 1;
    long long row = (long long) nx * (j + (long long) ny * k);
    float inv[9];
#pragma unroll
    for (int q = 0; q < 9; q++) inv[q] = inv_dc9[q];
    // (float)(a - b) / 2.0 / spacing, evaluated in double as the reference
    float dxv = (float) ((double) (img[row + in] - img[row + ip]) / 2.0 / (double) sx);
    float dyv = (float) ((double) (img[nx * (jn + (long long) ny * k) + i]
        - img[nx * (jp + (long long) ny * k) + i]) / 2.0 / (double) sy);
    float dzv = (float) ((double) (img[nx * (j + (long long) ny * kn) + i]
        - img[nx * (j + (long long) ny * kp) + i]) / 2.0 / (double) sz);
    float o0 = 0.f, o1 = 0.f, o2 = 0.f;
    o0 = __fadd_rn (o0, __fmul_rn (dxv, inv[0]));
    o1 = __fadd_rn (o1, __fmul_rn (dxv, inv[3]));
    o2 = __fadd_rn (o2, __fmul_rn (dxv, inv[6]));
    o0 = __fadd_rn (o0, __fmul_rn (dyv, inv[1]));
    o1 = __fadd_rn (o1, __fmul_rn (dyv, inv[4]));
    o2 = __fadd_rn (o2, __fmul_rn (dyv, inv[7]));
    o0 = __fadd_rn (o0, __fmul_rn (dzv, inv[2]));
    o1 = __fadd_rn (o1, __fmul_rn (dzv, inv[5]));
    o2 = __fadd_rn (o2, __fmul_rn (dzv, inv[8]));
    out[3 * v + 0] = o0;
    out[3 * v + 1] = o1;
    out[3 * v + 2] = o2;
}

cudaError_t
launch_volume_grad (const int dim[3], const float spacing[3],
    const float inv_dc[9], const float* img, float* grad, cudaStream_t st)
{
    long long n = (long long) dim[0] * dim[1] * dim[2];
    int threads = 256;
    long long blocks = (n + threads - 1) / threads;
    volume_grad_kernel<<<(unsigned) blocks, threads, 0, st>>> (dim[0], dim[1],
        dim[2], spacing[0], spacing[1], spacing[2], inv_dc, img, grad);
    return cudaGetLastError ();
}

__global__ void
pad_grad4_kernel (const float* __restrict__ g3, float4* __restrict__ g4,
    long long n)
{
    for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x) {
        g4[i] = make_float4 (g3[3 * i], g3[3 * i + 1], g3[3 * i + 2], 0.f);
    }
}

cudaError_t
launch_pad_grad4 (const float* grad3, float4* grad4, long long n,
    cudaStream_t st)
{
    pad_grad4_kernel<<<1184, 256, 0, st>>> (grad3, grad4, n);
    return cudaGetLastError ();
}

} // namespace b200

namespace b200 {

// The fixed ROI test of every fixed voxel as a byte (bit 0: at origin +
// step * ijk, POSITION_FROM_COORDS, src/base/volume_macros.h:82-97; bit 1:
// at the position LOOP_Z/Y/X accumulate, :38-76, which the reference's
// whole-image MI histogram scan uses).  One thread per image row walks x,
// accumulating as LOOP_X does.
__global__ void
fixed_roi_mask_kernel (int nx, int ny, int nz, RoiGeom fg, RoiGeom rg,
    const uint8_t* __restrict__ roi, uint8_t* __restrict__ out)
{
    const long long row = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= (long long) ny * nz) return;
    const int j = (int) (row % ny), k = (int) (row / ny);
    const float* o = fg.origin;
    const float* st = fg.step;
    float acc[3];
    acc[0] = __fadd_rn (__fadd_rn (o[0], __fmul_rn ((float) k, st[2])),
        __fmul_rn ((float) j, st[1]));
    acc[1] = __fadd_rn (__fadd_rn (o[1], __fmul_rn ((float) k, st[5])),
        __fmul_rn ((float) j, st[4]));
    acc[2] = __fadd_rn (__fadd_rn (o[2], __fmul_rn ((float) k, st[8])),
        __fmul_rn ((float) j, st[7]));
    uint8_t* dst = out + row * nx;
    for (int i = 0; i < nx; i++) {
        float p[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            p[d] = __fadd_rn (__fadd_rn (__fadd_rn (o[d],
                __fmul_rn ((float) i, st[3 * d])),
                __fmul_rn ((float) j, st[3 * d + 1])),
                __fmul_rn ((float) k, st[3 * d + 2]));
        }
        const bool b0 = inside_roi_dev (roi, rg.dim, rg.origin, rg.proj, p);
        const bool b1 = inside_roi_dev (roi, rg.dim, rg.origin, rg.proj, acc);
        dst[i] = (uint8_t) ((b0 ? 1 : 0) | (b1 ? 2 : 0));
#pragma unroll
        for (int d = 0; d < 3; d++) acc[d] = __fadd_rn (acc[d], st[3 * d]);
    }
}

cudaError_t
launch_fixed_roi_mask (const int fdim[3], const RoiGeom& fixed,
    const RoiGeom& roi_geom, const uint8_t* roi, uint8_t* out,
    cudaStream_t st)
{
    const long long rows = (long long) fdim[1] * fdim[2];
    const int threads = 128;
    fixed_roi_mask_kernel<<<(unsigned) ((rows + threads - 1) / threads),
        threads, 0, st>>> (fdim[0], fdim[1], fdim[2], fixed, roi_geom, roi, out);
    return cudaGetLastError ();
}

} // namespace b200
