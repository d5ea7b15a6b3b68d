// Mattes mutual information with partial-volume (PVI-8) histograms,
// flavour g semantics (Plastimatch src/register/bspline_mi.cxx:1505-1750):
//
//   set_images  EQSP bin ranges from the image min/max
//               (bspline_initialize_mi_hist_eqsp, src/register/
//               joint_histogram.cxx:115-139) and a one-byte bin image per
//               volume: bin = floor((v - offset) / delta), the reference's
//               binning arithmetic, evaluated once instead of per access.
//   pass 1      per voxel: the eight trilinear corner weights are added to
//               the moving and joint histograms, 1 to the fixed histogram
//               (Joint_histogram::add_pvi_8, joint_histogram.cxx:423-486).
//               Each CTA accumulates in shared memory; weights are summed as
//               64-bit integers in 2^-24 units, so the result is exact up to
//               one rounding per weight and independent of the order in
//               which threads add -- deterministic without float atomics.
//   score       S = -sum_j j log(N j / (f m)) / N over j > 0.001/bins^2
//               (mi_hist_score_omp, src/register/bspline_mi.cxx:285-309), and
//               the per-joint-bin factor log(N j / (f m)) - S used by pass 2
//               for j > 0.0001.
//   pass 2      dc/dv = -sum_pv dw_pv (factor) / N, rotated by proj with the
//               reference's in-place projection (bspline_mi_pvi_8_dc_dv_dcos,
//               src/register/bspline_mi.txx:9-120), then the tile adjoint.
#include <cfloat>
#include <cmath>
#include <vector>

#include "../../include/plastimatch_b200.h"
#include "fp32_tile.cuh"
#include "mi.cuh"

namespace b200 {


// ---- ranges and bin images -------------------------------------------------

__global__ void
minmax_kernel (const float* __restrict__ img, long long n, float* out)
{
    __shared__ float smn[256], smx[256];
    float mn = FLT_MAX, mx = -FLT_MAX;
    for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x) {
        float v = img[i];
        mn = fminf (mn, v);
        mx = fmaxf (mx, v);
    }
    smn[threadIdx.x] = mn;
    smx[threadIdx.x] = mx;
    __syncthreads ();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            smn[threadIdx.x] = fminf (smn[threadIdx.x], smn[threadIdx.x + o]);
            smx[threadIdx.x] = fmaxf (smx[threadIdx.x], smx[threadIdx.x + o]);
        }
        __syncthreads ();
    }
    if (threadIdx.x == 0) {
        out[2 * blockIdx.x] = smn[0];
        out[2 * blockIdx.x + 1] = smx[0];
    }
}

__global__ void
bin_image_kernel (const float* __restrict__ img, long long n, float offset,
    float delta, int bins, uint8_t* __restrict__ out)
{
    for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x) {
        // (v - offset) / delta in float, IEEE division, then floor
        float b = floorf (__fdiv_rn (img[i] - offset, delta));
        int bi = (int) fminf (fmaxf (b, 0.f), (float) (bins - 1));
        out[i] = (uint8_t) bi;
    }
}

// V-optimal bins: key = floor((v - offset) / delta) over MI_VOPT_KEYS fine
// keys, bin = key_lut[key] (the reference's lookup, bspline_mi.cxx:565-579).
__global__ void
bin_image_vopt_kernel (const float* __restrict__ img, long long n,
    float offset, float delta, const int* __restrict__ key_lut,
    uint8_t* __restrict__ out)
{
    for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x) {
        float b = floorf (__fdiv_rn (img[i] - offset, delta));
        int k = (int) fminf (fmaxf (b, 0.f), (float) (MI_VOPT_KEYS - 1));
        out[i] = (uint8_t) __ldg (key_lut + k);
    }
}

// The V-optimal histogram of one image (the reference's
// bspline_initialize_mi_hist_vopt, src/register/joint_histogram.cxx:
// 195-324, restated): MI_VOPT_KEYS equal keys over the value range, each
// key's voxel count and mean, and the split of the keys into `bins`
// contiguous bins that minimises the summed within-bin squared error of
// the key means (dynamic programme over prefix sums; ties go to the later
// split, as the reference's "<=" does).  Host code in double, in the
// reference's operation order, so the key table is the reference's.
static void
vopt_table (const float* img, size_t n, int bins, float* offset_out,
    float* delta_out, std::vector<int>& key_lut)
{
    const int K = MI_VOPT_KEYS;
    std::vector<double> hist (K, 0.0), avg (K, 0.0), s (K), ssq (K), cnt (K);
    float mn = img[0], mx = img[0];
    for (size_t i = 1; i < n; i++) {
        if (img[i] < mn) mn = img[i];
        else if (img[i] > mx) mx = img[i];
    }
    const float delta = (mx - mn) / (K - 1);
    const float offset = (float) (mn - 0.5 * delta);
    for (size_t i = 0; i < n; i++) {
        const float v = img[i] - offset;
        const int b = (int) std::floor (v / delta);
        hist[b] += 1.0;
        avg[b] += v;
    }
    for (int i = 0; i < K; i++) {
        if (hist[i] > 0) avg[i] = avg[i] / hist[i];
        else if (i > 0) avg[i] = avg[i - 1];
    }
    s[0] = avg[0];
    ssq[0] = avg[0] * avg[0];
    cnt[0] = hist[0];
    for (int i = 1; i < K; i++) {
        s[i] = s[i - 1] + avg[i];
        ssq[i] = ssq[i - 1] + avg[i] * avg[i];
        cnt[i] = cnt[i - 1] + hist[i];
    }
    auto bin_err = [&](int a, int b) {
        const double d = s[b] - s[a];
        const double v = (ssq[b] - ssq[a]) - (d * d) / ((double) b - (double) a + 1.0);
        return cnt[b] - cnt[a] < 1.0 ? DBL_MAX : v;
    };
    std::vector<double> err ((size_t) bins * K);
    std::vector<int> trk ((size_t) bins * K, 0);
    for (int i = 0; i < K; i++) err[i] = bin_err (0, i);
    for (int j = 1; j < bins; j++) {
        const double* prev = err.data () + (size_t) K * (j - 1);
        double* cur = err.data () + (size_t) K * j;
        int* tj = trk.data () + (size_t) K * j;
        for (int i = 0; i < K; i++) {
            double best = DBL_MAX;
            int arg = 0;
            for (int k = 0; k < i; k++) {
                const double c = prev[k] + bin_err (k + 1, i);
                if (c <= best) {
                    best = c;
                    arg = k;
                }
            }
            cur[i] = best;
            tj[i] = arg;
        }
    }
    key_lut.assign (K, 0);
    int curr = K - 1;
    for (int j = bins - 1; j >= 0; j--) {
        const int next = trk[(size_t) K * j + curr];
        const int bottom = j == 0 ? 0 : next + 1;
        for (int i = bottom; i <= curr; i++) key_lut[i] = j;
        curr = next;
    }
    *offset_out = offset;
    *delta_out = delta;
}

static int
vopt_bins (const float* d_img, size_t n, int bins, float* offset,
    float* delta, int* d_key, uint8_t* d_bin, cudaStream_t st)
{
    std::vector<float> h (n);
    std::vector<int> lut;
    if (cudaMemcpyAsync (h.data (), d_img, n * sizeof (float),
            cudaMemcpyDeviceToHost, st) != cudaSuccess
        || cudaStreamSynchronize (st) != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    vopt_table (h.data (), n, bins, offset, delta, lut);
    if (!(*delta > 0.f)) return B200BSP_E_BADARG;     // constant image
    if (cudaMemcpyAsync (d_key, lut.data (), MI_VOPT_KEYS * sizeof (int),
            cudaMemcpyHostToDevice, st) != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    bin_image_vopt_kernel<<<1184, 256, 0, st>>> (d_img, (long long) n, *offset,
        *delta, d_key, d_bin);
    if (cudaGetLastError () != cudaSuccess
        || cudaStreamSynchronize (st) != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    return B200BSP_OK;
}

static int
image_range (const float* d_img, size_t n, float* d_scratch, float* mn_out,
    float* mx_out, cudaStream_t st)
{
    const int blocks = 296;
    minmax_kernel<<<blocks, 256, 0, st>>> (d_img, (long long) n, d_scratch);
    std::vector<float> mm (2 * blocks);
    if (cudaMemcpyAsync (mm.data (), d_scratch, mm.size () * sizeof (float),
            cudaMemcpyDeviceToHost, st) != cudaSuccess
        || cudaStreamSynchronize (st) != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    float mn = FLT_MAX, mx = -FLT_MAX;
    for (int b = 0; b < blocks; b++) {
        mn = std::fmin (mn, mm[2 * b]);
        mx = std::fmax (mx, mm[2 * b + 1]);
    }
    *mn_out = mn;
    *mx_out = mx;
    return B200BSP_OK;
}

// Parzen fixed bins: floor((v - min) / delta) + 2 in [2, bins - 3].
__global__ void
parzen_bin_kernel (const float* __restrict__ img, long long n, float vmin,
    float delta, int bins, uint8_t* __restrict__ out)
{
    for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x) {
        const int b = (int) floorf (__fdiv_rn (img[i] - vmin, delta)) + 2;
        out[i] = (uint8_t) min (max (b, 2), bins - 3);
    }
}

static int
eqsp_range (const float* d_img, size_t n, int bins, float* d_scratch,
    float* offset, float* delta, cudaStream_t st)
{
    float mn, mx;
    int rc = image_range (d_img, n, d_scratch, &mn, &mx, st);
    if (rc) return rc;
    // delta = (max - min) / (bins - 1); offset = min - 0.5 * delta
    *delta = (mx - mn) / (float) (bins - 1);
    *offset = (float) (mn - 0.5 * (double) *delta);
    if (!(*delta > 0.f)) {
        *delta = 1.f;      // constant image: every voxel in bin 0
    }
    return B200BSP_OK;
}

int
mi_alloc (MiState* s, const BspGeom& g, int bins, int window, int hist)
{
    s->bins = bins;
    s->window = window;
    s->hist = hist;
    if (hist == B200BSP_MI_HIST_VOPT
        && (cudaMalloc (&s->d_fkey, MI_VOPT_KEYS * sizeof (int)) != cudaSuccess
            || cudaMalloc (&s->d_mkey, MI_VOPT_KEYS * sizeof (int)) != cudaSuccess)) {
        cudaGetLastError ();
        return B200BSP_E_OOM;
    }
    size_t nf = (size_t) g.fdim[0] * g.fdim[1] * g.fdim[2];
    size_t nm = (size_t) g.mdim[0] * g.mdim[1] * g.mdim[2];
    size_t nh = 2 * bins + bins * bins + 1;
    if (cudaMalloc (&s->d_fbin, nf) != cudaSuccess
        || cudaMalloc (&s->d_mbin, nm) != cudaSuccess
        || cudaMalloc (&s->d_hist, nh * sizeof (unsigned long long)) != cudaSuccess
        || cudaMalloc (&s->d_histd, nh * sizeof (double)) != cudaSuccess
        || cudaMalloc (&s->d_lut, bins * bins * sizeof (float)) != cudaSuccess
        || cudaMalloc (&s->d_nvf, 2 * sizeof (float)) != cudaSuccess
        || cudaMalloc (&s->d_minmax, 2 * 296 * sizeof (float)) != cudaSuccess
        || cudaMalloc (&s->d_part, (size_t) 64 * 3 * g.ntiles * sizeof (float))
            != cudaSuccess
        || cudaMalloc (&s->d_score_part, g.ntiles * sizeof (double)) != cudaSuccess
        || cudaMalloc (&s->d_count_part, g.ntiles * sizeof (int)) != cudaSuccess
        || cudaMallocHost (&s->h_histd, nh * sizeof (double)) != cudaSuccess
        || cudaMallocHost (&s->h_res, sizeof (DevResult)) != cudaSuccess) {
        cudaGetLastError ();
        return B200BSP_E_OOM;
    }
    return B200BSP_OK;
}

void
mi_free (MiState* s)
{
    cudaFree (s->d_fbin); cudaFree (s->d_mbin); cudaFree (s->d_hist);
    cudaFree (s->d_histd); cudaFree (s->d_lut); cudaFree (s->d_nvf);
    cudaFree (s->d_minmax); cudaFree (s->d_part); cudaFree (s->d_score_part);
    cudaFree (s->d_count_part);
    cudaFree (s->d_fkey); cudaFree (s->d_mkey);
    cudaFreeHost (s->h_histd); cudaFreeHost (s->h_res);
    *s = MiState ();
}

int
mi_set_images (MiState* s, const BspGeom& g, const float* d_fixed,
    const float* d_moving, size_t nf, size_t nm, cudaStream_t st)
{
    if (s->window == B200BSP_MI_PARZEN) {
        // value ranges mapped onto bins 2 .. bins - 2 (two padding bins at
        // either end hold the cubic window's tails)
        float fmn, fmx, mmn, mmx;
        int rc = image_range (d_fixed, nf, s->d_minmax, &fmn, &fmx, st);
        if (!rc) rc = image_range (d_moving, nm, s->d_minmax, &mmn, &mmx, st);
        if (rc) return rc;
        s->pz_fmin = fmn;
        s->pz_mmin = mmn;
        s->pz_fdelta = fmx > fmn ? (fmx - fmn) / (float) (s->bins - 4) : 1.f;
        s->pz_mdelta = mmx > mmn ? (mmx - mmn) / (float) (s->bins - 4) : 1.f;
        parzen_bin_kernel<<<1184, 256, 0, st>>> (d_fixed, (long long) nf,
            s->pz_fmin, s->pz_fdelta, s->bins, s->d_fbin);
        if (cudaGetLastError () != cudaSuccess) return B200BSP_E_CUDA;
        s->ready = true;
        return B200BSP_OK;
    }
    if (s->hist == B200BSP_MI_HIST_VOPT) {
        int rc = vopt_bins (d_fixed, nf, s->bins, &s->f_offset, &s->f_delta,
            s->d_fkey, s->d_fbin, st);
        if (!rc) rc = vopt_bins (d_moving, nm, s->bins, &s->m_offset,
            &s->m_delta, s->d_mkey, s->d_mbin, st);
        if (rc) return rc;
        s->ready = true;
        return B200BSP_OK;
    }
    int rc = eqsp_range (d_fixed, nf, s->bins, s->d_minmax, &s->f_offset,
        &s->f_delta, st);
    if (rc) return rc;
    rc = eqsp_range (d_moving, nm, s->bins, s->d_minmax, &s->m_offset,
        &s->m_delta, st);
    if (rc) return rc;
    bin_image_kernel<<<1184, 256, 0, st>>> (d_fixed, (long long) nf,
        s->f_offset, s->f_delta, s->bins, s->d_fbin);
    bin_image_kernel<<<1184, 256, 0, st>>> (d_moving, (long long) nm,
        s->m_offset, s->m_delta, s->bins, s->d_mbin);
    if (cudaGetLastError () != cudaSuccess) return B200BSP_E_CUDA;
    s->ready = true;
    return B200BSP_OK;
}

// ---- pass 1: histograms ----------------------------------------------------
//
// Weights are summed as integers in units of 2^-24 (one rounding per
// weight), so the histograms do not depend on the order of the additions.
// Voxels of a warp mostly fall into the same few bins (smooth regions), and
// same-address atomics of one warp are serialised; each voxel therefore
// first merges its eight corners by moving bin, and lanes whose corners all
// share one bin are combined across the warp (match + reduce) so that one
// lane per distinct (fixed, moving) bin pair updates shared memory.

constexpr int MIH_THREADS = 128;
constexpr float MI_WUNIT = 16777216.0f;      // 2^24
constexpr double MI_WUNIT_INV = 1.0 / 16777216.0;

__global__ void __launch_bounds__ (MIH_THREADS)
mi_hist_kernel (BspGeom g, const float* __restrict__ coeff,
    const float* __restrict__ luts, const uint8_t* __restrict__ fbin,
    const uint8_t* __restrict__ mbin, int B,
    unsigned long long* __restrict__ ghist)
{
    extern __shared__ unsigned long long hsm[];   // f[B], m[B], j[B*B]
    __shared__ float sC[192];
    __shared__ float slut[4 * 3 * 64];
    const int nh = 2 * B + B * B;
    const int vx = g.vpr[0], vy = g.vpr[1], vz = g.vpr[2];
    const int V = vx * vy * vz;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long* hf = hsm;
    unsigned long long* hm = hsm + B;
    unsigned long long* hj = hsm + 2 * B;
    for (int i = threadIdx.x; i < nh; i += MIH_THREADS) hsm[i] = 0ull;
    for (int o = threadIdx.x; o < 4 * (vx + vy + vz); o += MIH_THREADS) {
        slut[o] = luts[o];
    }
    const float* sbx = slut;
    const float* sby = slut + 4 * vx;
    const float* sbz = sby + 4 * vy;
    const int dx = g.mdim[0], dxy = g.mdim[0] * g.mdim[1];
    unsigned int cnt = 0;
    __syncthreads ();
    for (int t = blockIdx.x; t < g.ntiles; t += gridDim.x) {
        const int tx = t % g.rdims[0];
        const int ty = (t / g.rdims[0]) % g.rdims[1];
        const int tz = t / (g.rdims[0] * g.rdims[1]);
        for (int o = threadIdx.x; o < 192; o += MIH_THREADS) {
            int m = o / 3, c = o - 3 * m;
            int i = m & 3, j = (m >> 2) & 3, k = m >> 4;
            sC[o] = coeff[3 * ((tz + k) * g.cdims[1] * g.cdims[0]
                + (ty + j) * g.cdims[0] + (tx + i)) + c];
        }
        __syncthreads ();
        // warp-uniform trip count: every lane reaches the warp collectives
        for (int v0 = 32 * warp; v0 < V; v0 += MIH_THREADS) {
            const int v = v0 + lane;
            const int vv = v < V ? v : 0;
            int lx = vv % vx, ly = (vv / vx) % vy, lz = vv / (vx * vy);
            int fi = g.roi_off[0] + vx * tx + lx;
            int fj = g.roi_off[1] + vy * ty + ly;
            int fk = g.roi_off[2] + vz * tz + lz;
            bool live = v < V && fi < g.roi_off[0] + g.roi_dim[0]
                && fj < g.roi_off[1] + g.roi_dim[1]
                && fk < g.roi_off[2] + g.roi_dim[2];
            int fb = 0, mb[8];
            unsigned int q[8];
            live = live && roi_fixed_ok (g, fi + g.fdim[0] * (fj + g.fdim[1] * fk), 2);
            if (live) {
                float fxyz[3], d[3] = {0.f, 0.f, 0.f};
                fixed_position (g, fi, fj, fk, fxyz);
                int m = 0;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    float C = sbz[lz * 4 + k];
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        float Bv = sby[ly * 4 + j] * C;
#pragma unroll
                        for (int i = 0; i < 4; i++, m++) {
                            float A = sbx[lx * 4 + i] * Bv;
                            d[0] += A * sC[3 * m + 0];
                            d[1] += A * sC[3 * m + 1];
                            d[2] += A * sC[3 * m + 2];
                        }
                    }
                }
                Sample s;
                live = locate (g, fxyz, d, s) && roi_moving_ok (g, fxyz, d);
                if (live) {
                    const float* l1 = s.w1;
                    const float* l2 = s.w2;
                    const float w[8] = {l1[0] * l1[1] * l1[2],
                        l2[0] * l1[1] * l1[2], l1[0] * l2[1] * l1[2],
                        l2[0] * l2[1] * l1[2], l1[0] * l1[1] * l2[2],
                        l2[0] * l1[1] * l2[2], l1[0] * l2[1] * l2[2],
                        l2[0] * l2[1] * l2[2]};
                    const int nbr[8] = {s.mvf, s.mvf + 1, s.mvf + dx,
                        s.mvf + dx + 1, s.mvf + dxy, s.mvf + dxy + 1,
                        s.mvf + dxy + dx, s.mvf + dxy + dx + 1};
                    fb = fbin[fi + g.fdim[0] * (fj + g.fdim[1] * fk)];
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        mb[k] = mbin[nbr[k]];
                        q[k] = __float2uint_rn (w[k] * MI_WUNIT);
                    }
                }
            }
            // merge corners with equal moving bins into the first of them
            bool first[8];
            bool single = true;
#pragma unroll
            for (int k = 0; k < 8; k++) first[k] = live;
#pragma unroll
            for (int k = 1; k < 8; k++) {
#pragma unroll
                for (int k2 = 0; k2 < k; k2++) {
                    if (first[k] && first[k2] && mb[k2] == mb[k]) {
                        q[k2] += q[k];
                        first[k] = false;
                    }
                }
                single = single && !first[k];
            }
            const unsigned live_mask = __ballot_sync (0xffffffffu, live);
            if (live) {
                // fixed histogram: one count per voxel
                unsigned peers = __match_any_sync (live_mask, fb);
                if (lane == __ffs (peers) - 1) {
                    atomicAdd (&hf[fb], (unsigned long long) __popc (peers));
                }
                cnt++;
            }
            const unsigned single_mask = __ballot_sync (0xffffffffu,
                live && single);
            if (live && single) {
                const int key = fb * B + mb[0];
                unsigned peers = __match_any_sync (single_mask, key);
                unsigned sum = __reduce_add_sync (peers, q[0]);
                if (lane == __ffs (peers) - 1) {
                    atomicAdd (&hm[mb[0]], (unsigned long long) sum);
                    atomicAdd (&hj[key], (unsigned long long) sum);
                }
            } else if (live) {
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    if (first[k]) {
                        atomicAdd (&hm[mb[k]], (unsigned long long) q[k]);
                        atomicAdd (&hj[fb * B + mb[k]], (unsigned long long) q[k]);
                    }
                }
            }
        }
        __syncthreads ();
    }
    for (int i = threadIdx.x; i < nh; i += MIH_THREADS) {
        if (hsm[i]) atomicAdd (&ghist[i], hsm[i]);
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync (0xffffffffu, cnt, o);
    if (lane == 0 && cnt) atomicAdd (&ghist[nh], (unsigned long long) cnt);
}

// ---- Parzen windows: pass 1 ----------------------------------------------------
//
// Mattes MI with cubic B-spline Parzen windows (Mattes et al., IEEE TMI
// 22(1) 2003): each inside voxel adds the cubic window's four weights at
// its moving value to the joint histogram row of its fixed bin (integers in
// 2^-24 units, order-independent sums); lanes whose (fixed bin, first
// window bin) agree combine across the warp first.  Marginals are the joint
// histogram's sums (taken by the score kernel).

__device__ __forceinline__ void
parzen_hist_add (unsigned long long* hj, int B, bool live, int fb, float u,
    int lane, int& cnt)
{
    const int k0 = parzen_first_bin (u, B);
    unsigned int q[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        q[j] = __float2uint_rn (bspline3f ((float) (k0 + j) - u) * MI_WUNIT);
    }
    const unsigned live_mask = __ballot_sync (0xffffffffu, live);
    if (live) {
        cnt++;
        const int key = fb * B + k0;
        const unsigned peers = __match_any_sync (live_mask, key);
        unsigned sum[4];
#pragma unroll
        for (int j = 0; j < 4; j++) sum[j] = __reduce_add_sync (peers, q[j]);
        if (lane == __ffs (peers) - 1) {
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (sum[j]) atomicAdd (&hj[key + j], (unsigned long long) sum[j]);
            }
        }
    }
}

__global__ void __launch_bounds__ (MIH_THREADS)
parzen_hist_kernel (BspGeom g, const float* __restrict__ coeff,
    const float* __restrict__ luts, const uint8_t* __restrict__ fbin,
    const float* __restrict__ mimg, int B, float m_min, float m_delta,
    unsigned long long* __restrict__ ghist)
{
    extern __shared__ unsigned long long hsm[];   // j[B*B]
    __shared__ float sC[192];
    __shared__ float slut[4 * 3 * 64];
    const int vx = g.vpr[0], vy = g.vpr[1], vz = g.vpr[2];
    const int V = vx * vy * vz;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < B * B; i += MIH_THREADS) hsm[i] = 0ull;
    for (int o = threadIdx.x; o < 4 * (vx + vy + vz); o += MIH_THREADS) {
        slut[o] = luts[o];
    }
    const float* sbx = slut;
    const float* sby = slut + 4 * vx;
    const float* sbz = sby + 4 * vy;
    const int dx = g.mdim[0], dxy = g.mdim[0] * g.mdim[1];
    int cnt = 0;
    __syncthreads ();
    for (int t = blockIdx.x; t < g.ntiles; t += gridDim.x) {
        const int tx = t % g.rdims[0];
        const int ty = (t / g.rdims[0]) % g.rdims[1];
        const int tz = t / (g.rdims[0] * g.rdims[1]);
        for (int o = threadIdx.x; o < 192; o += MIH_THREADS) {
            int m = o / 3, c = o - 3 * m;
            int i = m & 3, j = (m >> 2) & 3, k = m >> 4;
            sC[o] = coeff[3 * ((tz + k) * g.cdims[1] * g.cdims[0]
                + (ty + j) * g.cdims[0] + (tx + i)) + c];
        }
        __syncthreads ();
        // warp-uniform trip count: every lane reaches the warp collectives
        for (int v0 = 32 * warp; v0 < V; v0 += MIH_THREADS) {
            const int v = v0 + lane;
            const int vv = v < V ? v : 0;
            int lx = vv % vx, ly = (vv / vx) % vy, lz = vv / (vx * vy);
            int fi = g.roi_off[0] + vx * tx + lx;
            int fj = g.roi_off[1] + vy * ty + ly;
            int fk = g.roi_off[2] + vz * tz + lz;
            bool live = v < V && fi < g.roi_off[0] + g.roi_dim[0]
                && fj < g.roi_off[1] + g.roi_dim[1]
                && fk < g.roi_off[2] + g.roi_dim[2];
            int fb = 0;
            float u = 2.f;
            live = live && roi_fixed_ok (g, fi + g.fdim[0] * (fj + g.fdim[1] * fk));
            if (live) {
                float fxyz[3], d[3] = {0.f, 0.f, 0.f};
                fixed_position (g, fi, fj, fk, fxyz);
                int m = 0;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    float C = sbz[lz * 4 + k];
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        float Bv = sby[ly * 4 + j] * C;
#pragma unroll
                        for (int i = 0; i < 4; i++, m++) {
                            float A = sbx[lx * 4 + i] * Bv;
                            d[0] += A * sC[3 * m + 0];
                            d[1] += A * sC[3 * m + 1];
                            d[2] += A * sC[3 * m + 2];
                        }
                    }
                }
                Sample s;
                live = locate (g, fxyz, d, s) && roi_moving_ok (g, fxyz, d);
                if (live) {
                    const Corners cr = load_corners (mimg, s.mvf, dx, dxy);
                    u = parzen_centre (trilinear (s, cr), m_min, m_delta);
                    fb = fbin[fi + g.fdim[0] * (fj + g.fdim[1] * fk)];
                }
            }
            parzen_hist_add (hsm, B, live, fb, u, lane, cnt);
        }
        __syncthreads ();
    }
    const int nh = 2 * B + B * B;
    for (int i = threadIdx.x; i < B * B; i += MIH_THREADS) {
        if (hsm[i]) atomicAdd (&ghist[2 * B + i], hsm[i]);
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync (0xffffffffu, cnt, o);
    if (lane == 0 && cnt) atomicAdd (&ghist[nh], (unsigned long long) cnt);
}

// Score and pass-2 table: p = joint / N (weights in 2^-24 units), p_f and
// p_m its row and column sums, S = -sum p log(p / (p_f p_m)) (terms with
// p = 0 drop out), the factor log(p / p_m) per joint bin, and
// 1 / (N delta_m) for pass 2.  Marginals and joint go to histd as weights.
__global__ void __launch_bounds__ (1024)
parzen_score_kernel (const unsigned long long* __restrict__ ghist, int B,
    float m_delta, double* __restrict__ histd, float* __restrict__ lut,
    float* __restrict__ nvf, DevResult* __restrict__ res)
{
    __shared__ double sh_v[32];
    __shared__ int sh_n[32];
    __shared__ double s_pf[MI_MAX_BINS], s_pm[MI_MAX_BINS];
    const int nh = 2 * B + B * B;
    const long long N = (long long) ghist[nh];
    const double* j = histd + 2 * B;
    for (int i = threadIdx.x; i < B * B; i += blockDim.x) {
        histd[2 * B + i] = (double) ghist[2 * B + i] * MI_WUNIT_INV;
    }
    __syncthreads ();
    for (int i = threadIdx.x; i < 2 * B; i += blockDim.x) {
        double v = 0.0;
        if (i < B) {
            for (int k = 0; k < B; k++) v += j[i * B + k];
            s_pf[i] = v;
        } else {
            for (int r = 0; r < B; r++) v += j[r * B + (i - B)];
            s_pm[i - B] = v;
        }
        histd[i] = v;
    }
    __syncthreads ();
    const double fnv = (double) N;
    double acc = 0.0;
    for (int jb = threadIdx.x; jb < B * B; jb += blockDim.x) {
        const int fb = jb / B, mb = jb - fb * B;
        const double pj = j[jb] / fnv;
        float f = 0.f;
        if (N > 0 && pj > 0.0) {
            const double pm = s_pm[mb] / fnv, pf = s_pf[fb] / fnv;
            acc -= pj * log (pj / (pf * pm));
            f = (float) log (pj / pm);
        }
        lut[jb] = f;
    }
    int dummy = 0;
    block_sum<1024> (acc, dummy, sh_v, sh_n);
    if (threadIdx.x == 0) {
        res->raw = acc;
        res->score = N > 0 ? acc : (double) FLT_MAX;
        res->score_f = N > 0 ? (float) acc : FLT_MAX;
        res->num_vox = N;
        res->error = 0;
        nvf[0] = (float) N;
        nvf[1] = N > 0 ? (float) (1.0 / (fnv * (double) m_delta)) : 0.f;
    }
}

// Pass 2 on the FP32 tile kernel: dc/dv = 1/(N delta_m) * sum over the
// window's bins of beta3'(k - u) log(p(f, k) / p_m(k)) times the world
// gradient of the trilinear interpolant (proj^T times the index gradient).
struct ParzenGradVoxel {
    static constexpr bool kNeedCorners = true;
    const uint8_t* fbin;
    const float* lut;
    const float* nvf;
    int B;
    float m_min, m_delta;
    __device__ __forceinline__ bool
    voxel (const BspGeom& g, int fidx, const Sample& s, const Corners& cr,
        float dc[3], double&) const
    {
        const float u = parzen_centre (trilinear (s, cr), m_min, m_delta);
        const int k0 = parzen_first_bin (u, B);
        const float* row = lut + (int) __ldg (fbin + fidx) * B;
        float sum = 0.f;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            sum += bspline3f_d ((float) (k0 + j) - u) * __ldg (row + k0 + j);
        }
        float gi[3];
        trilinear_igrad (s.w2, cr.m, s.clamp, gi);
        const float sc = __ldg (nvf + 1) * sum;
        const float* p = g.mproj;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            dc[c] = sc * (p[c] * gi[0] + p[3 + c] * gi[1] + p[6 + c] * gi[2]);
        }
        return true;
    }
};

// ---- score and pass-2 factor table -----------------------------------------

__global__ void __launch_bounds__ (1024)
mi_score_kernel (const unsigned long long* __restrict__ ghist, int B,
    double* __restrict__ histd, float* __restrict__ lut,
    float* __restrict__ nvf, DevResult* __restrict__ res)
{
    __shared__ double sh_v[32];
    __shared__ int sh_n[32];
    __shared__ float s_score;
    const int nh = 2 * B + B * B;
    for (int i = threadIdx.x; i < nh; i += blockDim.x) {
        histd[i] = i < B ? (double) ghist[i]
                         : (double) ghist[i] * MI_WUNIT_INV;
    }
    __syncthreads ();
    const long long N = (long long) ghist[nh];
    const double fnv = (double) N;
    const double thresh = 0.001 / (B * B);
    const double* f = histd;
    const double* m = histd + B;
    const double* j = histd + 2 * B;
    double acc = 0.0;
    for (int jb = threadIdx.x; jb < B * B; jb += blockDim.x) {
        int mb = jb % B, fb = jb / B;
        if (j[jb] > thresh) {
            acc -= j[jb] * (double) logf ((float) (fnv * j[jb] / (m[mb] * f[fb])));
        }
    }
    int dummy = 0;
    block_sum<1024> (acc, dummy, sh_v, sh_n);
    if (threadIdx.x == 0) {
        double S = N > 0 ? acc / fnv : (double) FLT_MAX;
        res->raw = acc;
        res->score = S;
        res->score_f = N > 0 ? (float) S : FLT_MAX;
        res->num_vox = N;
        res->error = 0;
        s_score = res->score_f;
        *nvf = (float) N;
    }
    __syncthreads ();
    const float num_vox_f = (float) N;
    for (int jb = threadIdx.x; jb < B * B; jb += blockDim.x) {
        int mb = jb % B, fb = jb / B;
        float val = 0.f;
        if (N > 0 && j[jb] > 0.0001) {
            val = logf ((float) (((double) num_vox_f * j[jb]) / (f[fb] * m[mb])))
                - s_score;
        }
        lut[jb] = val;
    }
}

// ---- pass 2: gradient --------------------------------------------------------

struct MiGradVoxel {
    static constexpr bool kNeedCorners = false;
    const uint8_t* fbin;
    const uint8_t* mbin;
    const float* lut;
    const float* nvf;
    int B;
    __device__ __forceinline__ bool
    voxel (const BspGeom& g, int fidx, const Sample& s, const Corners&,
        float dc[3], double&) const
    {
        const float* l1 = s.w1;
        const float* l2 = s.w2;
        // derivative of each corner weight along x, y, z (reference order)
        const float dw[24] = {
            (-1) * l1[1] * l1[2], l1[0] * (-1) * l1[2], l1[0] * l1[1] * (-1),
            (+1) * l1[1] * l1[2], l2[0] * (-1) * l1[2], l2[0] * l1[1] * (-1),
            (-1) * l2[1] * l1[2], l1[0] * (+1) * l1[2], l1[0] * l2[1] * (-1),
            (+1) * l2[1] * l1[2], l2[0] * (+1) * l1[2], l2[0] * l2[1] * (-1),
            (-1) * l1[1] * l2[2], l1[0] * (-1) * l2[2], l1[0] * l1[1] * (+1),
            (+1) * l1[1] * l2[2], l2[0] * (-1) * l2[2], l2[0] * l1[1] * (+1),
            (-1) * l2[1] * l2[2], l1[0] * (+1) * l2[2], l1[0] * l2[1] * (+1),
            (+1) * l2[1] * l2[2], l2[0] * (+1) * l2[2], l2[0] * l2[1] * (+1)};
        const int dx = g.mdim[0], dxy = g.mdim[0] * g.mdim[1];
        const int nbr[8] = {s.mvf, s.mvf + 1, s.mvf + dx, s.mvf + dx + 1,
            s.mvf + dxy, s.mvf + dxy + 1, s.mvf + dxy + dx,
            s.mvf + dxy + dx + 1};
        const int off = (int) __ldg (fbin + fidx) * B;
        float d0 = 0.f, d1 = 0.f, d2 = 0.f;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            float f = __ldg (lut + off + __ldg (mbin + nbr[k]));
            d0 -= dw[3 * k + 0] * f;
            d1 -= dw[3 * k + 1] * f;
            d2 -= dw[3 * k + 2] * f;
        }
        const float nv = *nvf;
        d0 = d0 / nv;
        d1 = d1 / nv;
        d2 = d2 / nv;
        // the reference projects in place: each row sees the updated rows above
        const float* p = g.mproj;
        d0 = d0 * p[0] + d1 * p[1] + d2 * p[2];
        d1 = d0 * p[3] + d1 * p[4] + d2 * p[5];
        d2 = d0 * p[6] + d1 * p[7] + d2 * p[8];
        dc[0] = d0;
        dc[1] = d1;
        dc[2] = d2;
        return true;
    }
};

int
mi_run (MiState* s, const BspGeom& g, const float* d_coeff,
    const float* d_moving, const float* d_luts, DevResult* d_res,
    float* grad_out, double* grad64_out, cudaStream_t st, int* launches,
    int passes)
{
    if (!s->ready) return B200BSP_E_STATE;
    const int B = s->bins;
    const int nh = 2 * B + B * B;
    if ((passes & MI_PASS_HIST)
        && cudaMemsetAsync (s->d_hist, 0, (nh + 1) * sizeof (unsigned long long),
            st) != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    int sms = 148;
    cudaDeviceGetAttribute (&sms, cudaDevAttrMultiProcessorCount, 0);
    PartLayout lay;
    lay.bx = lay.by = lay.bz = 1;
    lay.nbx = g.rdims[0]; lay.nby = g.rdims[1]; lay.nbz = g.rdims[2];
    lay.kx = lay.ky = lay.kz = 4;
    lay.slots = 64;
    if (s->window == B200BSP_MI_PARZEN) {
        const int grid = std::min (g.ntiles, 8 * sms);
        if (passes & MI_PASS_HIST) {
            parzen_hist_kernel<<<grid, MIH_THREADS,
                (size_t) B * B * sizeof (unsigned long long), st>>> (g,
                d_coeff, d_luts, s->d_fbin, d_moving, B, s->pz_mmin,
                s->pz_mdelta, s->d_hist);
        }
        if (!(passes & MI_PASS_GRAD)) {
            return cudaGetLastError () == cudaSuccess ? B200BSP_OK : B200BSP_E_CUDA;
        }
        parzen_score_kernel<<<1, 1024, 0, st>>> (s->d_hist, B, s->pz_mdelta,
            s->d_histd, s->d_lut, s->d_nvf, d_res);
        ParzenGradVoxel f{s->d_fbin, s->d_lut, s->d_nvf, B, s->pz_mmin,
            s->pz_mdelta};
        if (launch_fp32_tile (g, f, d_moving, d_coeff, d_luts, s->d_part,
                s->d_score_part, s->d_count_part, st) != cudaSuccess
            || launch_gather_grad (g, lay, s->d_part, d_res, 1, grad_out,
                grad64_out, nullptr, nullptr, nullptr, st) != cudaSuccess) {
            return B200BSP_E_CUDA;
        }
        if (launches) *launches += 4;
        return cudaGetLastError () == cudaSuccess ? B200BSP_OK : B200BSP_E_CUDA;
    }
    size_t hsmem = (size_t) nh * sizeof (unsigned long long);
    auto hk = mi_hist_kernel;
    if (hsmem > 48 * 1024
        && set_max_dynamic_smem ((const void*) hk, (int) hsmem) != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    int grid = std::min (g.ntiles, 8 * sms);
    if (passes & MI_PASS_HIST) {
        hk<<<grid, MIH_THREADS, hsmem, st>>> (g, d_coeff, d_luts, s->d_fbin,
            s->d_mbin, B, s->d_hist);
    }
    if (!(passes & MI_PASS_GRAD)) {
        return cudaGetLastError () == cudaSuccess ? B200BSP_OK : B200BSP_E_CUDA;
    }
    mi_score_kernel<<<1, 1024, 0, st>>> (s->d_hist, B, s->d_histd, s->d_lut,
        s->d_nvf, d_res);
    MiGradVoxel f{s->d_fbin, s->d_mbin, s->d_lut, s->d_nvf, B};
    if (launch_fp32_tile (g, f, nullptr, d_coeff, d_luts, s->d_part,
            s->d_score_part, s->d_count_part, st) != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    if (launch_gather_grad (g, lay, s->d_part, d_res, 1, grad_out, grad64_out,
            nullptr, nullptr, nullptr, st) != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    if (launches) *launches += 4;
    return cudaGetLastError () == cudaSuccess ? B200BSP_OK : B200BSP_E_CUDA;
}

// The same two passes on the tensor-core kernel (field and adjoint as
// GEMMs; the histograms in the same integer units, so pass 1 agrees with
// mi_run's up to the field's rounding); the caller has checked
// tc_mi_supported.
int
mi_run_tc (MiState* s, const BspGeom& g, const TcPlan& plan,
    const PartLayout& lay, const void* qlut, float* part, double* score_part,
    int* count_part, int* err, const float* d_coeff, const float* d_moving,
    DevResult* d_res, float* grad_out, double* grad64_out, cudaStream_t st,
    int* launches, int passes)
{
    if (!s->ready) return B200BSP_E_STATE;
    const int B = s->bins;
    const int nh = 2 * B + B * B;
    if ((passes & MI_PASS_HIST)
        && cudaMemsetAsync (s->d_hist, 0, (nh + 1) * sizeof (unsigned long long),
            st) != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    TcMiArgs mi;
    mi.fbin = s->d_fbin;
    mi.mbin = s->d_mbin;
    mi.bins = B;
    mi.lut = s->d_lut;
    mi.nvf = s->d_nvf;
    mi.hist = s->d_hist;
    mi.parzen = s->window == B200BSP_MI_PARZEN;
    mi.mimg = d_moving;
    mi.m_min = s->pz_mmin;
    mi.m_delta = s->pz_mdelta;
    if ((passes & MI_PASS_HIST)
        && launch_mi_tc (g, plan, true, mi, d_coeff, qlut, part, score_part,
            count_part, err, st) != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    if (!(passes & MI_PASS_GRAD)) {
        return cudaGetLastError () == cudaSuccess ? B200BSP_OK : B200BSP_E_CUDA;
    }
    if (mi.parzen) {
        parzen_score_kernel<<<1, 1024, 0, st>>> (s->d_hist, B, s->pz_mdelta,
            s->d_histd, s->d_lut, s->d_nvf, d_res);
    } else {
        mi_score_kernel<<<1, 1024, 0, st>>> (s->d_hist, B, s->d_histd,
            s->d_lut, s->d_nvf, d_res);
    }
    if (launch_mi_tc (g, plan, false, mi, d_coeff, qlut, part, score_part,
            count_part, err, st) != cudaSuccess
        || launch_gather_grad (g, lay, part, d_res, 1, grad_out, grad64_out,
            nullptr, nullptr, nullptr, st) != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    if (launches) *launches += 4;
    return cudaGetLastError () == cudaSuccess ? B200BSP_OK : B200BSP_E_CUDA;
}

// The two passes on the x-lane tensor-core kernel (any geometry; tiles
// with 3 <= vox_per_rgn[1] <= 10); the caller has checked
// xl_mi_supported.
int
mi_run_xl (MiState* s, const BspGeom& g, const XlPlan& plan,
    const PartLayout& lay, const void* tab, const float* luts, float* part,
    int* err, unsigned wait_limit, const float* d_coeff,
    const float* d_moving, DevResult* d_res, float* grad_out,
    double* grad64_out, cudaStream_t st, int* launches, int passes)
{
    if (!s->ready) return B200BSP_E_STATE;
    const int B = s->bins;
    const int nh = 2 * B + B * B;
    if ((passes & MI_PASS_HIST)
        && cudaMemsetAsync (s->d_hist, 0, (nh + 1) * sizeof (unsigned long long),
            st) != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    TcMiArgs mi;
    mi.fbin = s->d_fbin;
    mi.mbin = s->d_mbin;
    mi.bins = B;
    mi.lut = s->d_lut;
    mi.nvf = s->d_nvf;
    mi.hist = s->d_hist;
    mi.parzen = s->window == B200BSP_MI_PARZEN;
    mi.mimg = d_moving;
    mi.m_min = s->pz_mmin;
    mi.m_delta = s->pz_mdelta;
    if ((passes & MI_PASS_HIST)
        && launch_mi_xl (g, plan, true, mi, d_coeff, tab, luts, part, err,
            wait_limit, st) != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    if (!(passes & MI_PASS_GRAD)) {
        if (launches) *launches += 1;
        return cudaGetLastError () == cudaSuccess ? B200BSP_OK : B200BSP_E_CUDA;
    }
    if (mi.parzen) {
        parzen_score_kernel<<<1, 1024, 0, st>>> (s->d_hist, B, s->pz_mdelta,
            s->d_histd, s->d_lut, s->d_nvf, d_res);
    } else {
        mi_score_kernel<<<1, 1024, 0, st>>> (s->d_hist, B, s->d_histd,
            s->d_lut, s->d_nvf, d_res);
    }
    if (launch_mi_xl (g, plan, false, mi, d_coeff, tab, luts, part, err,
            wait_limit, st) != cudaSuccess
        || launch_gather_grad (g, lay, part, d_res, 1, grad_out, grad64_out,
            nullptr, nullptr, nullptr, st) != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    if (launches) *launches += 4;
    return cudaGetLastError () == cudaSuccess ? B200BSP_OK : B200BSP_E_CUDA;
}

int
mi_fetch (MiState* s, const DevResult* d_res, double* f_hist, double* m_hist,
    double* j_hist, cudaStream_t st)
{
    const int B = s->bins;
    const int nh = 2 * B + B * B;
    if (cudaMemcpyAsync (s->h_res, d_res, sizeof (DevResult),
            cudaMemcpyDeviceToHost, st) != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    if (f_hist || m_hist || j_hist) {
        if (cudaMemcpyAsync (s->h_histd, s->d_histd, nh * sizeof (double),
                cudaMemcpyDeviceToHost, st) != cudaSuccess
            || cudaStreamSynchronize (st) != cudaSuccess) {
            return B200BSP_E_CUDA;
        }
        if (f_hist) memcpy (f_hist, s->h_histd, B * sizeof (double));
        if (m_hist) memcpy (m_hist, s->h_histd + B, B * sizeof (double));
        if (j_hist) memcpy (j_hist, s->h_histd + 2 * B, B * B * sizeof (double));
    }
    return B200BSP_OK;
}

void
mi_finish (MiState* s, MiResult* r)
{
    r->score_f = s->h_res->score_f;
    r->score = s->h_res->score;
    r->num_vox = s->h_res->num_vox;
}

} // namespace b200
