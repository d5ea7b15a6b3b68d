// Analytic regulariser (Plastimatch src/register/
// bspline_regularize_analytic.cxx:166-337 and 637-1059, implementation 'c'):
// S = sum over tiles and terms of c^T V c with 32 weighted 64x64 matrices V
// per tile, and dS/dc condensed per knot.
//
// Every V is a Kronecker product X (x) Y (x) Z of three 4x4 one-dimensional
// integrals (get_Vmatrix, :282-337): X, built from grid spacing 0, acts on
// the tile's z knot digit, Y on the y digit and Z, built from grid
// spacing 2, on the x digit.  The tiles form a full Cartesian product, so
// the sum of the tile operators over the grid is again a Kronecker product
// of three banded (7-diagonal) knot-axis operators.  The device applies
// those separably instead of forming 64x64 matrices per tile:
//   pass 1  knot-x bands applied to each coefficient component
//   pass 2  knot-y bands applied to the pass-1 fields
//   pass 3  weighted knot-z bands, summed into the nine outputs below; the
//           gradient and the per-knot score follow, and the score is
//           reduced per block, then over the blocks by the last block to
//           finish, in a fixed order.
// Outputs of pass 3 (input component in brackets):
//   Dx[x] Dy[y] Dz[z]   same-component terms: V0..V8, V21..V31 on every
//                       component, V15..V20 on the components the elastic
//                       group gives them (region_smoothness_elastic_omp,
//                       :516-600)
//   Cxy[x] Cxz[x] Cyx[y] Cyz[y] Czx[z] Czy[z]   the elastic cross terms
//                       (V9+V10, V11+V12, V13+V14)
//   grad_x = 2 Dx + Cyx + Czx, grad_y = 2 Dy + Cxy + Czy,
//   grad_z = 2 Dz + Cxz + Cyz,
//   S = sum over knots of cx Dx + cy Dy + cz Dz + cy Cxy + cz Cxz + cz Cyz.
// All arithmetic is double; the gradient is added into the float gradient
// once per knot component.
#include <algorithm>
#include <cstring>
#include <map>

#include "kernels.cuh"
#include "regularize.cuh"

namespace b200 {

constexpr int REG_THREADS = 256;

// ---- one-dimensional integrals (host, double) ---------------------------------

// Uniform cubic B-spline pieces in power form: row j holds the coefficients
// of 1, u, u^2, u^3 of the basis function that weights knot j of a tile.
static const double BSPL[16] = {
    1.0 / 6.0, -1.0 / 2.0, 1.0 / 2.0, -1.0 / 6.0,
    2.0 / 3.0, 0.0, -1.0, 1.0 / 2.0,
    1.0 / 6.0, 1.0 / 2.0, 1.0 / 2.0, -1.0 / 2.0,
    0.0, 0.0, 0.0, 1.0 / 6.0};

// Polynomial coefficients of derivative `order` of the four pieces, in the
// physical coordinate (u / grid spacing).
static void
pieces (double out[16], double gs, int order)
{
    double r = 1.0 / gs;
    double scale[4] = {1.0, r, r * r, r * r * r};
    for (int j = 0; j < 4; j++) {
        for (int p = 0; p < 4; p++) {
            // d^order/dx^order of x^p = p!/(p-order)! x^(p-order)
            double v = 0.0;
            int q = p - order;                 // resulting power
            if (q >= 0) {
                double f = 1.0;
                for (int m = p; m > q; m--) f *= m;
                v = BSPL[4 * j + p] * scale[p] * f;
            }
            // stored at the power it multiplies after differentiation
            if (q >= 0) out[4 * j + q] = v;
        }
        for (int q = 4 - order; q < 4; q++) out[4 * j + q] = 0.0;
    }
}

// F[j][i] = integral over [0, gs] of piece_j^(p) * piece_i^(q).
static void
integral (double F[16], const double P[16], const double Qm[16], double gs)
{
    double I[7];
    double g = gs;
    for (int n = 0; n < 7; n++) {
        I[n] = g / (n + 1);
        g *= gs;
    }
    for (int j = 0; j < 4; j++) {
        for (int i = 0; i < 4; i++) {
            double s = 0.0;
            for (int a = 0; a < 4; a++) {
                for (int b = 0; b < 4; b++) {
                    s += P[4 * j + a] * Qm[4 * i + b] * I[a + b];
                }
            }
            F[4 * j + i] = s;
        }
    }
}

// Derivative-order pairs (row, column) of the factors the 32 terms use.
static const int PAIRS[6][2] = {{0, 0}, {1, 1}, {2, 2}, {3, 3}, {1, 0}, {0, 1}};

static int
pair_index (int a, int b)
{
    for (int k = 0; k < 6; k++) {
        if (PAIRS[k][0] == a && PAIRS[k][1] == b) return k;
    }
    return -1;
}

// Banded knot-axis operator: sum over tiles t of F[k - t][k' - t]; stored as
// band[k][d + 3] = G[k][k + d].
static void
assemble (double* band, const double F[16], int n, int ntiles)
{
    for (int k = 0; k < n; k++) {
        for (int d = -3; d <= 3; d++) {
            double s = 0.0;
            int k2 = k + d;
            if (k2 >= 0 && k2 < n) {
                int t0 = std::max (0, std::max (k - 3, k2 - 3));
                int t1 = std::min (ntiles - 1, std::min (k, k2));
                for (int t = t0; t <= t1; t++) s += F[4 * (k - t) + (k2 - t)];
            }
            band[7 * k + d + 3] = s;
        }
    }
}

// The 32 terms of analytic_init (:637-940): derivative orders of the X
// (knot z), Y (knot y) and Z (knot x) factors and the weight selector.
struct RegTerm { int xa, xb, ya, yb, za, zb, w; };
static const RegTerm TERMS[32] = {
    {2, 2, 0, 0, 0, 0, 0}, {0, 0, 2, 2, 0, 0, 0}, {0, 0, 0, 0, 2, 2, 0},
    {1, 1, 1, 1, 0, 0, 1}, {1, 1, 0, 0, 1, 1, 1}, {0, 0, 1, 1, 1, 1, 1},
    {1, 1, 0, 0, 0, 0, 2}, {0, 0, 1, 1, 0, 0, 2}, {0, 0, 0, 0, 1, 1, 2},
    {1, 0, 0, 1, 0, 0, 3}, {0, 1, 1, 0, 0, 0, 4}, {1, 0, 0, 0, 0, 1, 3},
    {0, 1, 0, 0, 1, 0, 4}, {0, 0, 1, 0, 0, 1, 3}, {0, 0, 0, 1, 1, 0, 4},
    {1, 1, 0, 0, 0, 0, 5}, {0, 0, 1, 1, 0, 0, 5}, {0, 0, 0, 0, 1, 1, 5},
    {1, 1, 0, 0, 0, 0, 6}, {0, 0, 1, 1, 0, 0, 6}, {0, 0, 0, 0, 1, 1, 6},
    {0, 0, 0, 0, 0, 0, 7},
    {3, 3, 0, 0, 0, 0, 8}, {0, 0, 3, 3, 0, 0, 8}, {0, 0, 0, 0, 3, 3, 8},
    {2, 2, 1, 1, 0, 0, 8}, {2, 2, 0, 0, 1, 1, 8}, {0, 0, 2, 2, 1, 1, 8},
    {1, 1, 2, 2, 0, 0, 8}, {1, 1, 0, 0, 2, 2, 8}, {0, 0, 1, 1, 2, 2, 8},
    {1, 1, 1, 1, 1, 1, 8},
};

// Term weights, in float arithmetic as the reference scales its V matrices.
static float
term_weight (int sel, const b200bsp_reg_parms* p)
{
    float lem = p->linear_elastic_multiplier;
    switch (sel) {
    case 0: return p->curvature_penalty;
    case 1: return p->curvature_penalty * p->curvature_mixed_weight;
    case 2: return p->diffusion_penalty;
    case 3: return p->lame_coefficient_1 * lem;
    case 4: return p->lame_coefficient_2 * lem;
    case 5: return lem * (2 * p->lame_coefficient_1 + p->lame_coefficient_2) / 2;
    case 6: return lem * (p->lame_coefficient_1) / 2;
    case 7: return p->total_displacement_penalty;
    case 8: return p->third_order_penalty;
    }
    return 0.f;
}

// Outputs of pass 3 and the coefficient component each one reads.
enum { O_DX, O_DY, O_DZ, O_CXY, O_CXZ, O_CYX, O_CYZ, O_CZX, O_CZY, O_N };
static const int OUT_COMP[O_N] = {0, 1, 2, 0, 0, 1, 1, 2, 2};

// Which outputs term t feeds.
static int
term_outputs (int t, int out[3])
{
    if (t <= 8 || t >= 21) {
        out[0] = O_DX; out[1] = O_DY; out[2] = O_DZ;
        return 3;
    }
    switch (t) {
    case 9: case 10: out[0] = O_CXY; out[1] = O_CYX; return 2;
    case 11: case 12: out[0] = O_CXZ; out[1] = O_CZX; return 2;
    case 13: case 14: out[0] = O_CYZ; out[1] = O_CZY; return 2;
    case 15: out[0] = O_DX; return 1;
    case 16: out[0] = O_DY; return 1;
    case 17: out[0] = O_DZ; return 1;
    case 18: out[0] = O_DY; out[1] = O_DZ; return 2;
    case 19: out[0] = O_DX; out[1] = O_DZ; return 2;
    case 20: out[0] = O_DX; out[1] = O_DY; return 2;
    }
    return 0;
}

// ---- device passes ----------------------------------------------------------
//
// Each block covers 32 knots along x times REG_TY knots along the pass's
// axis (256 threads: x fastest).  The pass's input fields over the block's
// knots and a halo of 3 on either side of that axis are staged in shared
// memory once, so the 7-tap stencils read each value from L2 once instead
// of seven times.  Taps outside the grid read zeros (the reference's sums
// skip them; adding a zero product leaves every sum unchanged).

constexpr int REG_TY = 8;                    // knots along the pass axis
constexpr int REG_TH = REG_TY + 6;           // with the halo

__global__ void __launch_bounds__ (REG_THREADS)
reg_pass_x (RegPlan plan, int cx, int cy, int nk, const double* __restrict__ gx,
    const float* __restrict__ coeff, double* __restrict__ t1)
{
    // block: knots kx0 .. kx0 + 31 (+ 3 either side) of rows ky0 .. ky0 + 7
    __shared__ float sc[3][REG_TY][32 + 6];
    __shared__ double sb[6][32][7];          // the six x bands of the block
    const int kx0 = blockIdx.x * 32, ky0 = blockIdx.y * REG_TY;
    const int kz = blockIdx.z;
    for (int i = threadIdx.x; i < 3 * REG_TY * 38; i += REG_THREADS) {
        const int c = i / (REG_TY * 38), r = (i / 38) % REG_TY, j = i % 38;
        const int kx = kx0 - 3 + j, ky = ky0 + r;
        sc[c][r][j] = kx >= 0 && kx < cx && ky < cy
            ? coeff[3 * (kx + cx * (ky + cy * kz)) + c] : 0.f;
    }
    for (int i = threadIdx.x; i < 6 * 32 * 7; i += REG_THREADS) {
        const int f = i / (32 * 7), j = i % (32 * 7);
        (&sb[0][0][0])[i] = kx0 + j / 7 < cx
            ? gx[((size_t) f * cx + kx0) * 7 + j] : 0.0;
    }
    __syncthreads ();
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int kx = kx0 + tx, ky = ky0 + ty;
    if (kx >= cx || ky >= cy) return;
    const int knot = kx + cx * (ky + cy * kz);
    for (int s = 0; s < plan.n1; s++) {
        const int c = plan.t1_c[s];
        const double* band = sb[plan.t1_xf[s]][tx];
        double acc = 0.0;
#pragma unroll
        for (int d = -3; d <= 3; d++) {
            acc += band[d + 3] * (double) sc[c][ty][tx + 3 + d];
        }
        t1[(size_t) s * nk + knot] = acc;
    }
}

__global__ void __launch_bounds__ (REG_THREADS)
reg_pass_y (RegPlan plan, int cx, int cy, int nk,
    const double* __restrict__ gy, const double* __restrict__ t1,
    double* __restrict__ t2)
{
    // block: knots kx0 .. kx0 + 31 of rows ky0 - 3 .. ky0 + 10, every
    // pass-1 field
    extern __shared__ double st[];           // [n1][REG_TH][32]
    __shared__ double sb[6][REG_TY][7];      // the six y bands of the block
    const int kx0 = blockIdx.x * 32, ky0 = blockIdx.y * REG_TY;
    const int kz = blockIdx.z;
    for (int i = threadIdx.x; i < plan.n1 * REG_TH * 32; i += REG_THREADS) {
        const int s = i / (REG_TH * 32), r = (i / 32) % REG_TH, j = i % 32;
        const int kx = kx0 + j, ky = ky0 - 3 + r;
        st[i] = kx < cx && ky >= 0 && ky < cy
            ? t1[(size_t) s * nk + kx + cx * (ky + cy * kz)] : 0.0;
    }
    for (int i = threadIdx.x; i < 6 * REG_TY * 7; i += REG_THREADS) {
        const int f = i / (REG_TY * 7), j = i % (REG_TY * 7);
        (&sb[0][0][0])[i] = ky0 + j / 7 < cy
            ? gy[((size_t) f * cy + ky0) * 7 + j] : 0.0;
    }
    __syncthreads ();
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int kx = kx0 + tx, ky = ky0 + ty;
    if (kx >= cx || ky >= cy) return;
    const int knot = kx + cx * (ky + cy * kz);
    for (int s = 0; s < plan.n2; s++) {
        const double* src = st + plan.t2_src[s] * (REG_TH * 32) + tx;
        const double* band = sb[plan.t2_yf[s]][ty];
        double acc = 0.0;
#pragma unroll
        for (int d = -3; d <= 3; d++) {
            acc += band[d + 3] * src[(ty + 3 + d) * 32];
        }
        t2[(size_t) s * nk + knot] = acc;
    }
}

__global__ void __launch_bounds__ (REG_THREADS)
reg_pass_z (RegPlan plan, int cx, int cy, int cz, int nk,
    const double* __restrict__ hz, const double* __restrict__ t2,
    const float* __restrict__ coeff, float* __restrict__ grad,
    double* __restrict__ grad64, double* __restrict__ part,
    unsigned* __restrict__ arrive, double* __restrict__ score)
{
    // block: knots kx0 .. kx0 + 31 of row ky, planes kz0 - 3 .. kz0 + 10,
    // every pass-2 field
    // [n2][REG_TH][32] pass-2 fields, then [ne][REG_TY][7] z bands
    extern __shared__ double st[];
    __shared__ double sh_v[REG_THREADS / 32];
    __shared__ int sh_n[REG_THREADS / 32];
    __shared__ bool s_last;
    const int kx0 = blockIdx.x * 32, ky = blockIdx.y;
    const int kz0 = blockIdx.z * REG_TY;
    const int plane = cx * cy;
    for (int i = threadIdx.x; i < plan.n2 * REG_TH * 32; i += REG_THREADS) {
        const int s = i / (REG_TH * 32), r = (i / 32) % REG_TH, j = i % 32;
        const int kx = kx0 + j, kz = kz0 - 3 + r;
        st[i] = kx < cx && kz >= 0 && kz < cz
            ? t2[(size_t) s * nk + kx + cx * ky + (size_t) plane * kz] : 0.0;
    }
    double* sb = st + plan.n2 * REG_TH * 32;
    for (int i = threadIdx.x; i < plan.ne * REG_TY * 7; i += REG_THREADS) {
        const int e = i / (REG_TY * 7), j = i % (REG_TY * 7);
        sb[i] = kz0 + j / 7 < cz ? hz[((size_t) e * cz + kz0) * 7 + j] : 0.0;
    }
    __syncthreads ();
    const int tx = threadIdx.x & 31, tz = threadIdx.x >> 5;
    const int kx = kx0 + tx, kz = kz0 + tz;
    double S = 0.0;
    if (kx < cx && kz < cz) {
        const int knot = kx + cx * ky + plane * kz;
        // each output sums its entries in the order they were formed
        double out[O_N];
#pragma unroll
        for (int o = 0; o < O_N; o++) {
            double v = 0.0;
            for (int e = plan.e_off[o]; e < plan.e_off[o + 1]; e++) {
                const double* src = st + plan.e_src[e] * (REG_TH * 32) + tx;
                const double* band = sb + (e * REG_TY + tz) * 7;
                double acc = 0.0;
#pragma unroll
                for (int d = -3; d <= 3; d++) {
                    acc += band[d + 3] * src[(tz + 3 + d) * 32];
                }
                v += acc;
            }
            out[o] = v;
        }
        double c0 = coeff[3 * knot + 0], c1 = coeff[3 * knot + 1];
        double c2 = coeff[3 * knot + 2];
        S = c0 * out[O_DX] + c1 * out[O_DY] + c2 * out[O_DZ]
            + c1 * out[O_CXY] + c2 * out[O_CXZ] + c2 * out[O_CYZ];
        const double g0 = 2.0 * out[O_DX] + out[O_CYX] + out[O_CZX];
        const double g1 = 2.0 * out[O_DY] + out[O_CXY] + out[O_CZY];
        const double g2 = 2.0 * out[O_DZ] + out[O_CXZ] + out[O_CYZ];
        if (grad64) {
            // stored for a later kernel to add (b200bsp_score)
            grad64[3 * knot + 0] = g0;
            grad64[3 * knot + 1] = g1;
            grad64[3 * knot + 2] = g2;
        } else if (grad) {
            grad[3 * knot + 0] = (float) ((double) grad[3 * knot + 0] + g0);
            grad[3 * knot + 1] = (float) ((double) grad[3 * knot + 1] + g1);
            grad[3 * knot + 2] = (float) ((double) grad[3 * knot + 2] + g2);
        }
    }
    int dummy = 0;
    block_sum<REG_THREADS> (S, dummy, sh_v, sh_n);
    // the last block to finish sums the block partials in block order
    // (the same order whichever block is last) and re-arms the counter
    const int nb = gridDim.x * gridDim.y * gridDim.z;
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    if (threadIdx.x == 0) {
        part[bid] = S;
        __threadfence ();
        s_last = atomicAdd (arrive, 1u) == (unsigned) nb - 1;
    }
    __syncthreads ();
    if (!s_last) return;
    __threadfence ();
    double v = 0.0;
    for (int i = threadIdx.x; i < nb; i += REG_THREADS) v += __ldcg (part + i);
    dummy = 0;
    __syncthreads ();
    block_sum<REG_THREADS> (v, dummy, sh_v, sh_n);
    if (threadIdx.x == 0) {
        *score = v;
        *arrive = 0u;
    }
}

// ---- host -------------------------------------------------------------------

int
reg_alloc (RegState* s, const BspGeom& g, const float grid_spac[3])
{
    for (int d = 0; d < 3; d++) {
        s->cdims[d] = g.cdims[d];
        s->gs[d] = (double) grid_spac[d];
    }
    s->nknots = g.nknots;
    // the staged fields exceed the default 48 KB of shared memory for the
    // larger plans (set once per context, on its device)
    const size_t slot = REG_TH * 32 * sizeof (double);
    if (set_max_dynamic_smem ((const void*) reg_pass_y,
            (int) (REG_T1_MAX * slot)) != cudaSuccess
        || set_max_dynamic_smem ((const void*) reg_pass_z,
            (int) (REG_T2_MAX * slot + REG_E_MAX * REG_TY * 7 * sizeof (double)))
            != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    // pass z's grid: 32 knots along x x one y row x REG_TY planes
    s->nblocks = ((g.cdims[0] + 31) / 32) * g.cdims[1]
        * ((g.cdims[2] + REG_TY - 1) / REG_TY);
    const int cx = g.cdims[0], cy = g.cdims[1], cz = g.cdims[2];
    if (cudaMalloc (&s->d_gx, sizeof (double) * 6 * cx * 7) != cudaSuccess
        || cudaMalloc (&s->d_gy, sizeof (double) * 6 * cy * 7) != cudaSuccess
        || cudaMalloc (&s->d_hz, sizeof (double) * REG_E_MAX * cz * 7) != cudaSuccess
        || cudaMalloc (&s->d_t1, sizeof (double) * REG_T1_MAX * (size_t) g.nknots)
            != cudaSuccess
        || cudaMalloc (&s->d_t2, sizeof (double) * REG_T2_MAX * (size_t) g.nknots)
            != cudaSuccess
        || cudaMalloc (&s->d_part, sizeof (double) * s->nblocks) != cudaSuccess
        || cudaMalloc (&s->d_arrive, sizeof (unsigned)) != cudaSuccess
        || cudaMemset (s->d_arrive, 0, sizeof (unsigned)) != cudaSuccess
        || cudaMalloc (&s->d_score, sizeof (double)) != cudaSuccess
        || cudaMallocHost (&s->h_score, sizeof (double)) != cudaSuccess) {
        cudaGetLastError ();
        return B200BSP_E_OOM;
    }
    // Unweighted knot-axis bands for the six factor kinds.  Knot x takes
    // the Z factor (grid spacing 2), knot y the Y factor (spacing 1), knot
    // z the X factor (spacing 0).
    std::vector<double> gxh (6 * cx * 7), gyh (6 * cy * 7);
    s->gz_host.assign (6 * cz * 7, 0.0);
    for (int f = 0; f < 6; f++) {
        double P[16], Qm[16], F[16];
        pieces (P, s->gs[2], PAIRS[f][0]);
        pieces (Qm, s->gs[2], PAIRS[f][1]);
        integral (F, P, Qm, s->gs[2]);
        assemble (&gxh[f * cx * 7], F, cx, g.rdims[0]);
        pieces (P, s->gs[1], PAIRS[f][0]);
        pieces (Qm, s->gs[1], PAIRS[f][1]);
        integral (F, P, Qm, s->gs[1]);
        assemble (&gyh[f * cy * 7], F, cy, g.rdims[1]);
        pieces (P, s->gs[0], PAIRS[f][0]);
        pieces (Qm, s->gs[0], PAIRS[f][1]);
        integral (F, P, Qm, s->gs[0]);
        assemble (&s->gz_host[f * cz * 7], F, cz, g.rdims[2]);
    }
    if (cudaMemcpy (s->d_gx, gxh.data (), gxh.size () * sizeof (double),
            cudaMemcpyHostToDevice) != cudaSuccess
        || cudaMemcpy (s->d_gy, gyh.data (), gyh.size () * sizeof (double),
            cudaMemcpyHostToDevice) != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    return B200BSP_OK;
}

void
reg_free (RegState* s)
{
    cudaFree (s->d_gx); cudaFree (s->d_gy); cudaFree (s->d_hz);
    cudaFree (s->d_t1); cudaFree (s->d_t2); cudaFree (s->d_part);
    cudaFree (s->d_arrive);
    cudaFree (s->d_score); cudaFreeHost (s->h_score);
    *s = RegState ();
}

// Build the pass plan and the weighted z bands for one set of weights.
static int
reg_prepare (RegState* s, const b200bsp_reg_parms* p, cudaStream_t st)
{
    RegPlan plan;
    memset (&plan, 0, sizeof plan);
    std::map<int, int> t1_of, t2_of, e_of;       // keys -> slot
    const int cz = s->cdims[2];
    std::vector<double> hz;
    for (int t = 0; t < 32; t++) {
        const RegTerm& T = TERMS[t];
        float w = term_weight (T.w, p);
        if (w == 0.f) continue;
        int xf = pair_index (T.za, T.zb);        // knot-x factor
        int yf = pair_index (T.ya, T.yb);        // knot-y factor
        int zf = pair_index (T.xa, T.xb);        // knot-z factor
        int outs[3];
        int no = term_outputs (t, outs);
        for (int q = 0; q < no; q++) {
            int o = outs[q], c = OUT_COMP[o];
            int k1 = c * 8 + xf;
            if (!t1_of.count (k1)) {
                int id = plan.n1++;
                plan.t1_c[id] = (unsigned char) c;
                plan.t1_xf[id] = (unsigned char) xf;
                t1_of[k1] = id;
            }
            int s1 = t1_of[k1];
            int k2 = s1 * 8 + yf;
            if (!t2_of.count (k2)) {
                int id = plan.n2++;
                plan.t2_src[id] = (unsigned char) s1;
                plan.t2_yf[id] = (unsigned char) yf;
                t2_of[k2] = id;
            }
            int s2 = t2_of[k2];
            int k3 = s2 * 16 + o;
            if (!e_of.count (k3)) {
                int id = plan.ne++;
                plan.e_src[id] = (unsigned char) s2;
                plan.e_out[id] = (unsigned char) o;
                e_of[k3] = id;
                hz.resize ((size_t) plan.ne * cz * 7, 0.0);
            }
            double* dst = &hz[(size_t) e_of[k3] * cz * 7];
            const double* src = &s->gz_host[(size_t) zf * cz * 7];
            for (int i = 0; i < cz * 7; i++) dst[i] += (double) w * src[i];
            if (plan.n1 > REG_T1_MAX || plan.n2 > REG_T2_MAX
                || plan.ne > REG_E_MAX) {
                return B200BSP_E_UNSUPPORTED;   // cannot happen: 32 terms
            }
        }
    }
    {
        // pass 3's entries grouped by output, in their order within each
        RegPlan q = plan;
        std::vector<double> hz2 (hz.size ());
        int n = 0;
        for (int o = 0; o < O_N; o++) {
            q.e_off[o] = (unsigned char) n;
            for (int e = 0; e < plan.ne; e++) {
                if (plan.e_out[e] != o) continue;
                q.e_src[n] = plan.e_src[e];
                q.e_out[n] = plan.e_out[e];
                std::copy (hz.begin () + (size_t) e * cz * 7,
                    hz.begin () + (size_t) (e + 1) * cz * 7,
                    hz2.begin () + (size_t) n * cz * 7);
                n++;
            }
        }
        q.e_off[O_N] = (unsigned char) n;
        plan = q;
        hz.swap (hz2);
    }
    if (!hz.empty ()
        && cudaMemcpyAsync (s->d_hz, hz.data (), hz.size () * sizeof (double),
            cudaMemcpyHostToDevice, st) != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    // a pageable source is staged before cudaMemcpyAsync returns; the
    // synchronisation keeps the plan update ordered for every caller
    if (cudaStreamSynchronize (st) != cudaSuccess) return B200BSP_E_CUDA;
    s->plan = plan;
    s->parms = *p;
    s->have_parms = true;
    return B200BSP_OK;
}

int
reg_run (RegState* s, const BspGeom& g, const b200bsp_reg_parms* p,
    const float* d_coeff, float* d_grad, cudaStream_t st, double* d_grad64)
{
    if (!s->have_parms || memcmp (&s->parms, p, sizeof *p) != 0) {
        int rc = reg_prepare (s, p, st);
        if (rc) return rc;
    }
    const int cx = g.cdims[0], cy = g.cdims[1], cz = g.cdims[2];
    const int nk = g.nknots;
    const int bx = (cx + 31) / 32;
    const size_t slot = REG_TH * 32 * sizeof (double);
    const size_t zbands = REG_TY * 7 * sizeof (double);
    if (s->plan.n1) {
        const dim3 gxy (bx, (cy + REG_TY - 1) / REG_TY, cz);
        reg_pass_x<<<gxy, REG_THREADS, 0, st>>> (s->plan, cx, cy, nk,
            s->d_gx, d_coeff, s->d_t1);
        reg_pass_y<<<gxy, REG_THREADS, s->plan.n1 * slot, st>>> (s->plan, cx,
            cy, nk, s->d_gy, s->d_t1, s->d_t2);
    }
    const dim3 gz (bx, cy, (cz + REG_TY - 1) / REG_TY);
    reg_pass_z<<<gz, REG_THREADS, s->plan.n2 * slot + s->plan.ne * zbands,
        st>>> (s->plan, cx, cy,
        cz, nk, s->d_hz, s->d_t2, d_coeff, d_grad, d_grad64, s->d_part,
        s->d_arrive, s->d_score);
    return cudaGetLastError () == cudaSuccess ? B200BSP_OK : B200BSP_E_CUDA;
}

int
reg_fetch (RegState* s, double* score, cudaStream_t st)
{
    if (cudaMemcpyAsync (s->h_score, s->d_score, sizeof (double),
            cudaMemcpyDeviceToHost, st) != cudaSuccess
        || cudaStreamSynchronize (st) != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    *score = *s->h_score;
    return B200BSP_OK;
}

} // namespace b200
