// Tensor-core (tcgen05) form of the MSE score + gradient.
//
// The B-spline field at the voxels of one tile is a contraction with a
// table shared by every tile: d(v) = sum_m Q[v][m] * C_tile[m], m over the
// tile's 64 knots, Q[v][m] = bx[lx][i] * by[ly][j] * bz[lz][k] (the
// reference's bspline_interp_pix_c weights, src/base/bspline_interpolate.cxx:
// 78-110).  A batch of T tiles along x turns this into one GEMM
//     D[voxel][(c,t)] = Q[voxel][m] * C[(c,t)][m]
// and the adjoint condense (bspline_update_sets_b, src/register/bspline.cxx:
// 347-374) into another:
//     G[(c,t)][m] = sum_voxel DCDV[(c,t)][voxel] * Q[voxel][m].
// Both run on the tensor cores (kind::f16, bf16 operands, f32 accumulation
// in TMEM).  Every bf16 operand is split x = hi + lo (two bf16), and each
// product takes the three terms hi*hi + hi*lo + lo*hi, which keeps ~16
// significant bits -- the error budget of the gradient (1e-3) is met with
// margin while the voxel arithmetic (positions, trilinear samples,
// differences) stays in f32 on the CUDA cores.
//
// Two CTAs share an SM (about 111 KB of shared memory and 256 TMEM columns
// each), so one CTA's tensor-core and synchronisation phases hide behind
// the other's voxel work.  Each CTA loops over batches of T <= 26 tiles:
//   1. stage the (T+3) x 4 x 4 knot block, build C (hi/lo, 128B-swizzled)
//   2. forward MMA -> D in TMEM; the voxel phase reads D, samples the moving
//      image and writes dc/dv (hi/lo) into the adjoint operand; adjoint MMA
//      accumulates G in TMEM (per 128-voxel block when a tile has more)
//   3. G is copied to shared memory and every knot of the batch footprint
//      sums its (at most four) contributions in a fixed order -> global.
// With one 128-voxel block per tile the batches are software-pipelined:
// the adjoint of batch b runs while batch b+1 is staged and the forward of
// batch b+1 runs while batch b is gathered.  The per-batch partial sums
// are combined per knot by the finish kernel (deterministic, no atomics).
#include <algorithm>
#include <vector>

#include <cuda_bf16.h>

#include "bsp_common.cuh"
#include "kernels.cuh"
#include "tc_ptx.cuh"
#include "../../include/plastimatch_b200.h"

namespace b200 {

constexpr int TC_THREADS = 256;               // compute warps
constexpr int TC_WARPS = TC_THREADS / 32;
constexpr int TC_BLOCK = TC_THREADS + 32;      // + one tensor-core issuing warp
constexpr int GS_STRIDE = 65;                  // odd: conflict-free G copy
constexpr int TC_TMAX = 26;          // tiles per batch at most
constexpr int TC_MAX_MBLK = 8;       // 128-voxel blocks per tile at most
                                     // (vox_per_rgn up to 10 x 10 x 10)
constexpr int TC_TMEM_COLS = 256;
constexpr int TC_D_COL = 0;          // forward accumulator [0, N)
constexpr int TC_G_COL = 128;        // adjoint accumulator [128, 192)
constexpr uint32_t TC_WAIT_LIMIT = 1u << 22;
// Samples per thread per iteration of the axis-aligned voxel phase (their
// loads go out together).
#ifndef TC_SPT
#define TC_SPT 2
#endif

// What the kernel computes (template argument MODE):
//   TC_MSE_NEAREST  MSE score + gradient, moving gradient at the nearest voxel
//   TC_MSE_LINEAR   MSE score + gradient, trilinear moving gradient
//   TC_MI_GRAD      Mattes MI pass 2: dc/dv from the PVI-8 factor table
//   TC_MI_HIST      Mattes MI pass 1: PVI-8 histograms (no adjoint)
//   TC_PZ_GRAD      Mattes MI with cubic B-spline Parzen windows, pass 2
//   TC_PZ_HIST      the same, pass 1 (joint histogram, no adjoint)
// The MI modes run the axis-aligned voxel phase only.
constexpr int TC_MSE_NEAREST = 0;
constexpr int TC_MSE_LINEAR = 1;
constexpr int TC_MI_GRAD = 2;
constexpr int TC_MI_HIST = 3;
constexpr int TC_PZ_GRAD = 4;
constexpr int TC_PZ_HIST = 5;

__host__ __device__ constexpr bool
tc_hist_mode (int mode)
{
    return mode == TC_MI_HIST || mode == TC_PZ_HIST;
}
constexpr float TC_MI_WUNIT = 16777216.0f;   // histogram weights in 2^-24

// Adjoint-operand rows: (c, t) -> r = 8 (3 (t >> 3) + c) + (t & 7), so the
// three components of one tile sit at the same place in consecutive 8-row
// groups.  T <= 26 needs 12 groups = 96 rows; the MMA reads 128 rows per
// K chunk, and rows 96..127 alias the next chunk (their G rows are never
// read).
constexpr int DC_CHUNK = 96 * 128;                 // one 64-voxel K chunk
constexpr int DC_HALF = 2 * DC_CHUNK;              // 128 voxels, hi or lo
constexpr int DC_TAIL = 32 * 128;                  // rows 96..127 over-read

// Shared-memory map (offsets from a 1024-byte aligned base).
constexpr int SM_Q = 0;                            // Q hi 16 KB, lo 16 KB
constexpr int SM_C = 32768;                        // C hi, lo: N*128 B each
constexpr int SM_C_BYTES = 2 * 80 * 128;           // N <= 80
constexpr int SM_DC = SM_C + SM_C_BYTES;           // DCDV hi, lo (+ tail);
                                                   // G copy after the adjoint
constexpr int SM_S = SM_DC + 2 * DC_HALF + DC_TAIL; // knot block (bf16 hi|lo)
constexpr int SM_S_FLOATS = 3 * 16 * (TC_TMAX + 3);
constexpr int SM_TOTAL = SM_S + SM_S_FLOATS * 4;
static_assert (3 * TC_TMAX * GS_STRIDE * 4 <= 2 * DC_HALF, "G copy fits the DCDV area");
static_assert (3 * TC_TMAX <= 80, "N fits the C area");

struct TcArgs {
    BspGeom g;
    int T, N, mblk, V, nbx, nbatches;
    // x-line voxel phase with axis-aligned geometry (see voxel_phase_axis):
    // T0 tiles per round, W = vx * T0 voxels per round row, plane = W * vy * vz
    // samples per round, multiply-high reciprocals of W and vx
    int axis, T0, W, plane;
    unsigned mW, mvx;
    const float4* mgrad4;     // moving gradient padded to float4
    const float* fimg;
    const float* mimg;
    const float* mgrad;
    const float* coeff;
    const uint4* qimg;
    float* part;          // [batch][c][knot of the (T+3) x 4 x 4 footprint]
    double* score_part;   // [batch]: sum of diff^2
    int* count_part;      // [batch]: voxels counted
    int* err;
    // Mattes MI modes (TC_MI_GRAD, TC_MI_HIST): bin images, bins, the pass-2
    // factor table [fixed bin][moving bin] and the voxel count (float), the
    // global histogram f[B], m[B], j[B*B], count
    const uint8_t* fbin;
    const uint8_t* mbin;
    int bins;
    const float* mi_lut;
    const float* mi_nvf;
    unsigned long long* hist;
    float pz_mmin, pz_mdelta;    // Parzen: moving value -> window centre
    unsigned wait_limit;         // polls before a wait gives up
};

__device__ __forceinline__ void
split_bf16 (float x, unsigned short& hi, unsigned short& lo)
{
    __nv_bfloat16 h = __float2bfloat16_rn (x);
    __nv_bfloat16 l = __float2bfloat16_rn (x - __bfloat162float (h));
    hi = __bfloat16_as_ushort (h);
    lo = __bfloat16_as_ushort (l);
}

// Split two floats into bf16 hi/lo pairs with packed conversions:
// hi = bf16(a) | bf16(b) << 16, lo likewise for the remainders.
__device__ __forceinline__ void
split_bf16x2 (float a, float b, uint32_t& hi, uint32_t& lo)
{
    __nv_bfloat162 h = __floats2bfloat162_rn (a, b);
    float ha = __uint_as_float ((uint32_t) __bfloat16_as_ushort (h.x) << 16);
    float hb = __uint_as_float ((uint32_t) __bfloat16_as_ushort (h.y) << 16);
    __nv_bfloat162 l = __floats2bfloat162_rn (a - ha, b - hb);
    hi = *(uint32_t*) &h;
    lo = *(uint32_t*) &l;
}

// dc/dv of one sample into the adjoint operand at p (hi at p, lo at
// p + DC_HALF; components 1024 bytes apart).
__device__ __forceinline__ void
store_dc (uint8_t* p, float dc0, float dc1, float dc2)
{
    uint32_t h01, l01, h2, l2;
    split_bf16x2 (dc0, dc1, h01, l01);
    split_bf16x2 (dc2, 0.f, h2, l2);
    *(unsigned short*) (p) = (unsigned short) h01;
    *(unsigned short*) (p + DC_HALF) = (unsigned short) l01;
    *(unsigned short*) (p + 1024) = (unsigned short) (h01 >> 16);
    *(unsigned short*) (p + DC_HALF + 1024) = (unsigned short) (l01 >> 16);
    *(unsigned short*) (p + 2048) = (unsigned short) h2;
    *(unsigned short*) (p + DC_HALF + 2048) = (unsigned short) l2;
}

// Mattes MI pass 2 at one sample (the reference's bspline_mi_pvi_8_dc_dv,
// src/register/bspline_mi.cxx): the derivative of each PVI-8 corner weight
// along x, y, z times that corner's factor f[fixed bin][corner bin],
// negated, divided by the voxel count, then projected by the moving
// image's projection matrix in place (each row sees the rows above already
// updated, as the reference does).  w2: the upper-corner fractions.
__device__ __forceinline__ void
mi_dc_dv (const TcArgs& a, const float w2[3], int fb, const int mb[8],
    float nv, float dc[3])
{
    const float* l2 = w2;
    const float l1[3] = {1.f - w2[0], 1.f - w2[1], 1.f - w2[2]};
    const float dw[24] = {
        (-1) * l1[1] * l1[2], l1[0] * (-1) * l1[2], l1[0] * l1[1] * (-1),
        (+1) * l1[1] * l1[2], l2[0] * (-1) * l1[2], l2[0] * l1[1] * (-1),
        (-1) * l2[1] * l1[2], l1[0] * (+1) * l1[2], l1[0] * l2[1] * (-1),
        (+1) * l2[1] * l1[2], l2[0] * (+1) * l1[2], l2[0] * l2[1] * (-1),
        (-1) * l1[1] * l2[2], l1[0] * (-1) * l2[2], l1[0] * l1[1] * (+1),
        (+1) * l1[1] * l2[2], l2[0] * (-1) * l2[2], l2[0] * l1[1] * (+1),
        (-1) * l2[1] * l2[2], l1[0] * (+1) * l2[2], l1[0] * l2[1] * (+1),
        (+1) * l2[1] * l2[2], l2[0] * (+1) * l2[2], l2[0] * l2[1] * (+1)};
    const float* lut = a.mi_lut + fb * a.bins;
    float d0 = 0.f, d1 = 0.f, d2 = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const float f = __ldg (lut + mb[k]);
        d0 -= dw[3 * k + 0] * f;
        d1 -= dw[3 * k + 1] * f;
        d2 -= dw[3 * k + 2] * f;
    }
    d0 = d0 / nv;
    d1 = d1 / nv;
    d2 = d2 / nv;
    const float* p = a.g.mproj;
    d0 = d0 * p[0] + d1 * p[1] + d2 * p[2];
    d1 = d0 * p[3] + d1 * p[4] + d2 * p[5];
    d2 = d0 * p[6] + d1 * p[7] + d2 * p[8];
    dc[0] = d0;
    dc[1] = d1;
    dc[2] = d2;
}

struct TcCtx {
    uint8_t* sm;
    uint32_t sm_base;
    uint32_t taddr;
    int tid, warp, lane, q, tg, t_lo, t_hi;
};

// Compute-warp barrier (named barrier 1 over the 256 compute threads).
__device__ __forceinline__ void
cbar ()
{
    named_bar_sync (1, TC_THREADS);
}

// Knot block S[c][k][j][x] of batch (tx0, ty, tz), each coefficient
// already split: bf16 hi in the low half-word, bf16 lo in the high one (the
// forward operand repeats every coefficient four times, so it is split once
// here).  Warp w covers knot rows jk = w, w + 8 (jk = j + 4k), lane x and
// x + 32.
__device__ __forceinline__ void
stage_batch (const TcArgs& a, const TcCtx& x, int tx0, int ty, int tz)
{
    const BspGeom& g = a.g;
    const int KX = a.T + 3;
    uint32_t* S = (uint32_t*) (x.sm + SM_S);
#pragma unroll
    for (int r = 0; r < 2; r++) {
        const int jk = x.warp + TC_WARPS * r;
        const int j = jk & 3, k = jk >> 2;
        const int row = (tz + k) * g.cdims[1] * g.cdims[0]
            + (ty + j) * g.cdims[0];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int xx = x.lane + 32 * h;
            if (xx < KX) {
                const int kx = tx0 + xx;
                float v0 = 0.f, v1 = 0.f, v2 = 0.f;
                if (kx < g.cdims[0]) {
                    const float* cp = a.coeff + 3 * (row + kx);
                    v0 = __ldg (cp + 0);
                    v1 = __ldg (cp + 1);
                    v2 = __ldg (cp + 2);
                }
                unsigned short h, l;
                split_bf16 (v0, h, l);
                S[(0 * 16 + jk) * KX + xx] = (uint32_t) h | ((uint32_t) l << 16);
                split_bf16 (v1, h, l);
                S[(1 * 16 + jk) * KX + xx] = (uint32_t) h | ((uint32_t) l << 16);
                split_bf16 (v2, h, l);
                S[(2 * 16 + jk) * KX + xx] = (uint32_t) h | ((uint32_t) l << 16);
            }
        }
    }
}

// C[(c,t)][m] for the forward B operand: row n = c*T + t, K = 64 slots,
// hi/lo bf16, 128B-swizzled K-major.
__device__ __forceinline__ void
build_c (const TcArgs& a, const TcCtx& x)
{
    const int T = a.T, N = a.N, KX = T + 3;
    const uint32_t* S = (const uint32_t*) (x.sm + SM_S);
    for (int o = x.tid; o < N * 8; o += TC_THREADS) {
        const int n = o >> 3, ch = o & 7;    // 16-byte chunk: slots 8ch..8ch+7
        const int c = (n >= T) + (n >= 2 * T);
        const int t = n - c * T;
        // slots 8ch + e: i = e & 3, j = (2ch + (e >> 2)) & 3, k = ch >> 1
        const uint32_t* r0 = S + (c * 16 + ((2 * ch) & 3) + 4 * (ch >> 1)) * KX + t;
        const uint32_t* r1 = r0 + KX;
        const bool live = c < 3;
        uint32_t hw[4], lw[4];
#pragma unroll
        for (int e = 0; e < 8; e += 2) {
            const uint32_t p0 = live ? ((e < 4) ? r0[e] : r1[e - 4]) : 0u;
            const uint32_t p1 = live ? ((e < 4) ? r0[e + 1] : r1[e - 3]) : 0u;
            hw[e >> 1] = __byte_perm (p0, p1, 0x5410);   // the two hi halves
            lw[e >> 1] = __byte_perm (p0, p1, 0x7632);   // the two lo halves
        }
        const uint32_t off = sw128_offset (n, 8 * ch, N);
        *(uint4*) (x.sm + SM_C + off) = make_uint4 (hw[0], hw[1], hw[2], hw[3]);
        *(uint4*) (x.sm + SM_C + N * 128 + off) = make_uint4 (lw[0], lw[1], lw[2], lw[3]);
    }
}

// Forward D = Q * C^T (three split terms, K = 64); caller is one thread.
__device__ __forceinline__ void
issue_forward (const TcArgs& a, const TcCtx& x, uint64_t* bar)
{
    const uint32_t idesc = idesc_bf16_f32 (128, a.N, 0, 0);
    const uint32_t q0 = x.sm_base + SM_Q, c0 = x.sm_base + SM_C;
    const uint32_t cl = c0 + (uint32_t) a.N * 128;
    tc_fence_after ();
#pragma unroll
    for (int term = 0; term < 3; term++) {
        uint32_t qa = term == 2 ? q0 + 16384 : q0;     // hi, hi, lo
        uint32_t cb = term == 1 ? cl : c0;             // hi, lo, hi
#pragma unroll
        for (int ks = 0; ks < 4; ks++) {
            tc_mma_bf16 (x.taddr + TC_D_COL,
                smem_desc_sw128 (qa + ks * 32, 16, 1024),
                smem_desc_sw128 (cb + ks * 32, 16, 1024), idesc,
                (term > 0 || ks > 0) ? 1u : 0u);
        }
    }
    tc_commit (bar);
}

// Adjoint G (+)= DCDV * Q over the 128 voxels of one M block (A K-major in
// 96-row chunks, B = the Q bytes read MN-major); caller is one thread.
__device__ __forceinline__ void
issue_adjoint (const TcCtx& x, bool accumulate, uint64_t* bar)
{
    const uint32_t idesc = idesc_bf16_f32 (128, 64, 0, 1);
    const uint32_t d0 = x.sm_base + SM_DC, q0 = x.sm_base + SM_Q;
    tc_fence_after ();
#pragma unroll
    for (int term = 0; term < 3; term++) {
        uint32_t da = term == 1 ? d0 + DC_HALF : d0;   // hi, lo, hi
        uint32_t qb = term == 2 ? q0 + 16384 : q0;     // hi, hi, lo
#pragma unroll
        for (int s = 0; s < 8; s++) {
            tc_mma_bf16 (x.taddr + TC_G_COL,
                smem_desc_sw128 (da + (s >> 2) * DC_CHUNK + (s & 3) * 32, 16, 1024),
                smem_desc_sw128 (qb + s * 2048, 16384, 1024), idesc,
                (accumulate || term > 0 || s > 0) ? 1u : 0u);
        }
    }
    tc_commit (bar);
}

// Per-thread voxel constants of one 128-voxel M block.
struct VoxelSlot {
    int lx, ly, lz;
    bool live;           // voxel index < voxels per tile
    uint32_t vpart;      // adjoint-operand byte offset part from the voxel
    uint32_t vunit;      // 16-byte unit of the voxel within its 128-B row
};

__device__ __forceinline__ VoxelSlot
voxel_slot (const TcArgs& a, const TcCtx& x, int mb)
{
    const BspGeom& g = a.g;
    VoxelSlot s;
    const int vl = 32 * x.q + x.lane, v = 128 * mb + vl;
    const int vx = g.vpr[0], vy = g.vpr[1];
    s.lx = v % vx;
    s.ly = (v / vx) % vy;
    s.lz = v / (vx * vy);
    s.live = v < a.V;
    s.vpart = (vl >> 6) * (uint32_t) DC_CHUNK + (vl & 7) * 2u;
    s.vunit = (vl & 63) >> 3;
    return s;
}

// Mattes MI pass 1 at one sample: the PVI-8 corner weights (products of
// the per-axis fractions, in the reference's order) as integers in 2^-24
// units, so the sums do not depend on their order.  Corners with equal
// moving bins are merged first; a sample then has one, two or (rarely)
// more (fixed, moving) bin pairs.  The first two pairs of every lane
// combine across the warp (match + reduce, one round each) so that one lane
// per distinct pair updates the shared joint histogram; further pairs go
// straight to the shared atomics.  The fixed histogram counts each first-
// pair group's voxels; the moving histogram is the joint one's column sums,
// taken when the CTA flushes.  Every lane of the warp calls this (warp
// collectives).
__device__ __forceinline__ void
mi_hist_add (const TcArgs& a, const TcCtx& x, bool live, const float w2[3],
    int fb, const int mb[8], int& cnt)
{
    const int B = a.bins;
    unsigned long long* hf = (unsigned long long*) (x.sm + SM_DC);
    unsigned long long* hj = hf + 2 * B;
    const float* l2 = w2;
    const float l1[3] = {1.f - w2[0], 1.f - w2[1], 1.f - w2[2]};
    const float w[8] = {l1[0] * l1[1] * l1[2], l2[0] * l1[1] * l1[2],
        l1[0] * l2[1] * l1[2], l2[0] * l2[1] * l1[2], l1[0] * l1[1] * l2[2],
        l2[0] * l1[1] * l2[2], l1[0] * l2[1] * l2[2], l2[0] * l2[1] * l2[2]};
    unsigned int q[8];
#pragma unroll
    for (int k = 0; k < 8; k++) q[k] = __float2uint_rn (w[k] * TC_MI_WUNIT);
    // the first pair: corner 0's bin with the weights of every corner in
    // it; the second: the first other bin in corner order, likewise; any
    // further bins (rare) go corner by corner to the atomics below (integer
    // sums, so grouping them does not change the histogram)
    const int mb1 = mb[0];
    int mb2 = mb1;
    bool two = false;
#pragma unroll
    for (int k = 1; k < 8; k++) {
        mb2 = (!two && mb[k] != mb1) ? mb[k] : mb2;
        two = two || mb[k] != mb1;
    }
    unsigned int q1 = q[0], q2 = 0;
    bool many = false;
#pragma unroll
    for (int k = 1; k < 8; k++) {
        q1 += mb[k] == mb1 ? q[k] : 0u;
        q2 += mb[k] == mb2 && mb[k] != mb1 ? q[k] : 0u;
        many = many || (mb[k] != mb1 && mb[k] != mb2);
    }
    two = two && live;
    many = many && live;
    const unsigned live_mask = __ballot_sync (0xffffffffu, live);
    if (live) {
        cnt++;
        // first pair (a warp's sum stays below 32 * (2^24 + 8) < 2^32); its
        // leader also counts the group's voxels into the fixed histogram
        const int key = fb * B + mb1;
        const unsigned peers = __match_any_sync (live_mask, key);
        const unsigned sum = __reduce_add_sync (peers, q1);
        if (x.lane == __ffs (peers) - 1) {
            atomicAdd (&hj[key], (unsigned long long) sum);
            atomicAdd (&hf[fb], (unsigned long long) __popc (peers));
        }
    }
    const unsigned two_mask = __ballot_sync (0xffffffffu, two);
    if (two) {
        const int key = fb * B + mb2;
        const unsigned peers = __match_any_sync (two_mask, key);
        const unsigned sum = __reduce_add_sync (peers, q2);
        if (x.lane == __ffs (peers) - 1) {
            atomicAdd (&hj[key], (unsigned long long) sum);
        }
    }
    if (many) {
#pragma unroll
        for (int k = 1; k < 8; k++) {
            if (mb[k] != mb1 && mb[k] != mb2) {
                atomicAdd (&hj[fb * B + mb[k]], (unsigned long long) q[k]);
            }
        }
    }
}

// Mattes MI with cubic B-spline Parzen windows, pass 1 at one sample: the
// window's four weights at the moving value u (integers in 2^-24 units)
// into the fixed bin's row of the shared joint histogram; lanes with the
// same (fixed bin, first window bin) combine across the warp first.  Every
// lane of the warp calls this.
__device__ __forceinline__ void
pz_hist_add (const TcArgs& a, const TcCtx& x, bool live, int fb, float u,
    int& cnt)
{
    const int B = a.bins;
    unsigned long long* hj = (unsigned long long*) (x.sm + SM_DC) + 2 * B;
    const int k0 = parzen_first_bin (u, B);
    unsigned int q[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        q[j] = __float2uint_rn (bspline3f ((float) (k0 + j) - u) * TC_MI_WUNIT);
    }
    const unsigned live_mask = __ballot_sync (0xffffffffu, live);
    if (live) {
        cnt++;
        const int key = fb * B + k0;
        const unsigned peers = __match_any_sync (live_mask, key);
        unsigned sum[4];
#pragma unroll
        for (int j = 0; j < 4; j++) sum[j] = __reduce_add_sync (peers, q[j]);
        if (x.lane == __ffs (peers) - 1) {
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (sum[j]) atomicAdd (&hj[key + j], (unsigned long long) sum[j]);
            }
        }
    }
}

// Pass 2 at one sample: 1/(N delta_m) * sum over the window's bins of
// beta3'(k - u) log(p(f, k) / p_m(k)), times the world gradient of the
// trilinear interpolant (proj^T times the index gradient; 0 along an axis
// the clamp holds).
__device__ __forceinline__ void
pz_dc_dv (const TcArgs& a, float u, int fb, const float w2[3],
    const float m[8], int clamp, float dc[3])
{
    const int B = a.bins;
    const int k0 = parzen_first_bin (u, B);
    const float* row = a.mi_lut + fb * B;
    float sum = 0.f;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        sum += bspline3f_d ((float) (k0 + j) - u) * __ldg (row + k0 + j);
    }
    float gi[3];
    trilinear_igrad (w2, m, clamp, gi);
    const float sc = __ldg (a.mi_nvf + 1) * sum;
    const float* p = a.g.mproj;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        dc[c] = sc * (p[c] * gi[0] + p[3 + c] * gi[1] + p[6 + c] * gi[2]);
    }
}

// Voxel phase for one M block: thread (quarter q, lane) owns one voxel of
// every tile in [t_lo, t_hi).  Tiles go four at a time: the field values
// come from TMEM, then all four correspondences, then all gathers (8
// corners, fixed value, moving gradient), then the arithmetic.  Sample
// indices are clamped inside the moving image even when the sample is
// rejected, so only the fixed-image load needs a guard.
template <int MODE>
__device__ __forceinline__ void
voxel_phase (const TcArgs& a, const TcCtx& x, const VoxelSlot& vs, int tx0,
    int ty, int tz, double& sc, int& cnt)
{
    const BspGeom& g = a.g;
    const int T = a.T;
    const uint32_t lb = x.taddr + ((uint32_t) (32 * x.q) << 16) + TC_D_COL;
    const int fj = g.roi_off[1] + g.vpr[1] * ty + vs.ly;
    const int fk = g.roi_off[2] + g.vpr[2] * tz + vs.lz;
    const bool yz_ok = vs.live && fj < g.roi_off[1] + g.roi_dim[1]
        && fk < g.roi_off[2] + g.roi_dim[2];
    const int fi0 = g.roi_off[0] + g.vpr[0] * (tx0 + x.t_lo) + vs.lx;
    float pj[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        pj[d] = g.img_origin[d] + fi0 * g.fstep[3 * d] + fj * g.fstep[3 * d + 1]
            + fk * g.fstep[3 * d + 2];
    }
    const float xstep[3] = {g.vpr[0] * g.fstep[0], g.vpr[0] * g.fstep[3],
        g.vpr[0] * g.fstep[6]};
    const int frow = g.fdim[0] * (fj + g.fdim[1] * fk) + fi0;
    const int fi_room = g.roi_off[0] + g.roi_dim[0] - fi0;   // fi - fi0 < room
    const int t_cnt = min (x.t_hi - x.t_lo, g.rdims[0] - tx0 - x.t_lo);
    const int dxm = g.mdim[0], dxym = g.mdim[0] * g.mdim[1];
    uint8_t* dch = x.sm + SM_DC + vs.vpart;
    float scf = 0.f;
    for (int t4 = 0; t4 < x.t_hi - x.t_lo; t4 += 4) {
        float dv[12];
        tmem_ld4x3_wait (lb + x.t_lo + t4, lb + T + x.t_lo + t4,
            lb + 2 * T + x.t_lo + t4, dv);
        bool ok[4];
        int mvf[4], mvr[4], clampb[4];
        float w2[4][3];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int tt = t4 + u;
            const float ft = (float) tt;
            float fxyz[3] = {fmaf (ft, xstep[0], pj[0]), fmaf (ft, xstep[1], pj[1]),
                fmaf (ft, xstep[2], pj[2])};
            float d[3] = {dv[u], dv[4 + u], dv[8 + u]};
            bool in = locate_fast_c (g, fxyz, d, mvf[u], mvr[u], w2[u],
                clampb[u]);
            ok[u] = in && yz_ok && tt < t_cnt && g.vpr[0] * tt < fi_room;
        }
        if constexpr (MODE >= TC_MI_GRAD) {
            // Mattes MI: the fixed voxel's bin (guarded: a dead slot may lie
            // past the image) and the corners' bins (PVI-8) or values
            // (Parzen), then the histogram or the dc/dv of each sample
            constexpr bool pz = MODE == TC_PZ_GRAD || MODE == TC_PZ_HIST;
            int fb[4];
            float crm[4][8];
            int mb[4][8];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                fb[u] = ok[u] ? (int) __ldg (a.fbin + frow + g.vpr[0] * (t4 + u)) : 0;
                const int o[8] = {0, 1, dxm, dxm + 1, dxym, dxym + 1,
                    dxym + dxm, dxym + dxm + 1};
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    if (pz) crm[u][k] = __ldg (a.mimg + mvf[u] + o[k]);
                    else mb[u][k] = __ldg (a.mbin + mvf[u] + o[k]);
                }
            }
            const float nv = MODE == TC_MI_GRAD ? __ldg (a.mi_nvf) : 0.f;
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int t = x.t_lo + t4 + u;
                float dc[3] = {0.f, 0.f, 0.f};
                if constexpr (MODE == TC_MI_HIST) {
                    mi_hist_add (a, x, ok[u], w2[u], fb[u], mb[u], cnt);
                } else if constexpr (MODE == TC_PZ_HIST) {
                    pz_hist_add (a, x, ok[u], fb[u],
                        parzen_centre (trilinear_lerp (w2[u], crm[u]),
                            a.pz_mmin, a.pz_mdelta), cnt);
                } else if (ok[u]) {
                    if constexpr (MODE == TC_MI_GRAD) {
                        mi_dc_dv (a, w2[u], fb[u], mb[u], nv, dc);
                    } else {
                        pz_dc_dv (a, parzen_centre (trilinear_lerp (w2[u],
                            crm[u]), a.pz_mmin, a.pz_mdelta), fb[u], w2[u],
                            crm[u], clampb[u], dc);
                    }
                }
                if (!tc_hist_mode (MODE) && t < x.t_hi) {
                    const uint32_t o = (3 * (t >> 3)) * 1024u + (t & 7) * 128u
                        + ((vs.vunit ^ (uint32_t) (t & 7)) << 4);
                    unsigned short hh, ll;
                    split_bf16 (dc[0], hh, ll);
                    *(unsigned short*) (dch + o) = hh;
                    *(unsigned short*) (dch + DC_HALF + o) = ll;
                    split_bf16 (dc[1], hh, ll);
                    *(unsigned short*) (dch + 1024 + o) = hh;
                    *(unsigned short*) (dch + DC_HALF + 1024 + o) = ll;
                    split_bf16 (dc[2], hh, ll);
                    *(unsigned short*) (dch + 2048 + o) = hh;
                    *(unsigned short*) (dch + DC_HALF + 2048 + o) = ll;
                }
            }
            continue;
        }
        float cr[4][8], fv[4], gx[4], gy[4], gz[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const float* mp = a.mimg + mvf[u];
            cr[u][0] = __ldg (mp);
            cr[u][1] = __ldg (mp + 1);
            cr[u][2] = __ldg (mp + dxm);
            cr[u][3] = __ldg (mp + dxm + 1);
            cr[u][4] = __ldg (mp + dxym);
            cr[u][5] = __ldg (mp + dxym + 1);
            cr[u][6] = __ldg (mp + dxym + dxm);
            cr[u][7] = __ldg (mp + dxym + dxm + 1);
            fv[u] = ok[u] ? __ldg (a.fimg + frow + g.vpr[0] * (t4 + u)) : 0.f;
            if (MODE == TC_MSE_NEAREST) {
                const float* gp = a.mgrad + 3 * mvr[u];
                gx[u] = __ldg (gp + 0);
                gy[u] = __ldg (gp + 1);
                gz[u] = __ldg (gp + 2);
            }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int t = x.t_lo + t4 + u;
            float dc0 = 0.f, dc1 = 0.f, dc2 = 0.f;
            if (ok[u]) {
                const float diff = trilinear_lerp (w2[u], cr[u]) - fv[u];
                scf = fmaf (diff, diff, scf);
                cnt++;
                if (MODE == TC_MSE_NEAREST) {
                    dc0 = diff * gx[u]; dc1 = diff * gy[u]; dc2 = diff * gz[u];
                } else {
                    float gr[3];
                    trilinear_lerp_grad (g, w2[u], cr[u], gr);
                    dc0 = diff * gr[0]; dc1 = diff * gr[1]; dc2 = diff * gr[2];
                }
            }
            if (t < x.t_hi) {
                // row r = 8 (3 (t >> 3) + c) + (t & 7)
                const uint32_t o = (3 * (t >> 3)) * 1024u + (t & 7) * 128u
                    + ((vs.vunit ^ (uint32_t) (t & 7)) << 4);
                unsigned short hh, ll;
                split_bf16 (dc0, hh, ll);
                *(unsigned short*) (dch + o) = hh;
                *(unsigned short*) (dch + DC_HALF + o) = ll;
                split_bf16 (dc1, hh, ll);
                *(unsigned short*) (dch + 1024 + o) = hh;
                *(unsigned short*) (dch + DC_HALF + 1024 + o) = ll;
                split_bf16 (dc2, hh, ll);
                *(unsigned short*) (dch + 2048 + o) = hh;
                *(unsigned short*) (dch + DC_HALF + 2048 + o) = ll;
            }
        }
    }
    sc += (double) scf;
}

// Voxel phase in x-line order (tiles of at most 128 voxels).  The batch is
// done in two rounds of at most 13 tiles.  In each round the compute warps
// first copy the field values D from TMEM (lane = voxel of a tile) into
// Dt[c][rho * W + x] in the idle C area, where rho = ly + vy lz is the row
// of the tile and x = vx * tile + lx runs along the whole round (W = vx *
// tiles); then thread s of the round takes sample s = rho * W + x, so a
// warp's 32 lanes are 32 consecutive x of one (or two) rows: every gather
// touches one or two cache lines and the fixed image is read coalesced.
template <int GRAD_MODE>
__device__ __forceinline__ void
voxel_phase_xline (const TcArgs& a, const TcCtx& x, const VoxelSlot& vs,
    int tx0, int ty, int tz, double& sc, int& cnt)
{
    const BspGeom& g = a.g;
    const int T = a.T;
    const int vx = g.vpr[0], vy = g.vpr[1], vz = g.vpr[2];
    const int nrho = vy * vz;
    const unsigned mvx = 0xFFFFFFFFu / (unsigned) vx + 1u;
    const unsigned mvy = 0xFFFFFFFFu / (unsigned) vy + 1u;
    const int T0 = (T + 1) >> 1;                   // tiles of round 0
    float* Dt = (float*) (x.sm + SM_C);
    const uint32_t lb = x.taddr + ((uint32_t) (32 * x.q) << 16) + TC_D_COL;
    const int rho_v = vs.ly + vy * vs.lz;           // this lane's tile row
    const int dxm = g.mdim[0], dxym = g.mdim[0] * g.mdim[1];
    const int fi_base = g.roi_off[0] + vx * tx0;
    const int fj_base = g.roi_off[1] + vy * ty;
    const int fk_base = g.roi_off[2] + vz * tz;
    const int fi_end = g.roi_off[0] + g.roi_dim[0];
    const int fj_end = g.roi_off[1] + g.roi_dim[1];
    const int fk_end = g.roi_off[2] + g.roi_dim[2];
    const int tx_room = g.rdims[0] - tx0;          // live tiles of the batch
    uint8_t* dch = x.sm + SM_DC;
    float scf = 0.f;

    // Padding voxels (V..127) carry no samples; their adjoint columns must be
    // zero in the rows of live tiles (the G copy of the previous batch
    // overwrote this area, and a non-finite bf16 there times Q = 0 would
    // still poison the accumulation).
    const int npad = 128 - a.V;
    for (int o = x.tid; o < npad * T; o += TC_THREADS) {
        const int tb = o / npad, v = a.V + (o - tb * npad);
        uint8_t* p = dch + (v >> 6) * DC_CHUNK + (3 * (tb >> 3)) * 1024
            + (tb & 7) * 128 + ((((v & 63) >> 3) ^ (tb & 7)) << 4) + (v & 7) * 2;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            *(unsigned short*) (p + 1024 * c) = 0;
            *(unsigned short*) (p + DC_HALF + 1024 * c) = 0;
        }
    }

    for (int r = 0; r < 2; r++) {
        const int rt0 = r * T0;                    // first tile of the round
        const int Tr = min (T0, T - rt0);
        if (Tr <= 0) break;
        const int W = vx * Tr, plane = nrho * W;
        // multiply-high reciprocals: floor(n / d) = umulhi(n, ceil(2^32 / d))
        // exactly for the n < 2^16 and 2 <= d <= 1024 used here (d = 1 is
        // the identity)
        const unsigned mW = 0xFFFFFFFFu / (unsigned) W + 1u;
        // 1. D -> Dt: warp group tg copies tiles [tg*h, tg*h + h) of the round
        {
            const int h = (Tr + 1) >> 1;
            const int u0 = x.tg * h, u1 = min (Tr, u0 + h);
            for (int t4 = u0; t4 < u1; t4 += 4) {
                float dv[12];
                tmem_ld4x3_wait (lb + rt0 + t4, lb + T + rt0 + t4,
                    lb + 2 * T + rt0 + t4, dv);
                if (vs.live) {
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const int tt = t4 + u;
                        if (tt < u1) {
                            const int o = rho_v * W + tt * vx + vs.lx;
                            Dt[o] = dv[u];
                            Dt[plane + o] = dv[4 + u];
                            Dt[2 * plane + o] = dv[8 + u];
                        }
                    }
                }
            }
        }
        cbar ();
        // 2. samples s = tid + 256 k of the round, four at a time
        const int total = plane;
        for (int s0 = x.tid; s0 < total; s0 += 4 * TC_THREADS) {
            bool ok[4];
            int mvf[4], mvr[4], fidx[4];
            uint32_t doff[4];
            float w2[4][3];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int sidx = s0 + u * TC_THREADS;
                const bool in_round = sidx < total;
                const int sc_ = in_round ? sidx : 0;
                // exact small-range divisions by multiply-high (no XU)
                const int rho = W > 1 ? (int) __umulhi ((unsigned) sc_, mW) : sc_;
                const int xx = sc_ - rho * W;
                const int tt = vx > 1 ? (int) __umulhi ((unsigned) xx, mvx) : xx;
                const int lx = xx - tt * vx;
                const int lz = vy > 1 ? (int) __umulhi ((unsigned) rho, mvy) : rho;
                const int ly = rho - lz * vy;
                const int fi = fi_base + vx * rt0 + xx;
                const int fj = fj_base + ly, fk = fk_base + lz;
                const int tb = rt0 + tt;                  // tile within batch
                const bool live = in_round && tb < tx_room && fi < fi_end
                    && fj < fj_end && fk < fk_end;
                const float ffi = i2f_small (fi), ffj = i2f_small (fj);
                const float ffk = i2f_small (fk);
                float fxyz[3];
#pragma unroll
                for (int dd = 0; dd < 3; dd++) {
                    fxyz[dd] = g.img_origin[dd] + ffi * g.fstep[3 * dd]
                        + ffj * g.fstep[3 * dd + 1] + ffk * g.fstep[3 * dd + 2];
                }
                float d[3] = {Dt[sc_], Dt[plane + sc_], Dt[2 * plane + sc_]};
                bool in = locate_nx (g, fxyz, d, mvf[u], mvr[u], w2[u]);
                ok[u] = in && live;
                fidx[u] = fi + g.fdim[0] * (fj + g.fdim[1] * fk);
                // adjoint operand offset: row r(c, tb), column v
                const int v = lx + vx * rho;
                doff[u] = in_round
                    ? (uint32_t) ((v >> 6) * DC_CHUNK + (3 * (tb >> 3)) * 1024
                        + (tb & 7) * 128 + ((((v & 63) >> 3) ^ (tb & 7)) << 4)
                        + (v & 7) * 2)
                    : 0xffffffffu;
            }
            float cr[4][8], fv[4], gx[4], gy[4], gz[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const float* mp = a.mimg + mvf[u];
                cr[u][0] = __ldg (mp);
                cr[u][1] = __ldg (mp + 1);
                cr[u][2] = __ldg (mp + dxm);
                cr[u][3] = __ldg (mp + dxm + 1);
                cr[u][4] = __ldg (mp + dxym);
                cr[u][5] = __ldg (mp + dxym + 1);
                cr[u][6] = __ldg (mp + dxym + dxm);
                cr[u][7] = __ldg (mp + dxym + dxm + 1);
                fv[u] = ok[u] ? __ldg (a.fimg + fidx[u]) : 0.f;
                if (GRAD_MODE == 0) {
                    const float* gp = a.mgrad + 3 * mvr[u];
                    gx[u] = __ldg (gp + 0);
                    gy[u] = __ldg (gp + 1);
                    gz[u] = __ldg (gp + 2);
                }
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                float dc0 = 0.f, dc1 = 0.f, dc2 = 0.f;
                if (ok[u]) {
                    const float diff = trilinear_lerp (w2[u], cr[u]) - fv[u];
                    scf = fmaf (diff, diff, scf);
                    cnt++;
                    if (GRAD_MODE == 0) {
                        dc0 = diff * gx[u]; dc1 = diff * gy[u]; dc2 = diff * gz[u];
                    } else {
                        float gr[3];
                        trilinear_lerp_grad (g, w2[u], cr[u], gr);
                        dc0 = diff * gr[0]; dc1 = diff * gr[1]; dc2 = diff * gr[2];
                    }
                }
                if (doff[u] != 0xffffffffu) {
                    uint8_t* p = dch + doff[u];
                    uint32_t h01, l01, h2, l2;
                    split_bf16x2 (dc0, dc1, h01, l01);
                    split_bf16x2 (dc2, 0.f, h2, l2);
                    *(unsigned short*) (p) = (unsigned short) h01;
                    *(unsigned short*) (p + DC_HALF) = (unsigned short) l01;
                    *(unsigned short*) (p + 1024) = (unsigned short) (h01 >> 16);
                    *(unsigned short*) (p + DC_HALF + 1024) = (unsigned short) (l01 >> 16);
                    *(unsigned short*) (p + 2048) = (unsigned short) h2;
                    *(unsigned short*) (p + DC_HALF + 2048) = (unsigned short) l2;
                }
            }
        }
        cbar ();                                   // Dt reused by the next round
    }
    sc += (double) scf;
}

// Voxel phase for axis-aligned geometry (step and projection matrices
// diagonal), in the x-line order of voxel_phase_xline with the per-sample
// work cut to what a sample needs: world positions come from per-batch
// tables (x along the batch, y and z per tile row, with the fixed-image row
// index), the field is read back as one (x, y) pair and one z, the clamp
// runs without conversions, every index stays inside its image so no load
// is guarded, and the moving gradient is one 16-byte load.  Both rounds use
// W = vx * T0 voxels per row so one sample -> (row, x) mapping serves every
// batch; a round-1 tile slot past the batch's last tile is dead.
template <int MODE>
__device__ __forceinline__ void
voxel_phase_axis (const TcArgs& a, const TcCtx& x, const VoxelSlot& vs,
    int tx0, int ty, int tz, double& sc, int& cnt)
{
    const BspGeom& g = a.g;
    const int T = a.T, T0 = a.T0, W = a.W, plane = a.plane;
    const int vx = g.vpr[0], vy = g.vpr[1], vz = g.vpr[2];
    const int nrho = vy * vz;
    float2* Dxy = (float2*) (x.sm + SM_C);
    float* Dz = (float*) (x.sm + SM_C + 8 * plane);
    uint4* rowtab = (uint4*) (x.sm + SM_S);
    float* posx = (float*) (x.sm + SM_S + 16 * nrho);
    uint8_t* dch = x.sm + SM_DC;
    const int dxm = g.mdim[0], dxym = g.mdim[0] * g.mdim[1];
    const int fi_base = g.roi_off[0] + vx * tx0;
    const int fj_base = g.roi_off[1] + vy * ty;
    const int fk_base = g.roi_off[2] + vz * tz;
    // batch x index X = vx * (batch tile) + lx is live below xlim
    const int xlim = min (min (g.rdims[0] - tx0, T) * vx,
        g.roi_off[0] + g.roi_dim[0] - fi_base);
    float scf = 0.f;

    // Padding voxels (V..127) carry no samples; zero their adjoint columns
    // in the rows of live tiles (see voxel_phase_xline).  The histogram
    // pass has no adjoint (its histograms live in that area).
    const int npad = tc_hist_mode (MODE) ? 0 : 128 - a.V;
    for (int o = x.tid; o < npad * T; o += TC_THREADS) {
        const int tb = o / npad, v = a.V + (o - tb * npad);
        uint8_t* p = dch + (v >> 6) * DC_CHUNK + (3 * (tb >> 3)) * 1024
            + (tb & 7) * 128 + ((((v & 63) >> 3) ^ (tb & 7)) << 4) + (v & 7) * 2;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            *(unsigned short*) (p + 1024 * c) = 0;
            *(unsigned short*) (p + DC_HALF + 1024 * c) = 0;
        }
    }
    // Position tables: x over both rounds, (y, z, fixed row, live) per row.
    // origin + step * index with the step's zero off-diagonal terms dropped
    // (they add exact zeros).
    for (int i = x.tid; i < 2 * W; i += TC_THREADS) {
        posx[i] = fmaf (i2f_small (fi_base + i), g.fstep[0], g.img_origin[0]);
    }
    for (int rho = x.tid; rho < nrho; rho += TC_THREADS) {
        const int lz = rho / vy, ly = rho - lz * vy;
        const int fj = fj_base + ly, fk = fk_base + lz;
        const bool live = fj < g.roi_off[1] + g.roi_dim[1]
            && fk < g.roi_off[2] + g.roi_dim[2];
        const float py = fmaf (i2f_small (fj), g.fstep[4], g.img_origin[1]);
        const float pz = fmaf (i2f_small (fk), g.fstep[8], g.img_origin[2]);
        const int row = g.fdim[0] * (min (fj, g.fdim[1] - 1)
            + g.fdim[1] * min (fk, g.fdim[2] - 1));
        rowtab[rho] = make_uint4 (__float_as_uint (py), __float_as_uint (pz),
            (uint32_t) row, live ? 1u : 0u);
    }

    const uint32_t lb = x.taddr + ((uint32_t) (32 * x.q) << 16) + TC_D_COL;
    const int rho_v = vs.ly + vy * vs.lz;
    for (int r = 0; r < 2; r++) {
        const int rt0 = r * T0;
        const int Tr = min (T0, T - rt0);
        if (Tr <= 0) break;
        // 1. field values of the round's tiles: TMEM -> (Dxy, Dz)[rho W + x]
        {
            const int h = (Tr + 1) >> 1;
            const int u0 = x.tg * h, u1 = min (Tr, u0 + h);
            for (int t4 = u0; t4 < u1; t4 += 4) {
                float dv[12];
                tmem_ld4x3_wait (lb + rt0 + t4, lb + T + rt0 + t4,
                    lb + 2 * T + rt0 + t4, dv);
                if (vs.live) {
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const int tt = t4 + u;
                        if (tt < u1) {
                            const int o = rho_v * W + tt * vx + vs.lx;
                            Dxy[o] = make_float2 (dv[u], dv[4 + u]);
                            Dz[o] = dv[8 + u];
                        }
                    }
                }
            }
        }
        cbar ();
        // 2. samples s + 256 u (u < TC_SPT), s = tid + 256 TC_SPT k; the MI
        //    histogram pass keeps every lane of a warp in the loop (warp
        //    collectives), the other modes let a lane leave at the plane end
        const int X0 = r * W;
        const int s_end = tc_hist_mode (MODE) ? plane + x.lane : plane;
        for (int s0 = x.tid; s0 < s_end; s0 += TC_SPT * TC_THREADS) {
            bool ok[TC_SPT];
            int mvf[TC_SPT], mvr[TC_SPT], fidx[TC_SPT];
            uint32_t doff[TC_SPT];
            float w2[TC_SPT][3];
            int clampb[TC_SPT];
#pragma unroll
            for (int u = 0; u < TC_SPT; u++) {
                const int sv = s0 + u * TC_THREADS;
                const bool in_plane = sv < plane;
                const int sc_ = in_plane ? sv : 0;
                const int rho = (int) __umulhi ((unsigned) sc_, a.mW);
                const int xx = sc_ - rho * W;
                const int tt = (int) __umulhi ((unsigned) xx, a.mvx);
                const int lx = xx - tt * vx;
                const int X = X0 + xx;
                const uint4 rw = rowtab[rho];
                const float2 dxy = Dxy[sc_];
                const float dz = Dz[sc_];
                const float ma[3] = {
                    ((posx[X] + dxy.x) - g.morigin[0]) * g.mproj[0],
                    ((__uint_as_float (rw.x) + dxy.y) - g.morigin[1]) * g.mproj[4],
                    ((__uint_as_float (rw.y) + dz) - g.morigin[2]) * g.mproj[8]};
                bool in = in_plane && rw.w != 0u && X < xlim;
                int f[3];
                bool up[3];
                clampb[u] = 0;
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    in = in && ma[d] > -0.5f && ma[d] < g.m_hi[d];
                    if (MODE == TC_PZ_GRAD && (ma[d] < 0.f || ma[d] >= g.m_fmax[d] + 1.f)) {
                        clampb[u] |= 1 << d;
                    }
                    // floor(max(ma, 0)) in the low mantissa bits of
                    // max(ma, 0) + 2^23 rounded down; corner clamped to
                    // dim - 2, fraction saturated to [0, 1] (li_clamp)
                    const float big = __fadd_rd (fmaxf (ma[d], 0.f), 8388608.f);
                    f[d] = min (__float_as_int (big) - 0x4B000000, g.mdim[d] - 2);
                    const float fc = fminf (big - 8388608.f, g.m_fmax[d]);
                    const float w = __saturatef (ma[d] - fc);
                    w2[u][d] = w;
                    up[d] = w >= 0.5f;
                }
                ok[u] = in;
                mvf[u] = f[0] + dxm * (f[1] + g.mdim[1] * f[2]);
                mvr[u] = mvf[u] + (up[0] ? 1 : 0) + (up[1] ? dxm : 0)
                    + (up[2] ? dxym : 0);
                fidx[u] = (int) rw.z + min (fi_base + X, g.fdim[0] - 1);
                const int v = lx + vx * rho;
                const int tb = rt0 + tt;
                doff[u] = in_plane
                    ? (uint32_t) ((v >> 6) * DC_CHUNK + (3 * (tb >> 3)) * 1024
                        + (tb & 7) * 128 + ((((v >> 3) ^ tb) & 7) << 4)
                        + (v & 7) * 2)
                    : 0xffffffffu;
            }
            if constexpr (MODE == TC_PZ_GRAD || MODE == TC_PZ_HIST) {
                float cr[TC_SPT][8];
                int fb[TC_SPT];
#pragma unroll
                for (int u = 0; u < TC_SPT; u++) {
                    const float* mp = a.mimg + mvf[u];
                    cr[u][0] = __ldg (mp);
                    cr[u][1] = __ldg (mp + 1);
                    cr[u][2] = __ldg (mp + dxm);
                    cr[u][3] = __ldg (mp + dxm + 1);
                    cr[u][4] = __ldg (mp + dxym);
                    cr[u][5] = __ldg (mp + dxym + 1);
                    cr[u][6] = __ldg (mp + dxym + dxm);
                    cr[u][7] = __ldg (mp + dxym + dxm + 1);
                    fb[u] = __ldg (a.fbin + fidx[u]);
                }
#pragma unroll
                for (int u = 0; u < TC_SPT; u++) {
                    const float uc = parzen_centre (trilinear_lerp (w2[u], cr[u]),
                        a.pz_mmin, a.pz_mdelta);
                    if constexpr (MODE == TC_PZ_HIST) {
                        pz_hist_add (a, x, ok[u], fb[u], uc, cnt);
                    } else {
                        float dc[3];
                        pz_dc_dv (a, uc, fb[u], w2[u], cr[u], clampb[u], dc);
                        if (!ok[u]) dc[0] = dc[1] = dc[2] = 0.f;
                        if (doff[u] != 0xffffffffu) store_dc (dch + doff[u], dc[0], dc[1], dc[2]);
                    }
                }
            } else if constexpr (MODE == TC_MSE_NEAREST || MODE == TC_MSE_LINEAR) {
                float cr[TC_SPT][8], fv[TC_SPT];
                float4 gr[TC_SPT];
#pragma unroll
                for (int u = 0; u < TC_SPT; u++) {
                    const float* mp = a.mimg + mvf[u];
                    cr[u][0] = __ldg (mp);
                    cr[u][1] = __ldg (mp + 1);
                    cr[u][2] = __ldg (mp + dxm);
                    cr[u][3] = __ldg (mp + dxm + 1);
                    cr[u][4] = __ldg (mp + dxym);
                    cr[u][5] = __ldg (mp + dxym + 1);
                    cr[u][6] = __ldg (mp + dxym + dxm);
                    cr[u][7] = __ldg (mp + dxym + dxm + 1);
                    fv[u] = __ldg (a.fimg + fidx[u]);
                    if (MODE == TC_MSE_NEAREST) gr[u] = __ldg (a.mgrad4 + mvr[u]);
                }
#pragma unroll
                for (int u = 0; u < TC_SPT; u++) {
                    float diff = trilinear_lerp (w2[u], cr[u]) - fv[u];
                    diff = ok[u] ? diff : 0.f;
                    scf = fmaf (diff, diff, scf);
                    cnt += ok[u] ? 1 : 0;
                    float dc0, dc1, dc2;
                    if (MODE == TC_MSE_NEAREST) {
                        dc0 = diff * gr[u].x; dc1 = diff * gr[u].y; dc2 = diff * gr[u].z;
                    } else {
                        float grd[3];
                        trilinear_lerp_grad (g, w2[u], cr[u], grd);
                        dc0 = diff * grd[0]; dc1 = diff * grd[1]; dc2 = diff * grd[2];
                    }
                    if (doff[u] != 0xffffffffu) store_dc (dch + doff[u], dc0, dc1, dc2);
                }
            } else {
                // PVI-8: the fixed voxel's bin and the bins of the eight
                // corners (the trilinear corners, in the same order)
                int fb[TC_SPT], mb[TC_SPT][8];
#pragma unroll
                for (int u = 0; u < TC_SPT; u++) {
                    const uint8_t* mp = a.mbin + mvf[u];
                    mb[u][0] = __ldg (mp);
                    mb[u][1] = __ldg (mp + 1);
                    mb[u][2] = __ldg (mp + dxm);
                    mb[u][3] = __ldg (mp + dxm + 1);
                    mb[u][4] = __ldg (mp + dxym);
                    mb[u][5] = __ldg (mp + dxym + 1);
                    mb[u][6] = __ldg (mp + dxym + dxm);
                    mb[u][7] = __ldg (mp + dxym + dxm + 1);
                    fb[u] = __ldg (a.fbin + fidx[u]);
                }
                if constexpr (MODE == TC_MI_GRAD) {
                    const float nv = __ldg (a.mi_nvf);
#pragma unroll
                    for (int u = 0; u < TC_SPT; u++) {
                        float dc[3];
                        mi_dc_dv (a, w2[u], fb[u], mb[u], nv, dc);
                        if (!ok[u]) dc[0] = dc[1] = dc[2] = 0.f;
                        if (doff[u] != 0xffffffffu) store_dc (dch + doff[u], dc[0], dc[1], dc[2]);
                    }
                } else {
#pragma unroll
                    for (int u = 0; u < TC_SPT; u++) {
                        mi_hist_add (a, x, ok[u], w2[u], fb[u], mb[u], cnt);
                    }
                }
            }
        }
        cbar ();                                   // Dxy/Dz reused next round
    }
    sc += (double) scf;
}

// Copy G (rows r -> (c, t), 64 slot columns) from TMEM to shared memory as
// Gs[(c*T + t)*65 + slot] (odd row stride: the per-lane rows land in
// distinct banks).  Warp (quarter q, group tg) takes rows 32q..+31, slots
// 32tg..+31.
__device__ __forceinline__ void
dump_g (const TcArgs& a, const TcCtx& x)
{
    const int r = 32 * x.q + x.lane, gi = r >> 3;
    const int c = gi % 3, t = 8 * (gi / 3) + (r & 7);
    float* Gs = (float*) (x.sm + SM_DC);
    const bool live = gi < 12 && t < a.T;
    float gv[16];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int col = 32 * x.tg + 16 * h;
        tmem_ld16_wait (x.taddr + ((uint32_t) (32 * x.q) << 16) + TC_G_COL + col,
            gv);
        if (live) {
            float* dst = Gs + (c * a.T + t) * GS_STRIDE + col;
#pragma unroll
            for (int e = 0; e < 16; e++) dst[e] = gv[e];
        }
    }
}

// Every knot (x, j, k) of the batch footprint sums slot (i, j, k) of the
// tiles t = x - i, i = 0..3 (slot order, as the reference's condense), and
// writes part[b][c][x + KX (j + 4k)].
__device__ __forceinline__ void
gather_knots (const TcArgs& a, const TcCtx& x, int b)
{
    const int T = a.T, KX = T + 3, KF = 16 * KX;
    const float* Gs = (const float*) (x.sm + SM_DC);
    float* dst = a.part + (size_t) b * 3 * KF;
    for (int row = x.warp; row < 48; row += TC_WARPS) {     // row = 16c + jk
        const int c = row >> 4, jk = row & 15;
        const int xx = x.lane;
        if (xx < KX) {
            float s = 0.f;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int t = xx - i;
                if (t >= 0 && t < T) s += Gs[(c * T + t) * GS_STRIDE + i + 4 * jk];
            }
            dst[c * KF + jk * KX + xx] = s;
        }
    }
}

// Compute warps wait for a tensor-core phase: lane 0 of each warp polls
// (bounded, and gives up early once another wait has failed), then all
// compute warps meet, so they leave the batch loop together on failure.
__device__ __forceinline__ bool
cwait (const TcArgs& a, const TcCtx& x, uint64_t* bar, uint32_t& ph,
    volatile int* s_abort, int code)
{
    if (x.lane == 0) {
        bool ok = false;
        for (uint32_t n = 0; n < a.wait_limit && !*s_abort; n++) {
            if (mbar_try_wait (bar, ph)) { ok = true; break; }
        }
        if (!ok) {
            *s_abort = 1;
            atomicExch (a.err, code);
        }
    }
    ph ^= 1;
    __syncwarp ();
    cbar ();
    tc_fence_after ();
    return *s_abort == 0;
}

// One arrival per compute warp, after the warp's shared-memory writes are
// made visible to the tensor cores.
__device__ __forceinline__ void
warp_arrive (const TcCtx& x, uint64_t* bar)
{
    fence_proxy_async_smem ();
    tc_fence_before ();
    __syncwarp ();
    if (x.lane == 0) mbar_arrive (bar);
}

// Tensor-core warp: for every batch and 128-voxel block, wait for the
// forward operands, issue the forward GEMM, wait for dc/dv, issue the
// adjoint (the MI histogram pass has no adjoint).  Bounded waits; gives up
// when a compute wait failed.
__device__ __forceinline__ void
mma_loop (const TcArgs& a, const TcCtx& x, int nb_local, bool adjoint,
    uint64_t* bars, volatile int* s_abort)
{
    uint32_t ph_c = 0, ph_dc = 0;
    for (int i = 0; i < nb_local && !*s_abort; i++) {
        for (int mb = 0; mb < a.mblk; mb++) {
            bool ok = false;
            for (uint32_t n = 0; n < a.wait_limit && !*s_abort; n++) {
                if (mbar_try_wait (&bars[0], ph_c)) { ok = true; break; }
            }
            if (!ok) { *s_abort = 1; atomicExch (a.err, 3); return; }
            ph_c ^= 1;
            issue_forward (a, x, &bars[2]);
            if (!adjoint) continue;
            ok = false;
            for (uint32_t n = 0; n < a.wait_limit && !*s_abort; n++) {
                if (mbar_try_wait (&bars[1], ph_dc)) { ok = true; break; }
            }
            if (!ok) { *s_abort = 1; atomicExch (a.err, 4); return; }
            ph_dc ^= 1;
            issue_adjoint (x, mb > 0, &bars[3]);
        }
    }
}

template <int MODE>
__global__ void __launch_bounds__ (TC_BLOCK, 2)
mse_tc_kernel (TcArgs a)
{
    extern __shared__ uint8_t smem_raw[];
    // bars: 0 C ready (8 arrivals), 1 dc/dv ready (8), 2 D full (commit),
    // 3 G full (commit)
    __shared__ uint64_t s_bar[4];
    __shared__ uint32_t s_taddr;
    __shared__ int s_abort;
    __shared__ double sh_v[TC_WARPS];
    __shared__ int sh_n[TC_WARPS];

    const BspGeom& g = a.g;
    TcCtx x;
    // Round up to 1024 B by offsetting smem_raw itself, so every access
    // through x.sm stays a shared-memory access (32-bit addresses).
    x.sm = smem_raw + ((1024u - (smem_addr (smem_raw) & 1023u)) & 1023u);
    x.sm_base = smem_addr (x.sm);
    x.tid = threadIdx.x;
    x.warp = x.tid >> 5;
    x.lane = x.tid & 31;
    x.q = x.warp & 3;                          // TMEM lane quarter
    x.tg = (x.warp >> 2) & 1;                  // tile group (2)
    x.t_lo = (a.T * x.tg) / 2;                 // balanced contiguous ranges
    x.t_hi = (a.T * (x.tg + 1)) / 2;
    const bool mma_warp = x.warp == TC_WARPS;

    if (x.tid == 0) {
        mbar_init (&s_bar[0], TC_WARPS);
        mbar_init (&s_bar[1], TC_WARPS);
        mbar_init (&s_bar[2], 1);
        mbar_init (&s_bar[3], 1);
        fence_barrier_init ();
        s_abort = 0;
    }
    if (mma_warp) {
        tmem_alloc (&s_taddr, TC_TMEM_COLS);
        tmem_relinquish ();
    } else {
        // Adjoint entries the voxel phase never writes (rows of tiles >= T)
        // only feed G rows that are never read; start them at zero anyway.
        for (int o = x.tid; o < (2 * DC_HALF + DC_TAIL) / 16; o += TC_THREADS) {
            ((uint4*) (x.sm + SM_DC))[o] = make_uint4 (0, 0, 0, 0);
        }
        if (a.mblk == 1) {
            for (int o = x.tid; o < 2048; o += TC_THREADS) {
                ((uint4*) (x.sm + SM_Q))[o] = a.qimg[o];
            }
        }
    }
    tc_fence_before ();
    __syncthreads ();
    tc_fence_after ();
    x.taddr = s_taddr;
    const int nb_local = (a.nbatches - (int) blockIdx.x + (int) gridDim.x - 1)
        / (int) gridDim.x;
    volatile int* abort_flag = &s_abort;

    if (mma_warp) {
        if (x.lane == 0) {
            mma_loop (a, x, nb_local, !tc_hist_mode (MODE), s_bar, abort_flag);
        }
        __syncwarp ();
    } else {
        uint32_t ph_d = 0, ph_g = 0;
        double sc = 0.0;
        int cnt = 0;
        auto coords = [&](int b, int& tx0, int& ty, int& tz) {
            tx0 = (b % a.nbx) * a.T;
            ty = (b / a.nbx) % g.rdims[1];
            tz = b / (a.nbx * g.rdims[1]);
        };
        // G -> shared -> the batch's partial gradient (the next writer of
        // the G copy's area, the voxel phase, starts after a compute
        // barrier).  The batch's score and count: each warp's tree sum into
        // shared memory before the barrier that follows the G copy, then
        // thread 0 adds the eight in warp order (no barrier of its own;
        // the slots are rewritten only a batch later).
        auto finish_batch = [&](int b) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                sc += __shfl_down_sync (0xffffffffu, sc, o);
                cnt += __shfl_down_sync (0xffffffffu, cnt, o);
            }
            if (x.lane == 0) {
                sh_v[x.warp] = sc;
                sh_n[x.warp] = cnt;
            }
            sc = 0.0;
            cnt = 0;
            dump_g (a, x);
            tc_fence_before ();
            cbar ();
            if (x.tid == 0) {
                double v = 0.0;
                int n = 0;
                for (int w = 0; w < TC_WARPS; w++) {
                    v += sh_v[w];
                    n += sh_n[w];
                }
                a.score_part[b] = v;
                a.count_part[b] = n;
            }
            gather_knots (a, x, b);
        };
        if (a.mblk == 1 && nb_local > 0) {
            const VoxelSlot vs0 = voxel_slot (a, x, 0);
            // Pipelined: the adjoint of batch b runs while batch b+1 is
            // staged; the forward of b+1 runs while batch b is gathered.
            int tx0, ty, tz;
            coords (blockIdx.x, tx0, ty, tz);
            stage_batch (a, x, tx0, ty, tz);
            cbar ();
            build_c (a, x);
            warp_arrive (x, &s_bar[0]);
            for (int i = 0; i < nb_local; i++) {
                const int b = blockIdx.x + i * gridDim.x;
                coords (b, tx0, ty, tz);
                if (!cwait (a, x, &s_bar[2], ph_d, abort_flag, 1)) break;
                if constexpr (MODE >= TC_MI_GRAD) {
                    voxel_phase_axis<MODE> (a, x, vs0, tx0, ty, tz, sc, cnt);
                } else if (a.axis) {
                    voxel_phase_axis<MODE> (a, x, vs0, tx0, ty, tz, sc, cnt);
                } else {
                    voxel_phase_xline<MODE> (a, x, vs0, tx0, ty, tz, sc, cnt);
                }
                if (!tc_hist_mode (MODE)) warp_arrive (x, &s_bar[1]);
                if (i + 1 < nb_local) {
                    int nx0, ny, nz;
                    coords (b + gridDim.x, nx0, ny, nz);
                    stage_batch (a, x, nx0, ny, nz);
                    cbar ();
                    build_c (a, x);
                    warp_arrive (x, &s_bar[0]);
                }
                if (tc_hist_mode (MODE)) continue;
                if (!cwait (a, x, &s_bar[3], ph_g, abort_flag, 2)) break;
                finish_batch (b);
            }
        } else {
            // Tiles of more than 128 voxels: Q is reloaded per 128-voxel
            // block, so batches run one after another.
            for (int i = 0; i < nb_local; i++) {
                const int b = blockIdx.x + i * gridDim.x;
                int tx0, ty, tz;
                coords (b, tx0, ty, tz);
                stage_batch (a, x, tx0, ty, tz);
                cbar ();
                build_c (a, x);
                bool ok = true;
                for (int mb = 0; mb < a.mblk && ok; mb++) {
                    const uint4* src = a.qimg + (size_t) mb * 2048;
                    for (int o = x.tid; o < 2048; o += TC_THREADS) {
                        ((uint4*) (x.sm + SM_Q))[o] = src[o];
                    }
                    warp_arrive (x, &s_bar[0]);
                    ok = cwait (a, x, &s_bar[2], ph_d, abort_flag, 1);
                    if (!ok) break;
                    voxel_phase<MODE> (a, x, voxel_slot (a, x, mb), tx0,
                        ty, tz, sc, cnt);
                    if (tc_hist_mode (MODE)) continue;
                    warp_arrive (x, &s_bar[1]);
                    ok = cwait (a, x, &s_bar[3], ph_g, abort_flag, 2);
                }
                if (!ok) break;
                if (!tc_hist_mode (MODE)) finish_batch (b);
            }
        }
        if constexpr (tc_hist_mode (MODE)) {
            // the CTA's histograms and count into the global ones (integer
            // sums: the order does not matter)
            cbar ();
            const int B = a.bins, nh = 2 * B + B * B;
            const unsigned long long* h = (const unsigned long long*) (x.sm + SM_DC);
            for (int i = x.tid; i < nh; i += TC_THREADS) {
                unsigned long long v = h[i];
                if (MODE == TC_PZ_HIST && i < 2 * B) {
                    v = 0;                          // marginals: score kernel
                } else if (i >= B && i < 2 * B) {   // moving: joint column sum
                    v = 0;
                    for (int fb = 0; fb < B; fb++) v += h[2 * B + fb * B + (i - B)];
                }
                if (v) atomicAdd (&a.hist[i], v);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                cnt += __shfl_down_sync (0xffffffffu, cnt, o);
            }
            if (x.lane == 0 && cnt) {
                atomicAdd (&a.hist[nh], (unsigned long long) cnt);
            }
        }
    }

    tc_fence_before ();
    __syncthreads ();
    if (mma_warp) {
        tmem_dealloc (x.taddr, TC_TMEM_COLS);
    }
}

bool
tc_plan (const BspGeom& g, TcPlan* p, int ctas_per_sm, int sm_count,
    int extra_row_batches)
{
    int V = g.vpr[0] * g.vpr[1] * g.vpr[2];
    int mblk = (V + 127) / 128;
    if (mblk > TC_MAX_MBLK) return false;
    // batches per row of tiles: the fewest that keep T <= TC_TMAX, plus the
    // autotuner's extra; a row split into several batches needs T >= 3
    // (the finish kernel's gather assumes a knot meets at most two)
    int nb_row = (g.rdims[0] + TC_TMAX - 1) / TC_TMAX + extra_row_batches;
    if (nb_row > g.rdims[0] || (nb_row > 1 && (g.rdims[0] + nb_row - 1) / nb_row < 3)) {
        return false;
    }
    int T = (g.rdims[0] + nb_row - 1) / nb_row;      // balanced batches
    p->bx = T;
    p->mblk = mblk;
    p->n_mma = ((3 * T + 15) / 16) * 16;
    p->nbatches = nb_row * g.rdims[1] * g.rdims[2];
    p->smem = SM_TOTAL + 1024;
    p->tmem_cols = TC_TMEM_COLS;
    p->threads = TC_BLOCK;
    p->grid = std::min (p->nbatches, std::max (1, ctas_per_sm) * sm_count);
    return true;
}

// Q image in global memory: per M block, hi then lo, each the exact
// 128-row x 64-slot 128B-swizzled shared-memory image (16 KB).
int
tc_build_tables (const BspGeom& g, const TcPlan& p, void** d_qlut)
{
    const int vx = g.vpr[0], vy = g.vpr[1], vz = g.vpr[2];
    const int V = vx * vy * vz;
    std::vector<float> lut[3];
    for (int d = 0; d < 3; d++) {
        int n = g.vpr[d];
        lut[d].resize (4 * n);
        for (int j = 0; j < 4; j++) {
            for (int v = 0; v < n; v++) {
                float i = (float) v / n;
                double r = 0;
                switch (j) {
                case 0: r = (1.0/6.0) * (- 1.0 * i*i*i + 3.0 * i*i - 3.0 * i + 1.0); break;
                case 1: r = (1.0/6.0) * (+ 3.0 * i*i*i - 6.0 * i*i + 4.0); break;
                case 2: r = (1.0/6.0) * (- 3.0 * i*i*i + 3.0 * i*i + 3.0 * i + 1.0); break;
                case 3: r = (1.0/6.0) * (+ 1.0 * i*i*i); break;
                }
                lut[d][v * 4 + j] = (float) r;
            }
        }
    }
    size_t bytes = (size_t) p.mblk * 32768;
    std::vector<uint8_t> img (bytes, 0);
    for (int v = 0; v < p.mblk * 128; v++) {
        int mb = v / 128, vl = v % 128;
        uint8_t* hi = img.data () + (size_t) mb * 32768;
        uint8_t* lo = hi + 16384;
        for (int m = 0; m < 64; m++) {
            float qv = 0.f;
            if (v < V) {
                int lx = v % vx, ly = (v / vx) % vy, lz = v / (vx * vy);
                int i = m & 3, j = (m >> 2) & 3, k = m >> 4;
                float C = lut[2][lz * 4 + k];
                float B = lut[1][ly * 4 + j] * C;
                qv = lut[0][lx * 4 + i] * B;
            }
            __nv_bfloat16 h = __float2bfloat16_rn (qv);
            __nv_bfloat16 l = __float2bfloat16_rn (qv - __bfloat162float (h));
            uint32_t off = sw128_offset (vl, m, 128);
            *(unsigned short*) (hi + off) = __bfloat16_as_ushort (h);
            *(unsigned short*) (lo + off) = __bfloat16_as_ushort (l);
        }
    }
    if (cudaMalloc (d_qlut, bytes) != cudaSuccess) return B200BSP_E_OOM;
    if (cudaMemcpy (*d_qlut, img.data (), bytes, cudaMemcpyHostToDevice)
        != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    return B200BSP_OK;
}

// Kernel arguments common to every mode; returns whether the axis-aligned
// voxel phase applies: diagonal step and projection, one 128-voxel block
// per tile, rounds whose field copy and position tables fit the C and
// knot-block areas, and divisors >= 2 for the multiply-high reciprocals.
static bool
tc_args (const BspGeom& g, const TcPlan& p, TcArgs& a)
{
    a = TcArgs ();
    a.g = g;
    a.wait_limit = TC_WAIT_LIMIT;
    a.T = p.bx;
    a.N = p.n_mma;
    a.mblk = p.mblk;
    a.V = g.vpr[0] * g.vpr[1] * g.vpr[2];
    a.T0 = (a.T + 1) / 2;
    a.W = g.vpr[0] * a.T0;
    a.plane = a.W * g.vpr[1] * g.vpr[2];
    bool diag = true;
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) {
            if (i != j && (g.fstep[3 * i + j] != 0.f || g.mproj[3 * i + j] != 0.f)) {
                diag = false;
            }
        }
    }
    a.mW = a.W >= 2 ? 0xFFFFFFFFu / (unsigned) a.W + 1u : 0u;
    a.mvx = g.vpr[0] >= 2 ? 0xFFFFFFFFu / (unsigned) g.vpr[0] + 1u : 0u;
    a.nbx = (g.rdims[0] + p.bx - 1) / p.bx;
    a.nbatches = p.nbatches;
    return diag && p.mblk == 1 && g.vpr[0] >= 2 && a.W >= 2
        && 12 * a.plane <= SM_C_BYTES
        && 2 * a.W + 4 * g.vpr[1] * g.vpr[2] <= SM_S_FLOATS;
}

template <int MODE>
static cudaError_t
launch_mode (const TcPlan& p, const TcArgs& a, cudaStream_t st)
{
    auto k = mse_tc_kernel<MODE>;
    cudaError_t e = set_max_dynamic_smem ((const void*) k, (int) p.smem);
    if (e != cudaSuccess) return e;
    k<<<p.grid, TC_BLOCK, p.smem, st>>> (a);
    return cudaGetLastError ();
}

cudaError_t
launch_mse_tc (const BspGeom& g, const TcPlan& p, int grad_mode,
    const float* fimg, const float* mimg, const float* mgrad,
    const float4* mgrad4, const float* coeff, const void* qimg, float* part,
    double* score_part, int* count_part, int* err, unsigned wait_limit,
    cudaStream_t st)
{
    TcArgs a;
    a.axis = tc_args (g, p, a) && (grad_mode == 1 || mgrad4 != nullptr);
    if (wait_limit > 0) a.wait_limit = wait_limit;
    a.mgrad4 = mgrad4;
    a.fimg = fimg; a.mimg = mimg; a.mgrad = mgrad; a.coeff = coeff;
    a.qimg = (const uint4*) qimg;
    a.part = part; a.score_part = score_part; a.count_part = count_part;
    a.err = err;
    return grad_mode == 0 ? launch_mode<TC_MSE_NEAREST> (p, a, st)
                          : launch_mode<TC_MSE_LINEAR> (p, a, st);
}

// MI on the tensor-core kernel: the axis-aligned voxel phase (one block per
// tile) or the general one (several 128-voxel blocks per tile); tiles of
// one block in rotated geometry take the FP32 passes.
bool
tc_mi_supported (const BspGeom& g, const TcPlan& p, int bins)
{
    TcArgs a;
    const bool axis = tc_args (g, p, a);
    return (axis || p.mblk > 1)
        && (2 * bins + bins * bins) * 8 <= 2 * DC_HALF + DC_TAIL;
}

cudaError_t
launch_mi_tc (const BspGeom& g, const TcPlan& p, bool hist_pass,
    const TcMiArgs& mi, const float* coeff, const void* qimg, float* part,
    double* score_part, int* count_part, int* err, cudaStream_t st)
{
    TcArgs a;
    a.axis = tc_args (g, p, a);
    if (!a.axis && p.mblk == 1) return cudaErrorInvalidValue;
    a.coeff = coeff;
    a.qimg = (const uint4*) qimg;
    a.part = part; a.score_part = score_part; a.count_part = count_part;
    a.err = err;
    a.fbin = mi.fbin; a.mbin = mi.mbin; a.bins = mi.bins;
    a.mi_lut = mi.lut; a.mi_nvf = mi.nvf; a.hist = mi.hist;
    if (mi.parzen) {
        a.mimg = mi.mimg;
        a.pz_mmin = mi.m_min;
        a.pz_mdelta = mi.m_delta;
        return hist_pass ? launch_mode<TC_PZ_HIST> (p, a, st)
                         : launch_mode<TC_PZ_GRAD> (p, a, st);
    }
    return hist_pass ? launch_mode<TC_MI_HIST> (p, a, st)
                     : launch_mode<TC_MI_GRAD> (p, a, st);
}

} // namespace b200
