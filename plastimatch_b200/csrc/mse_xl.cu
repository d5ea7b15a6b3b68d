// Tensor-core (tcgen05) form of the MSE score + gradient, x-lane layout.
//
// One batch is a row of T tiles along x at tile coordinates (ty, tz): its
// voxels are the block x in [0, T vx) x rows rho = (ly, lz).  The B-spline
// field there factors into two contractions (the basis is a tensor product,
// src/base/bspline_interpolate.cxx:78-110):
//   R_c[xk][rho]  = sum_{j,k} by[ly][j] bz[lz][k] C_c[xk][j][k]   (y and z)
//   D[x][(c,rho)] = sum_xk   Bx[x][xk] R_c[xk][rho]               (x)
// with xk the T + 3 knots of the batch along x and Bx the banded x basis
// (bx[x mod vx][xk - x div vx], zero off the band), shared by every batch.
// The x contraction runs on the tensor cores with the voxel x as the MMA's
// M dimension, so TMEM lane = voxel x: each thread of a warp owns one x of
// 32 consecutive ones and walks the rows rho of the batch, reading its
// field values straight from TMEM (no transposition through shared memory)
// while a warp's trilinear gathers and fixed-image reads stay coalesced.
// The adjoint of the condense (bspline_update_sets_b,
// src/register/bspline.cxx:347-374) runs the other way:
//   Rg[(c,xk)][rho] = sum_x Bx[x][xk] DCDV_c[x][rho]               (tensor cores)
//   G_c[xk][j][k]   = sum_rho by[ly][j] bz[lz][k] Rg[(c,xk)][rho]  (CUDA cores)
// The adjoint runs one MMA per component; its M dimension is four copies of
// the 32 knots (the basis table holds Bx four times side by side), so
// every TMEM lane quarter receives all of Rg_c and each of its lanes owns
// one knot for the y/z contraction -- done by lane quarter 3's warps when
// that quarter has no samples (at vox_per_rgn 5 a batch spans 90 voxels),
// else by the other quarters'.  G_c is the batch's partial gradient of its
// (T + 3) x 4 x 4 knot footprint; the finish kernel sums the partials of
// each knot in a fixed order (no float atomics).
//
// Precision: every tensor-core operand is split x = hi + lo (two bf16) and
// each product takes hi*hi + hi*lo + lo*hi with f32 accumulation in TMEM
// (~16 significant bits); the y/z contractions, positions, trilinear
// samples and differences are f32 on the CUDA cores.
//
// CTA (one per SM): 15 compute warps + 1 tensor-core warp (warp 15).  Warp
// w reads TMEM lane quarter w % 4 (x = 32 (w % 4) + lane); the warps of a
// quarter (four, three in the last) split the batch's rows.  The fourth
// quarter's compute warps also compute the y/z contraction of the step
// three ahead; the other three quarters' warps do the adjoint y/z
// contraction of the previous step.  Steps (batch, chunk of
// rows) are software-pipelined through triple-buffered R operands and
// double-buffered dc/dv operands and TMEM accumulators, with mbarrier
// handshakes:
//   B2 ready (R of step s)  -> MMA x-forward(s)  -> D full(s)
//   D full(s)               -> voxel phase(s)    -> DC ready(s)
//   DC ready(s)             -> MMA x-adjoint(s)  -> Rg full(s)
//   Rg full(s)              -> y/z adjoint(s) during step s + 1.
// Every wait is bounded (a runtime poll limit); on expiry the kernel raises
// the context's error flag and every warp leaves its loop.
#include <algorithm>
#include <vector>

#include <cuda_bf16.h>

#include "bsp_common.cuh"
#include "kernels.cuh"
#include "tc_ptx.cuh"
#include "../../include/plastimatch_b200.h"

namespace b200 {

namespace {

// 16 warps: warp 15 (lane quarter 3, the fourth warp of it) issues the
// MMAs, warps 0..14 compute; 512 threads leave 128 registers a thread
constexpr int XL_CW = 15;                    // compute warps
constexpr int XL_THREADS = 32 * XL_CW;
constexpr int XL_BLOCK = XL_THREADS + 32;    // + the tensor-core warp
constexpr int XL_KMAX = 32;                  // knots per batch along x
constexpr int XL_RC = 32;                    // rows per component block
constexpr int XL_N = 3 * XL_RC;              // MMA N: (c, rho)

// Shared memory (offsets from a 1024-byte aligned base).
constexpr int XS_TAB = 0;          // basis table, bf16 hi (32 KB) then lo
constexpr int XS_TAB_LO = 32768;
constexpr int XL_NB2 = 3;          // R operand buffers (steps of look-ahead)
constexpr int XS_B2 = 65536;       // R operand, XL_NB2 x (hi 8 KB, lo 8 KB)
constexpr int XS_B2_BUF = 16384;
constexpr int XS_B2_LO = 8192;
constexpr int XS_DC = XS_B2 + XL_NB2 * XS_B2_BUF;  // dc/dv operand, 2 x (hi, lo)
constexpr int XS_DC_BUF = 49152;
constexpr int XS_DC_LO = 24576;
constexpr int XS_DC_ATOM = XL_N * 128;         // 64-voxel K atom of one half
constexpr int XS_ROWS = XS_DC + 2 * XS_DC_BUF; // per-warp row table
constexpr int XL_ROWS_MAX = 12;    // rows of a warp (groups of four, 3-way split)
constexpr int XS_ROWS_BYTES = XL_CW * XL_ROWS_MAX * 16;
constexpr int XS_LUT = XS_ROWS + XS_ROWS_BYTES;   // by[vy][4], bz[vz][4]
constexpr int XS_LUT_FLOATS = 2 * 64 * 4;
constexpr int XS_TOTAL = XS_LUT + XS_LUT_FLOATS * 4;
static_assert (XS_TOTAL + 1024 <= 227 * 1024, "shared memory");

// TMEM columns: D[buf] at 128 buf, Rg[buf] at 256 + 128 buf.
constexpr int XT_COLS = 512;
constexpr int XT_D = 0;
constexpr int XT_RG = 256;

// What the kernel computes (template argument MODE).
constexpr int XM_MSE_NEAREST = 0;   // MSE, moving gradient at the nearest voxel
constexpr int XM_MSE_LINEAR = 1;    // MSE, trilinear moving gradient
constexpr int XM_MI_GRAD = 2;       // Mattes MI pass 2, PVI-8 factor table
constexpr int XM_MI_HIST = 3;       // Mattes MI pass 1, PVI-8 histograms
constexpr int XM_PZ_GRAD = 4;       // Parzen-window MI pass 2
constexpr int XM_PZ_HIST = 5;       // Parzen-window MI pass 1

__host__ __device__ constexpr bool
xl_hist_mode (int m)
{
    return m == XM_MI_HIST || m == XM_PZ_HIST;
}

__host__ __device__ constexpr bool
xl_mse_mode (int m)
{
    return m == XM_MSE_NEAREST || m == XM_MSE_LINEAR;
}

constexpr float XL_MI_WUNIT = 16777216.0f;   // histogram weights in 2^-24

// Barriers.
constexpr int XB_B2 = 0;       // + buf: R operand written (3 warp arrivals)
constexpr int XB_DC = XL_NB2;  // + buf: dc/dv written, D read (15 arrivals)
constexpr int XB_D = XB_DC + 2;    // + buf: x-forward MMA done (commit)
constexpr int XB_RG = XB_D + 2;    // + buf: x-adjoint MMA done (commit)
constexpr int XB_DRAIN = XB_RG + 2;    // every issued MMA done
// Longest sleep between two polls of a wait (the sleeps double from 32 ns):
// the compute warps' waits, the look-ahead warps', the tensor-core
// thread's wait for an R operand and for a step's dc/dv.
constexpr unsigned XL_SLEEP_COMPUTE = 128;
constexpr unsigned XL_SLEEP_AHEAD = 1024;
constexpr unsigned XL_SLEEP_B2 = 64;
constexpr unsigned XL_SLEEP_DC = 256;

}  // namespace

// n / d for 0 <= n < 2^31 by a multiply and a shift (Granlund and
// Montgomery, "Division by invariant integers using multiplication", PLDI
// 1994, round-up multiplier m = floor(2^32 (2^l - d) / d) + 1 with
// l = ceil(log2 d)).
struct XlDiv {
    uint32_t mul, shift;
};

static XlDiv
xl_div (uint32_t d)
{
    uint32_t l = 0;
    while ((1ull << l) < d) l++;
    XlDiv v;
    v.mul = (uint32_t) ((((1ull << 32) * ((1ull << l) - d)) / d) + 1);
    v.shift = l;
    return v;
}

__device__ __forceinline__ int
xl_q (int n, XlDiv v)
{
    return (int) ((__umulhi ((uint32_t) n, v.mul) + (uint32_t) n) >> v.shift);
}

struct XlArgs {
    BspGeom g;
    int T, KX, nbx, nbatches;
    int nlz, nch;            // z planes per row chunk, chunks per batch
    XlDiv d_nch, d_nbx, d_rdy, d_vy;   // by nch, nbx, rdims[1], vpr[1]
    unsigned wait_limit;
    int withhold;            // testing aid: the tensor-core warp issues
                             // nothing, so the first waits run out
    const float* fimg;
    const float* mimg;
    const float* mgrad;      // xyz interleaved (nearest-voxel mode)
    const float* coeff;
    const uint4* tab;        // the basis table image (64 KB)
    const float* luts;       // bx[vx][4], by[vy][4], bz[vz][4]
    float* part;             // [batch][c][xk + KX (j + 4 k)]
    double* score_part;      // [batch]
    int* count_part;         // [batch]
    int* err;
    // Mattes MI modes: bin images, bins, the pass-2 factor table [fixed
    // bin][moving bin], the voxel count (float; Parzen: [1] the pass-2
    // scale), the global histograms f[B], m[B], j[B*B], count; Parzen's
    // moving value -> window centre
    const uint8_t* fbin;
    const uint8_t* mbin;
    int bins;
    const float* mi_lut;
    const float* mi_nvf;
    unsigned long long* hist;
    float pz_mmin, pz_mdelta;
};

namespace {

struct XlCtx {
    uint8_t* sm;
    uint32_t sm_base;
    uint32_t taddr;
    int warp, lane, q, j4;
};

__device__ __forceinline__ uint32_t
split_word (float x)
{
    // bf16 hi in the low half-word, bf16 lo (x - hi) in the high one
    __nv_bfloat16 h = __float2bfloat16_rn (x);
    __nv_bfloat16 l = __float2bfloat16_rn (x - __bfloat162float (h));
    return (uint32_t) __bfloat16_as_ushort (h)
        | ((uint32_t) __bfloat16_as_ushort (l) << 16);
}

// Polls of one thread on an mbarrier phase with exponential back-off
// (sleeps of 32, 64, ... ns, at most cap): true once the phase completes,
// false after `limit` polls or once another warp has given up.
__device__ __forceinline__ bool
xl_poll (uint64_t* bar, uint32_t ph, unsigned cap, unsigned limit,
    volatile int* s_abort)
{
    unsigned t = 32;
    for (uint32_t n = 0; n < limit && !*s_abort; n++) {
        if (mbar_try_wait (bar, ph)) return true;
        __nanosleep (t);
        t = min (2 * t, cap);
    }
    return false;
}

// Bounded wait of one warp on an mbarrier phase: lane 0 polls, gives up
// after the limit or once another warp has given up.
__device__ __forceinline__ bool
xl_wait (const XlArgs& a, const XlCtx& x, uint64_t* bar, uint32_t ph,
    volatile int* s_abort, int code, unsigned cap)
{
    if (x.lane == 0) {
        const bool ok = xl_poll (bar, ph, cap, a.wait_limit, s_abort);
        if (!ok) {
            *s_abort = 1;
            atomicExch (a.err, code);
        }
    }
    __syncwarp ();
    return *s_abort == 0;
}

// Step s -> batch, chunk and the batch's tile coordinates.
struct XlStep {
    int b, ch, tx0, ty, tz, lz0, nlz;
};

__device__ __forceinline__ XlStep
xl_step (const XlArgs& a, int s)
{
    XlStep t;
    const int i = xl_q (s, a.d_nch);
    t.ch = s - i * a.nch;
    t.b = blockIdx.x + i * gridDim.x;
    const int q1 = xl_q (t.b, a.d_nbx);         // row of tiles
    t.tx0 = (t.b - q1 * a.nbx) * a.T;
    t.tz = xl_q (q1, a.d_rdy);
    t.ty = q1 - t.tz * a.g.rdims[1];
    t.lz0 = t.ch * a.nlz;
    t.nlz = min (a.nlz, a.g.vpr[2] - t.lz0);
    return t;
}

// y/z forward contraction of one step into the R operand buffer (K = xk
// rows, N = (c, rho) columns, MN-major, 128-byte swizzle): thread (c, xk)
// of the fourth lane quarter's warps 0..2.  The rows are unrolled (VY
// known at compile time) and stored two at a time (rows rho, rho + 1 of
// one component share a 32-bit word of the operand).
template <int VY>
__device__ __forceinline__ void
xl_yz_forward_t (const XlArgs& a, const XlCtx& x, const XlStep& t, int buf)
{
    constexpr int NLZ = XL_RC / VY;
    const BspGeom& g = a.g;
    const int c = x.j4, xk = x.lane;
    if (c >= 3) return;
    const float* by = (const float*) (x.sm + XS_LUT);
    const float* bz = by + 4 * VY;
    const int kx = t.tx0 + xk;
    const bool live = xk < a.KX && kx < g.cdims[0];
    float cf[16];
#pragma unroll
    for (int k = 0; k < 4; k++) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int knot = ((t.tz + k) * g.cdims[1] + t.ty + j) * g.cdims[0]
                + (live ? kx : 0);
            cf[4 * k + j] = live ? __ldg (a.coeff + 3 * knot + c) : 0.f;
        }
    }
    uint8_t* hi = x.sm + XS_B2 + buf * XS_B2_BUF;
    const uint32_t rowoff = (uint32_t) ((xk >> 3) * 1024 + (xk & 7) * 128);
    const int nrc = VY * t.nlz;
    auto word_off = [&](int n) {
        return (uint32_t) ((n >> 6) * 4096) + rowoff
            + (uint32_t) ((((n & 63) >> 3) ^ (xk & 7)) << 4)
            + (uint32_t) ((n & 7) * 2);
    };
    uint32_t w_even = 0;
#pragma unroll
    for (int l = 0; l < NLZ; l++) {
        if (l < t.nlz) {
            const float* bzl = bz + 4 * (t.lz0 + l);
            float z[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                z[j] = bzl[0] * cf[j] + bzl[1] * cf[4 + j] + bzl[2] * cf[8 + j]
                    + bzl[3] * cf[12 + j];
            }
#pragma unroll
            for (int ly = 0; ly < VY; ly++) {
                const int rho = ly + VY * l;
                const float r = by[4 * ly] * z[0] + by[4 * ly + 1] * z[1]
                    + by[4 * ly + 2] * z[2] + by[4 * ly + 3] * z[3];
                const uint32_t w = split_word (r);
                if ((rho & 1) == 0) {
                    w_even = w;
                    if (rho + 1 == nrc) {          // a last, unpaired row
                        const uint32_t off = word_off (c * XL_RC + rho);
                        *(unsigned short*) (hi + off) = (unsigned short) w;
                        *(unsigned short*) (hi + XS_B2_LO + off)
                            = (unsigned short) (w >> 16);
                    }
                } else {
                    const uint32_t off = word_off (c * XL_RC + rho - 1);
                    *(uint32_t*) (hi + off) = __byte_perm (w_even, w, 0x5410);
                    *(uint32_t*) (hi + XS_B2_LO + off)
                        = __byte_perm (w_even, w, 0x7632);
                }
            }
        }
    }
}

// The look-ahead warps' L2 prefetch of step t's fixed-image rows (the only
// reads of the voxel phase whose addresses do not depend on the
// displacement), one 128-byte line a thread: thread i of the 96 takes
// lines i, i + 96, ...
__device__ __forceinline__ void
xl_prefetch_fixed (const XlArgs& a, const XlCtx& x, const XlStep& t)
{
    const BspGeom& g = a.g;
    const int i = 32 * x.j4 + x.lane;
    const int x0 = g.roi_off[0] + g.vpr[0] * t.tx0;
    const int x1 = min (x0 + a.T * g.vpr[0], g.roi_off[0] + g.roi_dim[0]);
    const int y0 = g.roi_off[1] + g.vpr[1] * t.ty;
    const int y1 = min (y0 + g.vpr[1], g.roi_off[1] + g.roi_dim[1]);
    const int z0 = g.roi_off[2] + g.vpr[2] * t.tz + t.lz0;
    const int z1 = min (z0 + t.nlz, g.roi_off[2] + g.roi_dim[2]);
    if (x1 <= x0 || y1 <= y0 || z1 <= z0) return;
    const size_t fdx = g.fdim[0], fdxy = (size_t) g.fdim[0] * g.fdim[1];
    // lines of a row: from the line holding x0 to the one holding x1 - 1
    const uintptr_t base = (uintptr_t) a.fimg;
    const int ny = y1 - y0;
    const int nrow = ny * (z1 - z0);
    // every row spans the same number of lines or one more; take the most
    const int nl = (int) ((4 * (x1 - x0) + 127) >> 7) + 1;
    for (int r = i; r < nrow * nl; r += 96) {
        const int row = r / nl, l = r - row * nl;
        const size_t o = ((size_t) (z0 + row / ny) * fdxy
            + (size_t) (y0 + row % ny) * fdx + x0) * 4;
        const uintptr_t first = (base + o) & ~(uintptr_t) 127;
        const uintptr_t line = first + 128 * (uintptr_t) l;
        if (line < base + o + 4 * (size_t) (x1 - x0)) {
            asm volatile ("prefetch.global.L2 [%0];" :: "l"(line));
        }
    }
}

__device__ __forceinline__ void
xl_yz_forward (const XlArgs& a, const XlCtx& x, const XlStep& t, int buf)
{
    switch (a.g.vpr[1]) {
    case 3: xl_yz_forward_t<3> (a, x, t, buf); break;
    case 4: xl_yz_forward_t<4> (a, x, t, buf); break;
    case 5: xl_yz_forward_t<5> (a, x, t, buf); break;
    case 6: xl_yz_forward_t<6> (a, x, t, buf); break;
    case 7: xl_yz_forward_t<7> (a, x, t, buf); break;
    case 8: xl_yz_forward_t<8> (a, x, t, buf); break;
    case 9: xl_yz_forward_t<9> (a, x, t, buf); break;
    case 10: xl_yz_forward_t<10> (a, x, t, buf); break;
    default: break;                  // the plan admits no other vy
    }
}

// y/z adjoint contraction of one step for knot plane k, given the
// thread's row of Rg_c (rg, 32 columns): accumulates G[j] over the batch's
// chunks.
template <int VY>
__device__ __forceinline__ void
xl_yz_adjoint_t (const XlArgs& a, const XlCtx& x, const XlStep& t,
    const float rg[32], int k, float G[4])
{
    constexpr int NLZ = XL_RC / VY;
    const float* by = (const float*) (x.sm + XS_LUT);
    const float* bz = by + 4 * VY;
    float z[VY];
#pragma unroll
    for (int ly = 0; ly < VY; ly++) z[ly] = 0.f;
#pragma unroll
    for (int l = 0; l < NLZ; l++) {
        if (l < t.nlz) {
            const float w = bz[4 * (t.lz0 + l) + k];
#pragma unroll
            for (int ly = 0; ly < VY; ly++) z[ly] = fmaf (w, rg[ly + VY * l], z[ly]);
        }
    }
#pragma unroll
    for (int ly = 0; ly < VY; ly++) {
#pragma unroll
        for (int j = 0; j < 4; j++) G[j] = fmaf (by[4 * ly + j], z[ly], G[j]);
    }
}

__device__ __forceinline__ void
xl_yz_adjoint (const XlArgs& a, const XlCtx& x, const XlStep& t,
    const float rg[32], int k, float G[4])
{
    switch (a.g.vpr[1]) {
    case 3: xl_yz_adjoint_t<3> (a, x, t, rg, k, G); break;
    case 4: xl_yz_adjoint_t<4> (a, x, t, rg, k, G); break;
    case 5: xl_yz_adjoint_t<5> (a, x, t, rg, k, G); break;
    case 6: xl_yz_adjoint_t<6> (a, x, t, rg, k, G); break;
    case 7: xl_yz_adjoint_t<7> (a, x, t, rg, k, G); break;
    case 8: xl_yz_adjoint_t<8> (a, x, t, rg, k, G); break;
    case 9: xl_yz_adjoint_t<9> (a, x, t, rg, k, G); break;
    case 10: xl_yz_adjoint_t<10> (a, x, t, rg, k, G); break;
    default: break;                  // the plan admits no other vy
    }
}

// The thread's row of Rg_c from its lane quarter (every quarter holds all
// of it).
__device__ __forceinline__ void
xl_load_rg (const XlCtx& x, int buf, int c, float rg[32])
{
    tmem_ld32_wait (x.taddr + ((uint32_t) (32 * x.q) << 16) + XT_RG
        + 128 * buf + XL_RC * c, rg);
}

// Mattes MI pass 2 at one sample (bspline_mi_pvi_8_dc_dv_dcos,
// src/register/bspline_mi.txx:9-120): the derivative of each PVI-8 corner
// weight along x, y, z times that corner's factor f[fixed bin][corner bin],
// negated, divided by the voxel count, then projected by the moving
// image's projection matrix in place (each row sees the rows above already
// updated, as the reference does).  w2: the upper-corner fractions.
__device__ __forceinline__ void
xl_mi_dc_dv (const XlArgs& a, const float w2[3], int fb, const int mb[8],
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

// Mattes MI pass 1 at one sample: the PVI-8 corner weights as integers in
// 2^-24 units (sums independent of their order), corners with equal moving
// bins merged; the first two (fixed, moving) pairs of every lane combine
// across the warp (match + reduce) so one lane per distinct pair updates
// the shared joint histogram, further pairs go straight to the shared
// atomics; the fixed histogram counts each first-pair group's voxels (the
// moving one is the joint's column sums, taken at the flush).  Every lane
// of the warp calls this (warp collectives).
__device__ __forceinline__ void
xl_mi_hist_add (const XlArgs& a, unsigned long long* hf, bool live,
    const float w2[3], int fb, const int mb[8], int lane, int& cnt)
{
    const int B = a.bins;
    unsigned long long* hj = hf + 2 * B;
    const float* l2 = w2;
    const float l1[3] = {1.f - w2[0], 1.f - w2[1], 1.f - w2[2]};
    const float w[8] = {l1[0] * l1[1] * l1[2], l2[0] * l1[1] * l1[2],
        l1[0] * l2[1] * l1[2], l2[0] * l2[1] * l1[2], l1[0] * l1[1] * l2[2],
        l2[0] * l1[1] * l2[2], l1[0] * l2[1] * l2[2], l2[0] * l2[1] * l2[2]};
    unsigned int q[8];
#pragma unroll
    for (int k = 0; k < 8; k++) q[k] = __float2uint_rn (w[k] * XL_MI_WUNIT);
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
        const int key = fb * B + mb1;
        const unsigned peers = __match_any_sync (live_mask, key);
        const unsigned sum = __reduce_add_sync (peers, q1);
        if (lane == __ffs (peers) - 1) {
            atomicAdd (&hj[key], (unsigned long long) sum);
            atomicAdd (&hf[fb], (unsigned long long) __popc (peers));
        }
    }
    const unsigned two_mask = __ballot_sync (0xffffffffu, two);
    if (two) {
        const int key = fb * B + mb2;
        const unsigned peers = __match_any_sync (two_mask, key);
        const unsigned sum = __reduce_add_sync (peers, q2);
        if (lane == __ffs (peers) - 1) {
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

// Parzen-window MI pass 1 at one sample: the cubic window's four weights
// at the moving value's window centre u (2^-24 units) into the fixed bin's
// row of the shared joint histogram; lanes with the same (fixed bin, first
// window bin) combine across the warp first.  Every lane calls this.
__device__ __forceinline__ void
xl_pz_hist_add (const XlArgs& a, unsigned long long* hf, bool live, int fb,
    float u, int lane, int& cnt)
{
    const int B = a.bins;
    unsigned long long* hj = hf + 2 * B;
    const int k0 = parzen_first_bin (u, B);
    unsigned int q[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        q[j] = __float2uint_rn (bspline3f ((float) (k0 + j) - u) * XL_MI_WUNIT);
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

// Parzen-window MI pass 2 at one sample: 1/(N delta_m) times the sum over
// the window's bins of beta3'(k - u) log(p(f, k) / p_m(k)) (the factor
// table), times the world gradient of the trilinear interpolant (proj^T
// times the index gradient; 0 along an axis the clamp holds).
__device__ __forceinline__ void
xl_pz_dc_dv (const XlArgs& a, float u, int fb, const float w2[3],
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

// The voxel phase of one step for warp (quarter q, rows part j4): the
// warp's rows [ra, rb) of the chunk, four at a time (their field values as
// three 4-column TMEM loads); the MSE modes issue the gathers of all four
// samples before using any, the MI modes two at a time.
template <int MODE, bool AXIS, bool ROI>
__device__ __forceinline__ void
xl_voxel (const XlArgs& a, const XlCtx& x, const XlStep& t, int buf,
    float& scf, int& cnt)
{
    constexpr int NS = xl_mse_mode (MODE) ? 4 : 2;
    const BspGeom& g = a.g;
    const int vy = g.vpr[1];
    const int nrc = vy * t.nlz;
    // the quarter's rows split among its compute warps (three in quarter
    // 3) in whole groups of four, so that one group at most is partial
    const int parts = x.q == 3 ? 3 : 4;
    const int ng = (nrc + 3) >> 2;
    const int ra = 4 * (ng * x.j4 / parts);
    const int rb = min (4 * (ng * (x.j4 + 1) / parts), nrc);
    const int nr = rb - ra;
    if (nr <= 0) return;
    // one row per lane: (y, z) part of the world position and the fixed
    // image's row index (-1: row outside the ROI)
    float4* rows = (float4*) (x.sm + XS_ROWS) + XL_ROWS_MAX * x.warp;
    if (x.lane < nr) {
        const int rho = ra + x.lane;
        const int qy = xl_q (rho, a.d_vy);
        const int ly = rho - qy * vy, lz = t.lz0 + qy;
        const int fj = g.roi_off[1] + vy * t.ty + ly;
        const int fk = g.roi_off[2] + g.vpr[2] * t.tz + lz;
        const bool live = fj < g.roi_off[1] + g.roi_dim[1]
            && fk < g.roi_off[2] + g.roi_dim[2];
        const float ffj = (float) fj, ffk = (float) fk;
        float p[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            p[d] = __fadd_rn (__fadd_rn (g.img_origin[d],
                __fmul_rn (g.fstep[3 * d + 1], ffj)),
                __fmul_rn (g.fstep[3 * d + 2], ffk));
        }
        rows[x.lane] = make_float4 (p[0], p[1], p[2],
            __int_as_float (live ? g.fdim[0] * (fj + g.fdim[1] * fk) : -1));
    }
    __syncwarp ();

    const int X = 32 * x.q + x.lane;
    const int fi = g.roi_off[0] + g.vpr[0] * t.tx0 + X;
    const bool xlive = X < min (a.T, g.rdims[0] - t.tx0) * g.vpr[0]
        && fi < g.roi_off[0] + g.roi_dim[0];
    const int fic = min (fi, g.fdim[0] - 1);
    const float ffi = (float) fi;
    const float xp[3] = {__fmul_rn (g.fstep[0], ffi), __fmul_rn (g.fstep[3], ffi),
        __fmul_rn (g.fstep[6], ffi)};
    const int dxm = g.mdim[0], dxym = g.mdim[0] * g.mdim[1];
    // the moving geometry in registers for the row loop
    float m_org[3], m_prj[3], m_hi[3], m_fmax[3];
    int m_cmax[3];
#pragma unroll
    for (int e = 0; e < 3; e++) {
        m_org[e] = g.morigin[e];
        m_prj[e] = g.mproj[4 * e];
        m_hi[e] = g.m_hi[e];
        m_fmax[e] = g.m_fmax[e];
        m_cmax[e] = g.mdim[e] - 2;
    }
    // adjoint operand: row n = c * 32 + rho, column (K) x
    uint8_t* dcb = x.sm + XS_DC + buf * XS_DC_BUF + (X >> 6) * XS_DC_ATOM
        + (X & 7) * 2;
    const int xch = (X & 63) >> 3;
    const uint32_t tl = x.taddr + ((uint32_t) (32 * x.q) << 16) + XT_D
        + 128 * buf;

    for (int r0 = ra; r0 < rb; r0 += 4) {
        float dv[12];
        tmem_ld4x3_wait (tl + r0, tl + XL_RC + r0, tl + 2 * XL_RC + r0, dv);
#pragma unroll
        for (int u0 = 0; u0 < 4; u0 += NS) {
            if (r0 + u0 >= rb) break;          // all rows past the warp's
            bool ok[NS], rowv[NS];
            int mvf[NS], mvr[NS], fidx[NS], clampb[NS];
            float w2[NS][3];
#pragma unroll
            for (int h = 0; h < NS; h++) {
                const int u = u0 + h;
                const int rho = r0 + u;
                rowv[h] = rho < rb;
                const float4 rw = rows[rowv[h] ? rho - ra : 0];
                const int frow = __float_as_int (rw.w);
                const float d[3] = {dv[u], dv[4 + u], dv[8 + u]};
                const float fxyz[3] = {__fadd_rn (rw.x, xp[0]),
                    __fadd_rn (rw.y, xp[1]), __fadd_rn (rw.z, xp[2])};
                float tt[3];
#pragma unroll
                for (int e = 0; e < 3; e++) {
                    tt[e] = __fsub_rn (__fadd_rn (fxyz[e], d[e]), m_org[e]);
                }
                bool in = rowv[h] && xlive && frow >= 0;
                int f[3];
                bool up[3];
                clampb[h] = 0;
#pragma unroll
                for (int e = 0; e < 3; e++) {
                    float ma;
                    if (AXIS) {
                        ma = __fmul_rn (tt[e], m_prj[e]);
                    } else {
                        ma = __fadd_rn (__fadd_rn (__fmul_rn (tt[0], g.mproj[3 * e]),
                            __fmul_rn (tt[1], g.mproj[3 * e + 1])),
                            __fmul_rn (tt[2], g.mproj[3 * e + 2]));
                    }
                    in = in && ma > -0.5f && ma < m_hi[e];
                    if (MODE == XM_PZ_GRAD
                        && (ma < 0.f || ma >= m_fmax[e] + 1.f)) {
                        clampb[h] |= 1 << e;      // li_clamp holds this axis
                    }
                    // li_clamp without conversions: floor(max(ma, 0)) from
                    // an add rounded down to 2^23, corner clamped to dim - 2,
                    // fraction saturated to [0, 1]
                    const float big = __fadd_rd (fmaxf (ma, 0.f), 8388608.f);
                    f[e] = min (__float_as_int (big) - 0x4B000000, m_cmax[e]);
                    const float fc = fminf (big - 8388608.f, m_fmax[e]);
                    const float w = __saturatef (ma - fc);
                    w2[h][e] = w;
                    up[e] = w >= 0.5f;
                }
                fidx[h] = max (frow, 0) + fic;
                if (ROI) {
                    // the image ROIs (flavour i): fixed at the voxel,
                    // moving at the moving position
                    in = in && roi_fixed_ok (g, fidx[h])
                        && roi_moving_ok (g, fxyz, d);
                }
                ok[h] = in;
                mvf[h] = f[0] + dxm * (f[1] + g.mdim[1] * f[2]);
                mvr[h] = mvf[h] + (up[0] ? 1 : 0) + (up[1] ? dxm : 0)
                    + (up[2] ? dxym : 0);
            }
            auto store_dc = [&](int h, const float dc[3]) {
                if (rowv[h]) {
                    const int rho = r0 + u0 + h;
                    uint8_t* p = dcb + (rho >> 3) * 1024 + (rho & 7) * 128
                        + ((xch ^ (rho & 7)) << 4);
                    // hi = bf16(v), lo = bf16(v - hi), two values a convert
                    const __nv_bfloat162 h01 = __floats2bfloat162_rn (dc[0], dc[1]);
                    const __nv_bfloat162 h22 = __floats2bfloat162_rn (dc[2], dc[2]);
                    const float2 f01 = __bfloat1622float2 (h01);
                    const __nv_bfloat162 l01 = __floats2bfloat162_rn (
                        dc[0] - f01.x, dc[1] - f01.y);
                    const float f2 = __low2float (h22);
                    const __nv_bfloat162 l22 = __floats2bfloat162_rn (
                        dc[2] - f2, dc[2] - f2);
                    *(__nv_bfloat16*) (p) = __low2bfloat16 (h01);
                    *(__nv_bfloat16*) (p + 4096) = __high2bfloat16 (h01);
                    *(__nv_bfloat16*) (p + 8192) = __low2bfloat16 (h22);
                    *(__nv_bfloat16*) (p + XS_DC_LO) = __low2bfloat16 (l01);
                    *(__nv_bfloat16*) (p + XS_DC_LO + 4096) = __high2bfloat16 (l01);
                    *(__nv_bfloat16*) (p + XS_DC_LO + 8192) = __low2bfloat16 (l22);
                }
            };
            if constexpr (xl_mse_mode (MODE)) {
                float cr[NS][8], fv[NS], gr[NS][3];
#pragma unroll
                for (int h = 0; h < NS; h++) {
                    const float* mp = a.mimg + mvf[h];
                    cr[h][0] = __ldg (mp);
                    cr[h][1] = __ldg (mp + 1);
                    cr[h][2] = __ldg (mp + dxm);
                    cr[h][3] = __ldg (mp + dxm + 1);
                    cr[h][4] = __ldg (mp + dxym);
                    cr[h][5] = __ldg (mp + dxym + 1);
                    cr[h][6] = __ldg (mp + dxym + dxm);
                    cr[h][7] = __ldg (mp + dxym + dxm + 1);
                    fv[h] = __ldg (a.fimg + fidx[h]);
                    if (MODE == XM_MSE_NEAREST) {
                        const float* gp = a.mgrad + 3 * mvr[h];
                        gr[h][0] = __ldg (gp);
                        gr[h][1] = __ldg (gp + 1);
                        gr[h][2] = __ldg (gp + 2);
                    }
                }
#pragma unroll
                for (int h = 0; h < NS; h++) {
                    float diff = trilinear_lerp (w2[h], cr[h]) - fv[h];
                    diff = ok[h] ? diff : 0.f;
                    scf = fmaf (diff, diff, scf);
                    cnt += ok[h] ? 1 : 0;
                    float dc[3];
                    if (MODE == XM_MSE_NEAREST) {
                        dc[0] = diff * gr[h][0];
                        dc[1] = diff * gr[h][1];
                        dc[2] = diff * gr[h][2];
                    } else {
                        float gl[3];
                        trilinear_lerp_grad (g, w2[h], cr[h], gl);
                        dc[0] = diff * gl[0];
                        dc[1] = diff * gl[1];
                        dc[2] = diff * gl[2];
                    }
                    store_dc (h, dc);
                }
            } else if constexpr (MODE == XM_MI_GRAD || MODE == XM_MI_HIST) {
                // PVI-8: the fixed voxel's bin and the bins of the eight
                // trilinear corners, in li_value's order
                int fb[NS], mb[NS][8];
#pragma unroll
                for (int h = 0; h < NS; h++) {
                    const uint8_t* mp = a.mbin + mvf[h];
                    mb[h][0] = __ldg (mp);
                    mb[h][1] = __ldg (mp + 1);
                    mb[h][2] = __ldg (mp + dxm);
                    mb[h][3] = __ldg (mp + dxm + 1);
                    mb[h][4] = __ldg (mp + dxym);
                    mb[h][5] = __ldg (mp + dxym + 1);
                    mb[h][6] = __ldg (mp + dxym + dxm);
                    mb[h][7] = __ldg (mp + dxym + dxm + 1);
                    fb[h] = __ldg (a.fbin + fidx[h]);
                }
                if constexpr (MODE == XM_MI_GRAD) {
                    const float nv = __ldg (a.mi_nvf);
#pragma unroll
                    for (int h = 0; h < NS; h++) {
                        float dc[3] = {0.f, 0.f, 0.f};
                        if (ok[h]) xl_mi_dc_dv (a, w2[h], fb[h], mb[h], nv, dc);
                        store_dc (h, dc);
                    }
                } else {
                    unsigned long long* hsm = (unsigned long long*) (x.sm + XS_DC);
#pragma unroll
                    for (int h = 0; h < NS; h++) {
                        xl_mi_hist_add (a, hsm, ok[h], w2[h], fb[h], mb[h],
                            x.lane, cnt);
                    }
                }
            } else {
                // Parzen windows: the trilinear moving value's window
                float cr[NS][8];
                int fb[NS];
#pragma unroll
                for (int h = 0; h < NS; h++) {
                    const float* mp = a.mimg + mvf[h];
                    cr[h][0] = __ldg (mp);
                    cr[h][1] = __ldg (mp + 1);
                    cr[h][2] = __ldg (mp + dxm);
                    cr[h][3] = __ldg (mp + dxm + 1);
                    cr[h][4] = __ldg (mp + dxym);
                    cr[h][5] = __ldg (mp + dxym + 1);
                    cr[h][6] = __ldg (mp + dxym + dxm);
                    cr[h][7] = __ldg (mp + dxym + dxm + 1);
                    fb[h] = __ldg (a.fbin + fidx[h]);
                }
#pragma unroll
                for (int h = 0; h < NS; h++) {
                    const float u = parzen_centre (trilinear_lerp (w2[h], cr[h]),
                        a.pz_mmin, a.pz_mdelta);
                    if constexpr (MODE == XM_PZ_HIST) {
                        unsigned long long* hsm = (unsigned long long*) (x.sm + XS_DC);
                        xl_pz_hist_add (a, hsm, ok[h], fb[h], u, x.lane, cnt);
                    } else {
                        float dc[3] = {0.f, 0.f, 0.f};
                        if (ok[h]) {
                            xl_pz_dc_dv (a, u, fb[h], w2[h], cr[h], clampb[h], dc);
                        }
                        store_dc (h, dc);
                    }
                }
            }
        }
    }
}

// x-forward MMA of a step: D[x][(c, rho)] = Bx[x][xk] R[xk][(c, rho)],
// K = 32 knots, three split terms; one thread.  buf: the D accumulator,
// rbuf: the R operand buffer.
__device__ __forceinline__ void
xl_issue_forward (const XlCtx& x, int buf, int rbuf, uint64_t* bar)
{
    const uint32_t idesc = idesc_bf16_f32 (128, XL_N, 0, 1);
    const uint32_t ta = x.sm_base + XS_TAB;
    const uint32_t tb = x.sm_base + XS_B2 + rbuf * XS_B2_BUF;
#pragma unroll
    for (int term = 0; term < 3; term++) {
        const uint32_t A = term == 2 ? ta + XS_TAB_LO : ta;     // hi, hi, lo
        const uint32_t B = term == 1 ? tb + XS_B2_LO : tb;      // hi, lo, hi
#pragma unroll
        for (int ks = 0; ks < 2; ks++) {
            tc_mma_bf16 (x.taddr + XT_D + 128 * buf,
                smem_desc_sw128 (A + ks * 32, 16, 1024),
                smem_desc_sw128 (B + ks * 2048, 4096, 1024), idesc,
                (term > 0 || ks > 0) ? 1u : 0u);
        }
    }
    tc_commit (bar);
}

// x-adjoint MMAs of a step, one per component c:
// Rg_c[(q, xk)][rho] = Bx[x][xk] DC_c[x][rho] (the table read MN-major: M =
// four identical copies of the 32 knots, so every TMEM lane quarter q holds
// all of Rg_c), N = the component's 32 rows, K = 128 voxels, three split
// terms; Rg_c in columns 32 c of the buffer.  One thread.
__device__ __forceinline__ void
xl_issue_adjoint (const XlCtx& x, int buf, uint64_t* bar)
{
    const uint32_t idesc = idesc_bf16_f32 (128, XL_RC, 1, 0);
    const uint32_t ta = x.sm_base + XS_TAB;
    const uint32_t td = x.sm_base + XS_DC + buf * XS_DC_BUF;
#pragma unroll
    for (int c = 0; c < 3; c++) {
#pragma unroll
        for (int term = 0; term < 3; term++) {
            const uint32_t A = term == 2 ? ta + XS_TAB_LO : ta;
            // the component's 32 rows: four 8-row groups of 1024 bytes
            const uint32_t B = (term == 1 ? td + XS_DC_LO : td) + 4096 * c;
#pragma unroll
            for (int ks = 0; ks < 8; ks++) {
                tc_mma_bf16 (x.taddr + XT_RG + 128 * buf + XL_RC * c,
                    smem_desc_sw128 (A + ks * 2048, 16384, 1024),
                    smem_desc_sw128 (B + (ks >> 2) * XS_DC_ATOM + (ks & 3) * 32,
                        16, 1024), idesc, (term > 0 || ks > 0) ? 1u : 0u);
            }
        }
    }
    tc_commit (bar);
}

// A look-ahead warp's share of step sn: its component of the R operand into
// buffer rbuf, then (MSE) its share of the L2 prefetch of the step's fixed
// rows.
template <int MODE>
__device__ __forceinline__ bool
xl_produce (const XlArgs& a, const XlCtx& x, uint64_t* s_bar, int sn,
    int rbuf)
{
    const XlStep tn = xl_step (a, sn);
    xl_yz_forward (a, x, tn, rbuf);
    fence_proxy_async_smem ();
    __syncwarp ();
    if (x.lane == 0) mbar_arrive (&s_bar[XB_B2 + rbuf]);
    if (xl_mse_mode (MODE)) xl_prefetch_fixed (a, x, tn);
    return true;
}

}  // namespace

template <int MODE, bool AXIS, bool ROI>
__global__ void __launch_bounds__ (XL_BLOCK, 1)
mse_xl_kernel (XlArgs a)
{
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t s_bar[XB_DRAIN + 1];
    __shared__ uint32_t s_taddr;
    __shared__ int s_abort;
    // each compute warp's score and count of the batch that ends at a
    // step, by step parity (summed by the tensor-core thread)
    __shared__ double s_wsc[2][XL_CW];
    __shared__ int s_wcnt[2][XL_CW];

    const BspGeom& g = a.g;
    XlCtx x;
    x.sm = smem_raw + ((1024u - (smem_addr (smem_raw) & 1023u)) & 1023u);
    x.sm_base = smem_addr (x.sm);
    const int tid = threadIdx.x;
    x.warp = tid >> 5;
    x.lane = tid & 31;
    x.q = x.warp & 3;
    x.j4 = x.warp >> 2;
    const bool mma_warp = x.warp == XL_CW;

    if (tid == 0) {
        for (int i = 0; i < XL_NB2; i++) mbar_init (&s_bar[XB_B2 + i], 3);
        mbar_init (&s_bar[XB_DC], XL_CW);
        mbar_init (&s_bar[XB_DC + 1], XL_CW);
        mbar_init (&s_bar[XB_D], 1);
        mbar_init (&s_bar[XB_D + 1], 1);
        mbar_init (&s_bar[XB_RG], 1);
        mbar_init (&s_bar[XB_RG + 1], 1);
        mbar_init (&s_bar[XB_DRAIN], 1);
        fence_barrier_init ();
        s_abort = 0;
    }
    if (mma_warp) {
        tmem_alloc (&s_taddr, XT_COLS);
        tmem_relinquish ();
    } else {
        // the basis table; both dc/dv buffers zeroed (entries the voxel
        // phase never writes stay zero); the y and z basis values
        uint4* tab = (uint4*) (x.sm + XS_TAB);
        for (int o = tid; o < 65536 / 16; o += XL_THREADS) tab[o] = a.tab[o];
        uint4* dcz = (uint4*) (x.sm + XS_DC);
        for (int o = tid; o < 2 * XS_DC_BUF / 16; o += XL_THREADS) {
            dcz[o] = make_uint4 (0, 0, 0, 0);
        }
        float* lut = (float*) (x.sm + XS_LUT);
        const int nby = 4 * g.vpr[1], nbz = 4 * g.vpr[2];
        for (int o = tid; o < nby + nbz; o += XL_THREADS) {
            lut[o] = a.luts[4 * g.vpr[0] + o];
        }
        fence_proxy_async_smem ();
    }
    tc_fence_before ();
    __syncthreads ();
    tc_fence_after ();
    x.taddr = s_taddr;
    volatile int* abort_flag = &s_abort;
    const int nb_local = (a.nbatches - (int) blockIdx.x + (int) gridDim.x - 1)
        / (int) gridDim.x;
    const int S = nb_local * a.nch;

    if (mma_warp) {
        if (x.lane == 0 && !a.withhold) {
            // phase parities, bit buf of each word (no local arrays)
            uint32_t ph_b2 = 0, ph_dc = 0;
            auto wait = [&](uint64_t* bar, uint32_t& ph, int buf, int code,
                    unsigned cap) {
                if (xl_poll (bar, (ph >> buf) & 1u, cap, a.wait_limit,
                        abort_flag)) {
                    ph ^= 1u << buf;
                    return true;
                }
                *abort_flag = 1;
                atomicExch (a.err, code);
                return false;
            };
            int rb = 0;                      // s % XL_NB2
            for (int s = 0; s <= S; s++) {
                if (s < S) {
                    if (!wait (&s_bar[XB_B2 + rb], ph_b2, rb, 3, XL_SLEEP_B2)) {
                        break;
                    }
                    tc_fence_after ();
                    xl_issue_forward (x, s & 1, rb, &s_bar[XB_D + (s & 1)]);
                    rb = rb + 1 == XL_NB2 ? 0 : rb + 1;
                }
                if (s >= 1) {
                    // the voxel phase of step s - 1 is done with D (and
                    // has written dc/dv, except in the histogram passes)
                    const int pb = (s - 1) & 1;
                    if (!wait (&s_bar[XB_DC + pb], ph_dc, pb, 4, XL_SLEEP_DC)) {
                        break;
                    }
                    tc_fence_after ();
                    if (!xl_hist_mode (MODE)) {
                        xl_issue_adjoint (x, pb, &s_bar[XB_RG + pb]);
                    }
                    if (xl_mse_mode (MODE)) {
                        // the batch's score and count, warps in order
                        const XlStep tp = xl_step (a, s - 1);
                        if (tp.ch == a.nch - 1) {
                            double v = 0.0;
                            int n = 0;
#pragma unroll
                            for (int w = 0; w < XL_CW; w++) {
                                v += s_wsc[pb][w];
                                n += s_wcnt[pb][w];
                            }
                            a.score_part[tp.b] = v;
                            a.count_part[tp.b] = n;
                        }
                    }
                }
            }
        }
        __syncwarp ();
    } else {
        uint32_t ph_d = 0, ph_rg = 0;       // phase parity of buffer b: bit b
        const bool yz_fwd_warp = x.q == 3;
        const bool vox_live = 32 * x.q < a.T * g.vpr[0];
        // the y/z adjoint: by lane quarter 3's warps (one component each,
        // every knot plane) when that quarter has no samples, else by the
        // other quarters' warps (component q, knot plane j4)
        const bool adj_q3 = 32 * 3 >= a.T * g.vpr[0];
        const bool adj_warp = adj_q3 ? x.q == 3 : x.q < 3;
        float G[4] = {0.f, 0.f, 0.f, 0.f};
        double sc = 0.0;
        int cnt = 0;
        bool ok = true;
        if (yz_fwd_warp) {
            for (int s = 0; s < XL_NB2 && s < S && ok; s++) {
                ok = xl_produce<MODE> (a, x, s_bar, s, s);
            }
        }
        // adjoint y/z of step sp (quarters 0..2): accumulate, and write
        // the batch's partial gradient at its last chunk
        auto yz_adjoint = [&](int sp) {
            const int pb = sp & 1;
            if (!xl_wait (a, x, &s_bar[XB_RG + pb], (ph_rg >> pb) & 1u,
                    abort_flag, 2, XL_SLEEP_COMPUTE)) {
                return false;
            }
            ph_rg ^= 1u << pb;
            tc_fence_after ();
            const XlStep t = xl_step (a, sp);
            if (adj_q3) {
                // component j4, the four knot planes one after another,
                // added into the batch's partial gradient (stored by the
                // first chunk; the same thread owns those entries)
                const int c = x.j4;
                float* dst = a.part + ((size_t) t.b * 3 + c) * (16 * a.KX)
                    + x.lane;
                float rg[32];
                xl_load_rg (x, pb, c, rg);
                for (int k = 0; k < 4; k++) {
                    float Gk[4] = {0.f, 0.f, 0.f, 0.f};
                    xl_yz_adjoint (a, x, t, rg, k, Gk);
                    if (x.lane < a.KX) {
#pragma unroll
                        for (int j = 0; j < 4; j++) {
                            float* p = dst + a.KX * (j + 4 * k);
                            *p = t.ch == 0 ? Gk[j] : *p + Gk[j];
                        }
                    }
                }
                tc_fence_before ();
                return true;
            }
            if (t.ch == 0) G[0] = G[1] = G[2] = G[3] = 0.f;
            float rg[32];
            xl_load_rg (x, pb, x.q, rg);
            xl_yz_adjoint (a, x, t, rg, x.j4, G);
            tc_fence_before ();
            if (t.ch == a.nch - 1 && x.lane < a.KX) {
                const int KF = 16 * a.KX;
                float* dst = a.part + ((size_t) t.b * 3 + x.q) * KF + x.lane
                    + a.KX * 4 * x.j4;
#pragma unroll
                for (int j = 0; j < 4; j++) dst[a.KX * j] = G[j];
            }
            return true;
        };
        for (int s = 0; s < S && ok; s++) {
            const int buf = s & 1;
            if (!xl_wait (a, x, &s_bar[XB_D + buf], (ph_d >> buf) & 1u,
                    abort_flag, 1,
                    yz_fwd_warp ? XL_SLEEP_AHEAD : XL_SLEEP_COMPUTE)) {
                ok = false;
                break;
            }
            ph_d ^= 1u << buf;
            tc_fence_after ();
            const XlStep t = xl_step (a, s);
            if (vox_live) {
                float scf = 0.f;
                xl_voxel<MODE, AXIS, ROI> (a, x, t, buf, scf, cnt);
                sc += (double) scf;
            }
            if (xl_mse_mode (MODE) && t.ch == a.nch - 1) {
                // the warp's score and count of the batch (fixed tree
                // order), for the tensor-core thread once this step's
                // dc/dv barrier completes
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    sc += __shfl_down_sync (0xffffffffu, sc, o);
                    cnt += __shfl_down_sync (0xffffffffu, cnt, o);
                }
                if (x.lane == 0) {
                    s_wsc[buf][x.warp] = sc;
                    s_wcnt[buf][x.warp] = cnt;
                }
                sc = 0.0;
                cnt = 0;
            }
            fence_proxy_async_smem ();
            tc_fence_before ();
            __syncwarp ();
            if (x.lane == 0) mbar_arrive (&s_bar[XB_DC + buf]);
            if (yz_fwd_warp) {
                // the forward MMA of step s has read R buffer s % XL_NB2:
                // step s + XL_NB2 goes there
                if (s + XL_NB2 < S) {
                    ok = xl_produce<MODE> (a, x, s_bar, s + XL_NB2,
                        s % XL_NB2);
                }
            }
            if (ok && adj_warp && s >= 1 && !xl_hist_mode (MODE)) {
                ok = yz_adjoint (s - 1);
            }
        }
        if (ok && adj_warp && S >= 1 && !xl_hist_mode (MODE)) {
            yz_adjoint (S - 1);
        }
        if constexpr (xl_hist_mode (MODE)) {
            // the CTA's histograms and voxel count into the global ones
            // (integer sums: the order does not matter); the moving
            // histogram is the joint one's column sums; Parzen keeps the
            // joint one only (its score kernel forms the marginals)
            named_bar_sync (1, XL_THREADS);
            const int B = a.bins, nh = 2 * B + B * B;
            const unsigned long long* h = (const unsigned long long*) (x.sm + XS_DC);
            for (int i = tid; i < nh; i += XL_THREADS) {
                unsigned long long v = h[i];
                if (MODE == XM_PZ_HIST && i < 2 * B) {
                    v = 0;
                } else if (i >= B && i < 2 * B) {
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

    if (mma_warp && x.lane == 0 && !a.withhold) {
        // every MMA this thread issued completes before TMEM is released,
        // also when a wait gave up (the MMAs themselves wait on nothing)
        tc_commit (&s_bar[XB_DRAIN]);
        int never = 0;
        xl_poll (&s_bar[XB_DRAIN], 0, XL_SLEEP_AHEAD, a.wait_limit + 1000u,
            &never);
    }
    tc_fence_before ();
    __syncthreads ();
    if (mma_warp) tmem_dealloc (x.taddr, XT_COLS);
}

// ------------------------------------------------------------------ host --

bool
xl_plan (const BspGeom& g, XlPlan* p, int sm_count, int extra_row_batches)
{
    const int vx = g.vpr[0], vy = g.vpr[1], vz = g.vpr[2];
    if (vy < 3 || vy > 10 || vx < 1 || vz < 1) return false;
    // tiles per batch: T vx <= 128 voxels and T + 3 <= 32 knots along x;
    // the fewest batches per row, balanced; a split row needs T >= 3 (the
    // finish kernel's gather assumes a knot meets at most two batches)
    const int tmax = std::min (128 / vx, XL_KMAX - 3);
    if (tmax < 1) return false;
    const int nb_row = (g.rdims[0] + tmax - 1) / tmax + extra_row_batches;
    if (nb_row > g.rdims[0]) return false;
    const int T = (g.rdims[0] + nb_row - 1) / nb_row;
    if (nb_row > 1 && T < 3) return false;
    p->T = T;
    p->nbx = nb_row;
    p->nbatches = nb_row * g.rdims[1] * g.rdims[2];
    // rows per chunk: whole z planes of vy rows, at most 32 rows
    const int nlz_max = XL_RC / vy;
    p->nch = (vz + nlz_max - 1) / nlz_max;
    p->nlz = (vz + p->nch - 1) / p->nch;
    p->smem = XS_TOTAL + 1024;
    p->threads = XL_BLOCK;
    p->grid = std::min (p->nbatches, sm_count);
    p->score_parts = p->nbatches;
    return true;
}

// The basis table image: 128 voxel rows x 128 columns m = q * 32 + xk
// (four copies of the 32 knot columns), bf16 hi then lo,
// each the exact 128-byte-swizzled shared-memory image (32 KB).  Row x of a
// batch, x < T vx, holds bx[x mod vx][xk - x div vx] on the band.
int
xl_build_table (const BspGeom& g, const XlPlan& p, const float* bx_lut,
    void** d_tab)
{
    const int vx = g.vpr[0];
    std::vector<uint8_t> img (65536, 0);
    for (int xr = 0; xr < 128; xr++) {
        for (int m = 0; m < 128; m++) {
            const int xk = m & 31;
            float v = 0.f;
            if (xr < p.T * vx) {
                const int i = xk - xr / vx;
                if (i >= 0 && i < 4) v = bx_lut[4 * (xr % vx) + i];
            }
            __nv_bfloat16 h = __float2bfloat16_rn (v);
            __nv_bfloat16 l = __float2bfloat16_rn (v - __bfloat162float (h));
            const uint32_t off = sw128_offset (xr, m, 128);
            *(unsigned short*) (img.data () + off) = __bfloat16_as_ushort (h);
            *(unsigned short*) (img.data () + 32768 + off) = __bfloat16_as_ushort (l);
        }
    }
    if (cudaMalloc (d_tab, img.size ()) != cudaSuccess) return B200BSP_E_OOM;
    if (cudaMemcpy (*d_tab, img.data (), img.size (), cudaMemcpyHostToDevice)
        != cudaSuccess) {
        return B200BSP_E_CUDA;
    }
    return B200BSP_OK;
}

template <int MODE, bool AXIS, bool ROI>
static cudaError_t
xl_launch_t (const XlPlan& p, const XlArgs& a, cudaStream_t st)
{
    auto k = mse_xl_kernel<MODE, AXIS, ROI>;
    cudaError_t e = set_max_dynamic_smem ((const void*) k, (int) p.smem);
    if (e != cudaSuccess) return e;
    k<<<p.grid, XL_BLOCK, p.smem, st>>> (a);
    return cudaGetLastError ();
}

static bool
xl_axis_aligned (const BspGeom& g)
{
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) {
            if (i != j && (g.fstep[3 * i + j] != 0.f || g.mproj[3 * i + j] != 0.f)) {
                return false;
            }
        }
    }
    return true;
}

cudaError_t
launch_mi_xl (const BspGeom& g, const XlPlan& p, bool hist_pass,
    const TcMiArgs& mi, const float* coeff, const void* tab,
    const float* luts, float* part, int* err, unsigned wait_limit,
    cudaStream_t st)
{
    XlArgs a = {};
    a.g = g;
    a.T = p.T;
    a.KX = p.T + 3;
    a.nbx = p.nbx;
    a.nbatches = p.nbatches;
    a.nlz = p.nlz;
    a.nch = p.nch;
    a.d_nch = xl_div (p.nch);
    a.d_nbx = xl_div (p.nbx);
    a.d_rdy = xl_div (g.rdims[1]);
    a.d_vy = xl_div (g.vpr[1]);
    a.wait_limit = wait_limit;
    a.coeff = coeff;
    a.tab = (const uint4*) tab;
    a.luts = luts;
    a.part = part;
    a.err = err;
    a.fbin = mi.fbin; a.mbin = mi.mbin; a.bins = mi.bins;
    a.mi_lut = mi.lut; a.mi_nvf = mi.nvf; a.hist = mi.hist;
    a.mimg = mi.mimg;
    a.pz_mmin = mi.m_min;
    a.pz_mdelta = mi.m_delta;
    const bool axis = xl_axis_aligned (g);
    if (mi.parzen) {
        if (hist_pass) {
            return axis ? xl_launch_t<XM_PZ_HIST, true, false> (p, a, st)
                        : xl_launch_t<XM_PZ_HIST, false, false> (p, a, st);
        }
        return axis ? xl_launch_t<XM_PZ_GRAD, true, false> (p, a, st)
                    : xl_launch_t<XM_PZ_GRAD, false, false> (p, a, st);
    }
    if (hist_pass) {
        return axis ? xl_launch_t<XM_MI_HIST, true, false> (p, a, st)
                    : xl_launch_t<XM_MI_HIST, false, false> (p, a, st);
    }
    return axis ? xl_launch_t<XM_MI_GRAD, true, false> (p, a, st)
                : xl_launch_t<XM_MI_GRAD, false, false> (p, a, st);
}

bool
xl_mi_supported (int bins)
{
    return (size_t) (2 * bins + bins * bins) * 8 <= 2 * XS_DC_BUF;
}

cudaError_t
launch_mse_xl (const BspGeom& g, const XlPlan& p, int grad_mode,
    const float* fimg, const float* mimg, const float* mgrad,
    const float* coeff, const void* tab, const float* luts, float* part,
    double* score_part, int* count_part, int* err, unsigned wait_limit,
    int withhold, cudaStream_t st)
{
    XlArgs a = {};
    a.g = g;
    a.T = p.T;
    a.KX = p.T + 3;
    a.nbx = p.nbx;
    a.nbatches = p.nbatches;
    a.nlz = p.nlz;
    a.nch = p.nch;
    a.d_nch = xl_div (p.nch);
    a.d_nbx = xl_div (p.nbx);
    a.d_rdy = xl_div (g.rdims[1]);
    a.d_vy = xl_div (g.vpr[1]);
    a.wait_limit = wait_limit;
    a.withhold = withhold;
    a.fimg = fimg; a.mimg = mimg; a.mgrad = mgrad; a.coeff = coeff;
    a.tab = (const uint4*) tab;
    a.luts = luts;
    a.part = part; a.score_part = score_part; a.count_part = count_part;
    a.err = err;
    const bool axis = xl_axis_aligned (g);
    const bool roi = g.fmask || g.mroi;
    if (roi) {
        if (grad_mode == 0) {
            return axis ? xl_launch_t<0, true, true> (p, a, st)
                        : xl_launch_t<0, false, true> (p, a, st);
        }
        return axis ? xl_launch_t<1, true, true> (p, a, st)
                    : xl_launch_t<1, false, true> (p, a, st);
    }
    if (grad_mode == 0) {
        return axis ? xl_launch_t<0, true, false> (p, a, st)
                    : xl_launch_t<0, false, false> (p, a, st);
    }
    return axis ? xl_launch_t<1, true, false> (p, a, st)
                : xl_launch_t<1, false, false> (p, a, st);
}

}  // namespace b200
