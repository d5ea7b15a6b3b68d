// Self-test of the tensor-core building blocks used by mse_tc.cu: the
// split-bf16 forward GEMM D = Q * C^T (A K-major, B K-major) and adjoint
// GEMM G = DCDV * Q (A K-major, B = the same Q bytes read MN-major), with
// operands placed in the same 128-byte-swizzled shared-memory layouts.
// Exported as an internal symbol for the test suite; not part of the
// public ABI.
#include <cuda_bf16.h>

#include "tc_ptx.cuh"

namespace b200 {

__device__ __forceinline__ void
split16 (float x, unsigned short& hi, unsigned short& lo)
{
    __nv_bfloat16 h = __float2bfloat16_rn (x);
    __nv_bfloat16 l = __float2bfloat16_rn (x - __bfloat162float (h));
    hi = __bfloat16_as_ushort (h);
    lo = __bfloat16_as_ushort (l);
}

// q: 128 x 64, c: N x 64, dcdv: 128 x 128 (row-major float);
// d_out: 128 x N, g_out: 128 x 64.
__global__ void __launch_bounds__ (128, 1)
tc_selftest_kernel (const float* q, const float* c, const float* dcdv, int N,
    float* d_out, float* g_out, int* err)
{
    extern __shared__ uint8_t raw[];
    __shared__ uint64_t bar;
    __shared__ uint32_t s_taddr;
    uint8_t* sm = (uint8_t*) (((uintptr_t) raw + 1023) & ~(uintptr_t) 1023);
    uint32_t base = smem_addr (sm);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // Q hi/lo at 0/16K, C hi/lo at 32K/32K+N*128, DCDV hi/lo after (32K each)
    const uint32_t oq = 0, oc = 32768, odc = 32768 + 2 * 256 * 128;
    for (int e = tid; e < 128 * 64; e += 128) {
        int r = e / 64, k = e % 64;
        unsigned short h, l;
        split16 (q[e], h, l);
        uint32_t off = sw128_offset (r, k, 128);
        *(unsigned short*) (sm + oq + off) = h;
        *(unsigned short*) (sm + oq + 16384 + off) = l;
    }
    for (int e = tid; e < N * 64; e += 128) {
        int r = e / 64, k = e % 64;
        unsigned short h, l;
        split16 (c[e], h, l);
        uint32_t off = sw128_offset (r, k, N);
        *(unsigned short*) (sm + oc + off) = h;
        *(unsigned short*) (sm + oc + N * 128 + off) = l;
    }
    for (int e = tid; e < 128 * 128; e += 128) {
        int r = e / 128, k = e % 128;
        unsigned short h, l;
        split16 (dcdv[e], h, l);
        uint32_t off = sw128_offset (r, k, 128);
        *(unsigned short*) (sm + odc + off) = h;
        *(unsigned short*) (sm + odc + 32768 + off) = l;
    }
    if (tid == 0) {
        mbar_init (&bar, 1);
        fence_barrier_init ();
    }
    if (warp == 0) {
        tmem_alloc (&s_taddr, 512);
        tmem_relinquish ();
    }
    fence_proxy_async_smem ();
    tc_fence_before ();
    __syncthreads ();
    tc_fence_after ();
    uint32_t taddr = s_taddr;
    if (tid == 0) {
        uint32_t idf = idesc_bf16_f32 (128, N, 0, 0);
        uint32_t ida = idesc_bf16_f32 (128, 64, 0, 1);
        const int ta[3] = {0, 0, 1}, tb[3] = {0, 1, 0};
        uint32_t acc = 0;
        for (int term = 0; term < 3; term++) {
            for (int ks = 0; ks < 4; ks++) {
                uint64_t ad = smem_desc_sw128 (base + oq + ta[term] * 16384 + ks * 32, 16, 1024);
                uint64_t bd = smem_desc_sw128 (base + oc + tb[term] * N * 128 + ks * 32, 16, 1024);
                tc_mma_bf16 (taddr, ad, bd, idf, acc);
                acc = 1;
            }
        }
        const int aa[3] = {0, 1, 0}, bb[3] = {0, 0, 1};
        for (int term = 0; term < 3; term++) {
            for (int s = 0; s < 8; s++) {
                uint64_t ad = smem_desc_sw128 (base + odc + aa[term] * 32768
                    + (s >> 2) * 16384 + (s & 3) * 32, 16, 1024);
                uint64_t bd = smem_desc_sw128 (base + oq + bb[term] * 16384 + s * 2048,
                    16384, 1024);
                tc_mma_bf16 (taddr + 256, ad, bd, ida, (term > 0 || s > 0) ? 1u : 0u);
            }
        }
        tc_commit (&bar);
        if (!mbar_wait_bounded (&bar, 0, 1u << 22)) atomicExch (err, 1);
    }
    __syncthreads ();
    tc_fence_after ();
    int row = 32 * warp + lane;
    for (int col = 0; col < N; col += 16) {
        float v[16];
        tmem_ld16_wait (taddr + ((uint32_t) (32 * warp) << 16) + col, v);
        for (int i = 0; i < 16 && col + i < N; i++) d_out[row * N + col + i] = v[i];
    }
    for (int col = 0; col < 64; col += 16) {
        float v[16];
        tmem_ld16_wait (taddr + ((uint32_t) (32 * warp) << 16) + 256 + col, v);
        for (int i = 0; i < 16; i++) g_out[row * 64 + col + i] = v[i];
    }
    tc_fence_before ();
    __syncthreads ();
    if (warp == 0) tmem_dealloc (taddr, 512);
}

} // namespace b200

// Internal test hook: all pointers are device pointers.
extern "C" int
b200bsp_internal_tc_selftest (const float* q, const float* c,
    const float* dcdv, int N, float* d_out, float* g_out, int* err)
{
    if (N < 16 || N > 256 || N % 16) return -1;
    size_t smem = 1024 + 32768 + 2 * 256 * 128 + 65536;
    cudaFuncSetAttribute (b200::tc_selftest_kernel,
        cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    b200::tc_selftest_kernel<<<1, 128, smem>>> (q, c, dcdv, N, d_out, g_out, err);
    if (cudaGetLastError () != cudaSuccess) return -3;
    return cudaDeviceSynchronize () == cudaSuccess ? 0 : -3;
}
