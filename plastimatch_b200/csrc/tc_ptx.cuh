// Thin wrappers over the sm_100a PTX used by the tensor-core kernels:
// tcgen05 (TMEM allocation, MMA, commit, loads, fences), mbarriers and the
// shared-memory matrix / instruction descriptors of tcgen05.mma.
//
// Descriptor bit layouts follow the PTX ISA "tcgen05 shared memory
// descriptor" and "instruction descriptor" tables (kind::f16).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace b200 {

__device__ __forceinline__ uint32_t
smem_addr (const void* p)
{
    return (uint32_t) __cvta_generic_to_shared (p);
}

// ---- mbarrier ------------------------------------------------------------

__device__ __forceinline__ void
mbar_init (uint64_t* bar, uint32_t count)
{
    asm volatile ("mbarrier.init.shared::cta.b64 [%0], %1;"
        :: "r"(smem_addr (bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool
mbar_try_wait (uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile (
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok) : "r"(smem_addr (bar)), "r"(parity) : "memory");
    return ok != 0;
}

// One poll that may suspend the thread for up to `ns` nanoseconds while
// the phase is incomplete (it resumes as soon as the phase completes).
__device__ __forceinline__ bool
mbar_try_wait_sleep (uint64_t* bar, uint32_t parity, uint32_t ns)
{
    uint32_t ok;
    asm volatile (
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok) : "r"(smem_addr (bar)), "r"(parity), "r"(ns) : "memory");
    return ok != 0;
}

// Bounded wait: returns false after `limit` unsuccessful polls (each poll
// may itself suspend for a hardware-chosen time).
__device__ __forceinline__ bool
mbar_wait_bounded (uint64_t* bar, uint32_t parity, uint32_t limit)
{
    for (uint32_t i = 0; i < limit; i++) {
        if (mbar_try_wait (bar, parity)) return true;
    }
    return false;
}

// Arrive once on `bar` (count-based phase completion).
__device__ __forceinline__ void
mbar_arrive (uint64_t* bar)
{
    asm volatile ("mbarrier.arrive.shared::cta.b64 _, [%0];"
        :: "r"(smem_addr (bar)) : "memory");
}

// Named barrier over `nthreads` threads (a multiple of 32).
__device__ __forceinline__ void
named_bar_sync (int id, int nthreads)
{
    asm volatile ("bar.sync %0, %1;" :: "r"(id), "r"(nthreads) : "memory");
}

__device__ __forceinline__ void
fence_barrier_init ()
{
    asm volatile ("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Make generic-proxy shared-memory writes visible to the async proxy
// (tensor-core operand reads).
__device__ __forceinline__ void
fence_proxy_async_smem ()
{
    asm volatile ("fence.proxy.async.shared::cta;" ::: "memory");
}

// ---- tcgen05 -------------------------------------------------------------

__device__ __forceinline__ void
tmem_alloc (uint32_t* dst_smem, uint32_t ncols)
{
    asm volatile ("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
        :: "r"(smem_addr (dst_smem)), "r"(ncols) : "memory");
}

__device__ __forceinline__ void
tmem_relinquish ()
{
    asm volatile ("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;"
        ::: "memory");
}

__device__ __forceinline__ void
tmem_dealloc (uint32_t taddr, uint32_t ncols)
{
    asm volatile ("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
        :: "r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void
tc_fence_before ()
{
    asm volatile ("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void
tc_fence_after ()
{
    asm volatile ("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// D[tmem] (+)= A[smem desc] * B[smem desc], kind::f16 (bf16 in, f32 acc).
__device__ __forceinline__ void
tc_mma_bf16 (uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
    uint32_t idesc, uint32_t accumulate)
{
    asm volatile (
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        :: "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc),
           "r"(accumulate) : "memory");
}

// Arrive on `bar` once all previously issued tcgen05.mma of this thread
// have completed.
__device__ __forceinline__ void
tc_commit (uint64_t* bar)
{
    asm volatile (
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
        :: "r"(smem_addr (bar)) : "memory");
}

__device__ __forceinline__ void
tc_wait_ld ()
{
    asm volatile ("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 32 lanes x 8 consecutive 32-bit columns: thread i gets lane (base+i).
__device__ __forceinline__ void
tmem_ld8 (uint32_t taddr, float* v)
{
    uint32_t r[8];
    asm volatile (
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]),
          "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = __uint_as_float (r[i]);
}

__device__ __forceinline__ void
tmem_ld16 (uint32_t taddr, float* v)
{
    uint32_t r[16];
    asm volatile (
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]),
          "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
          "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float (r[i]);
}

// Three 8-column loads and the wait in one statement, so no use of the
// registers can be scheduled before tcgen05.wait::ld.
__device__ __forceinline__ void
tmem_ld8x3_wait (uint32_t a0, uint32_t a1, uint32_t a2, float* v)
{
    uint32_t r[24];
    asm volatile (
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7}, [%24];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 "
        "{%8, %9, %10, %11, %12, %13, %14, %15}, [%25];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 "
        "{%16, %17, %18, %19, %20, %21, %22, %23}, [%26];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]),
          "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
          "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23])
        : "r"(a0), "r"(a1), "r"(a2) : "memory");
#pragma unroll
    for (int i = 0; i < 24; i++) v[i] = __uint_as_float (r[i]);
}

// Three 4-column loads and the wait in one statement.
__device__ __forceinline__ void
tmem_ld4x3_wait (uint32_t a0, uint32_t a1, uint32_t a2, float* v)
{
    uint32_t r[12];
    asm volatile (
        "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%12];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%4, %5, %6, %7}, [%13];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%8, %9, %10, %11}, [%14];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]),
          "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11])
        : "r"(a0), "r"(a1), "r"(a2) : "memory");
#pragma unroll
    for (int i = 0; i < 12; i++) v[i] = __uint_as_float (r[i]);
}

__device__ __forceinline__ void
tmem_ld16_wait (uint32_t taddr, float* v)
{
    uint32_t r[16];
    asm volatile (
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]),
          "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
          "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr) : "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float (r[i]);
}

// 32 lanes x 32 consecutive columns, then the wait (one statement).
__device__ __forceinline__ void
tmem_ld32_wait (uint32_t taddr, float* v)
{
    uint32_t r[32];
    asm volatile (
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]),
          "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
          "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
          "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr) : "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float (r[i]);
}

// ---- descriptors ---------------------------------------------------------

// Shared-memory matrix descriptor, 128-byte swizzle (layout type 2),
// version 1 (sm_100), base offset 0: operand atoms must be 1024-B aligned.
__host__ __device__ __forceinline__ uint64_t
smem_desc_sw128 (uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes)
{
    uint64_t d = 0;
    d |= (uint64_t) ((saddr >> 4) & 0x3FFF);
    d |= (uint64_t) ((lbo_bytes >> 4) & 0x3FFF) << 16;
    d |= (uint64_t) ((sbo_bytes >> 4) & 0x3FFF) << 32;
    d |= (uint64_t) 1 << 46;          // version
    d |= (uint64_t) 2 << 61;          // SWIZZLE_128B
    return d;
}

// Instruction descriptor, kind::f16: D f32, A and B bf16, dense.
// a_mn / b_mn select MN-major operands.
__host__ __device__ __forceinline__ uint32_t
idesc_bf16_f32 (int M, int N, int a_mn, int b_mn)
{
    uint32_t d = 0;
    d |= 1u << 4;                      // D format f32
    d |= 1u << 7;                      // A format bf16
    d |= 1u << 10;                     // B format bf16
    d |= (uint32_t) (a_mn & 1) << 15;
    d |= (uint32_t) (b_mn & 1) << 16;
    d |= (uint32_t) ((N >> 3) & 0x3F) << 17;
    d |= (uint32_t) ((M >> 4) & 0x1F) << 24;
    return d;
}

// Byte offset of element (row r, column k) of a bf16 operand stored in the
// canonical K-major 128-byte-swizzle layout: 8-row x 64-element atoms of
// 1024 B, atoms of one 64-column chunk stacked by rows, chunks `rows*128`
// bytes apart.  The 16-byte unit index within a 128-byte row is XORed with
// (row % 8).  The same bytes read as an MN-major operand give element
// (K = r, MN = k) when the MN extent is 64.
__host__ __device__ __forceinline__ uint32_t
sw128_offset (uint32_t r, uint32_t k, uint32_t rows)
{
    return (k >> 6) * (rows * 128u) + (r >> 3) * 1024u + (r & 7u) * 128u
        + ((((k & 63u) >> 3) ^ (r & 7u)) << 4) + (k & 7u) * 2u;
}

} // namespace b200
