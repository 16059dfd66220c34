// Minimal sm_100a tensor-core (tcgen05 / UMMA) toolkit used by the split-precision FFT.
//
// * Tensor memory (TMEM): 128 lanes x 512 32-bit columns per SM; an address is (lane << 16) | column.
//   A warp may touch only its lane quarter 32 * (warp % 4) .. +31 with tcgen05.ld / tcgen05.st.
// * tcgen05.mma.cta_group::1.kind::f16: D[M x N] (fp32, TMEM) (+)= A[M x K] * B[K x N], K = 16 per
//   instruction, fp16 operands.  A comes from shared memory (descriptor) or from TMEM (M lanes, two
//   fp16 per 32-bit column, even k in the low half); B always from shared memory.  One thread issues.
// * Shared-memory operands use the no-swizzle canonical layout: 8 x 16-byte "core matrices" (8 rows of
//   16 bytes, 128 contiguous bytes).  K-major: a core matrix is 8 M/N rows x 8 consecutive k; MN-major:
//   8 consecutive k rows x 8 consecutive M/N elements.  The descriptor's SBO is the byte stride between
//   core matrices adjacent along M/N, LBO the stride between core matrices adjacent along K.
// * Completion: tcgen05.commit arrives on an mbarrier once every MMA issued before it by this thread
//   has finished; waits are bounded and report a timeout instead of spinning forever.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace pfa {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---------------------------------------------------------------------------------------- descriptors
// Shared-memory matrix descriptor, no swizzle (layout type 0), descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of kind::f16 with fp16 A and B and an fp32 accumulator.
//   a_mn / b_mn: operand stored MN-major (else K-major); neg_a / neg_b: negate that operand.
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N, bool a_mn, bool b_mn, bool neg_a = false,
                                                 bool neg_b = false) {
    return (1u << 4)                              // D format: f32
           | (0u << 7) | (0u << 10)                // A, B format: f16
           | ((neg_a ? 1u : 0u) << 13) | ((neg_b ? 1u : 0u) << 14)
           | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16)
           | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// ---------------------------------------------------------------------------------------- MMA issue
// D (+)= A(smem) * B(smem)
__device__ __forceinline__ void mma_ss(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                       bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate ? 1u : 0u)
        : "memory");
}

// D (+)= A(TMEM) * B(smem)
__device__ __forceinline__ void mma_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc,
                                       bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate ? 1u : 0u)
        : "memory");
}

// arrive on `bar` when all MMAs issued so far by this thread are complete
__device__ __forceinline__ void commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// ---------------------------------------------------------------------------------------- fences
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// ---------------------------------------------------------------------------------------- mbarrier
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }

// Wait for the phase with parity `parity` to complete; gives up after `limit` polls (returns false).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit = 1u << 26) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// ---------------------------------------------------------------------------------------- TMEM
// Allocation by one full warp; the base address is written to shared memory `slot`.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(base), "r"(ncols) : "memory");
}

// 32 lanes x 32 bits, 16 consecutive columns: thread t gets lane (taddr.lane + t), columns c..c+15
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
        "%13, %14, %15, %16};\n" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
        "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&r)[8]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};\n" ::"r"(taddr),
                 "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }

// ---------------------------------------------------------------------------------------- layouts
// Byte offset of element (row, k) of a K-major no-swizzle operand with `kdim` columns of 16-bit
// elements: core matrices ordered K-fastest (LBO = 128, SBO = kdim * 16).
__host__ __device__ constexpr uint32_t kmajor_off(int row, int k, int kdim) {
    return (uint32_t)(((row >> 3) * (kdim >> 3) + (k >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2);
}
// Byte offset of element (k, col) of an MN-major no-swizzle operand with `ndim` columns: core matrices
// ordered MN-fastest (SBO = 128 between adjacent MN groups, LBO = ndim * 16 between adjacent K groups).
__host__ __device__ constexpr uint32_t mnmajor_off(int k, int col, int ndim) {
    return (uint32_t)(((k >> 3) * (ndim >> 3) + (col >> 3)) * 128 + (k & 7) * 16 + (col & 7) * 2);
}

}  // namespace tc
}  // namespace pfa
