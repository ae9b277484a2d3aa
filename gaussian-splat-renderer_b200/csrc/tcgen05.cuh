// Fifth-generation tensor core helpers for sm_100a (tcgen05): shared-memory matrix descriptors in
// the no-swizzle K-major layout, the instruction descriptor of a BF16 x BF16 -> FP32 product,
// tensor-memory (TMEM) allocation, the single-thread MMA issue with its mbarrier commit, TMEM
// loads into registers, and the fences between them. Only what the colour decode uses.
//
// Layout of an R x K BF16 operand (K-major, no swizzle) in shared memory: 8 x 8 "core matrices"
// of 8 rows x 16 bytes stored as 128 contiguous bytes; element (r, k) lives at
//   (r / 8) * (K / 8) * 128 + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2.
// One MMA consumes K = 16 (two core-matrix columns): its descriptor starts at the k-step's first
// column (ks * 256 bytes), the leading-dimension offset is the distance between the two columns
// (128 bytes) and the stride-dimension offset the distance between row groups ((K / 8) * 128).
#pragma once

#include <cstdint>

namespace gsr {
namespace tc {

__device__ __forceinline__ uint32_t smem32(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

// Byte offset of element (r, k) of an R x K operand in the layout above.
__host__ __device__ constexpr uint32_t operandOffset(uint32_t r, uint32_t k, uint32_t K) {
    return (r >> 3) * (K >> 3) * 128u + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// Shared-memory matrix descriptor: start address, leading- and stride-dimension byte offsets
// (all >> 4), version 1 (sm_100), base offset 0, no swizzle.
__device__ __forceinline__ uint64_t smemDescriptor(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}
// The descriptor of k-step ks (K = 16 columns) of an operand with K columns at `base`.
__device__ __forceinline__ uint64_t operandDescriptor(uint32_t base, uint32_t ks, uint32_t K) {
    return smemDescriptor(base + ks * 256u, 128u, (K >> 3) * 128u);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major, M x N.
__host__ __device__ constexpr uint32_t instrDescriptorBf16(uint32_t M, uint32_t N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

// TMEM allocation of `cols` columns (a power of two >= 32) by one whole warp; the base address
// is written to shared memory.
__device__ __forceinline__ void tmemAlloc(uint32_t* slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem32(slot)), "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmemFree(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

__device__ __forceinline__ void fenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes made visible to the tensor core's (async proxy) reads.
__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D[tmem] (+)= A x B, issued by one thread.
__device__ __forceinline__ void mma(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
        "}" ::"r"(dTmem),
        "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(accumulate ? 1u : 0u)
        : "memory");
}
// The MMAs this thread issued so far arrive on the mbarrier once they have completed.
__device__ __forceinline__ void commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem32(mbar))
                 : "memory");
}

// 32 lanes x 32 bits, repeated 16 / 32 times along the columns: thread i of the warp gets 16 /
// 32 consecutive columns of TMEM lane (warp quarter x 32 + i) starting at taddr's column.
__device__ __forceinline__ void ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}
__device__ __forceinline__ void waitLd() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void mbarInit(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem32(mbar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Waits for the phase with the given parity to complete, at most `limit` polls; false on expiry.
__device__ __forceinline__ bool mbarWait(uint64_t* mbar, uint32_t parity, uint32_t limit) {
    for (uint32_t n = 0; n < limit; ++n) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem32(mbar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

}  // namespace tc
}  // namespace gsr
