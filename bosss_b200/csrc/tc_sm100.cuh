// tc_sm100.cuh -- 5th-generation tensor-core (tcgen05) primitives for sm_100a, inline PTX.
//
// Only what the split-precision contraction kernels use: tensor-memory allocation, the
// shared-memory matrix descriptor of a K-major operand without swizzle, the instruction
// descriptor of an 8-bit integer MMA with 32-bit integer accumulation (kind::i8), the MMA
// itself issued by one thread, completion tracking through an mbarrier, and loads of the
// accumulator from tensor memory. Single CTA (cta_group::1), no clusters, no multicast.
//
// Operand layout in shared memory (K-major, SWIZZLE_NONE): the operand tile of R rows and
// K bytes is stored as K/16 column chunks of R rows x 16 bytes each, chunk c at byte offset
// c * R * 16, row r of the chunk at r * 16. In the canonical form of the descriptor this is
// core matrices of 8 rows x 16 bytes (128 contiguous bytes), stride-dimension byte offset
// (SBO, between 8-row groups) = 128, leading-dimension byte offset (LBO, between the two
// 16-byte K chunks of one MMA) = R * 16. One kind::i8 MMA consumes K = 32 bytes (two
// chunks); the next K step starts 2 * R * 16 bytes further.
//
// Accumulator layout (M = 128, cta_group::1): row i of D is tensor-memory lane i, column j
// is the 32-bit column (base + j). Warp w of the CTA may read lanes 32 (w % 4) .. +31.
#pragma once
#include <cstdint>

namespace bosss {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor: K-major, no swizzle (layout type 0), version 1 (sm_100)
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;   // descriptor version
    return d;                 // base offset 0, LBO mode 0, swizzle none
}

// instruction descriptor of kind::i8: signed 8-bit A and B (both K-major), S32 accumulator
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N) {
    return (2u << 4)                        // D format S32
           | (1u << 7) | (1u << 10)         // A, B signed 8-bit
           | ((uint32_t)(N >> 3) << 17)     // N / 8
           | ((uint32_t)(M >> 4) << 24);    // M / 16
}

// tensor-memory allocation by one whole warp; the address is written to *slot (shared)
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D[taddr] (+)= A * B^T, one thread issues
__device__ __forceinline__ void mma_i8(uint32_t taddr, uint64_t adesc, uint64_t bdesc, uint32_t idesc, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(taddr),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)accumulate));
}

// the mbarrier receives one arrival when all previously issued MMAs of this thread are done
__device__ __forceinline__ void commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}

// bounded wait for phase `parity` of the mbarrier; false if it did not complete
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t max_iters) {
    const uint32_t a = smem_u32(mbar);
    for (uint32_t it = 0; it < max_iters; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred q;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, q;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 16 consecutive 32-bit accumulator columns of this thread's lane
__device__ __forceinline__ void ld16(uint32_t taddr, int32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

}  // namespace tc
}  // namespace bosss
