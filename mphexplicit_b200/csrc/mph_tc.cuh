// tcgen05 (5th-generation tensor core) primitives for sm_100a, written as
// inline PTX: shared-memory matrix descriptors, the BF16 MMA with an FP32
// accumulator in tensor memory (TMEM), commit to an mbarrier, TMEM
// allocation and loads, and the proxy/thread-sync fences around them.
//
// Operand layout used throughout: the no-swizzle "core matrix" layout.  A
// bf16 tile with R rows and C columns (C contiguous) is stored as 8x8 core
// matrices of 128 contiguous bytes:
//     byte(r, c) = (r / 8) * (C * 16) + (c / 8) * 128 + (r % 8) * 16 + (c % 8) * 2
// The same bytes serve as a K-major operand (rows = M or N, columns = K) and
// as an MN-major operand (columns = M or N, rows = K):
//     K-major : leading byte offset (K direction) 128, stride byte offset C*16,
//               one K=16 step advances the start address by 256 bytes;
//     MN-major: leading byte offset (K direction) C*16, stride byte offset 128,
//               one K=16 step advances the start address by 32*C bytes.
#pragma once
#include <cstdint>

namespace mph {
namespace tc {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (r, c) in a core-matrix tile with C columns
__host__ __device__ __forceinline__ uint32_t core_off(int r, int c, int C) {
    return (uint32_t)((r >> 3) * (C * 16) + (c >> 3) * 128 + (r & 7) * 16 + (c & 7) * 2);
}

// Shared-memory matrix descriptor (no swizzle): start address, leading and
// stride byte offsets (all in 16-byte units), descriptor version 1 (bits 46-47).
__device__ __forceinline__ uint64_t desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}
__device__ __forceinline__ uint64_t desc_k(uint32_t saddr, int C) { return desc(saddr, 128, (uint32_t)C * 16); }
__device__ __forceinline__ uint64_t desc_mn(uint32_t saddr, int C) { return desc(saddr, (uint32_t)C * 16, 128); }

// Instruction descriptor, kind::f16 with BF16 inputs and an FP32 accumulator:
// D format bits 4-5, A/B format bits 7-9 / 10-12, A/B major bits 15/16,
// N>>3 bits 17-22, M>>4 bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A * B, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

// Arrive once on the mbarrier when every MMA issued so far by this thread is done.
__device__ __forceinline__ void commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Wait for the phase with the given parity to complete; gives up after
// `limit` polls and returns false (the caller records the error).
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, long long limit) {
    for (long long it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// TMEM allocation by one full warp; the base address is written to *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (warp w of the
// warpgroup reads lanes 32w..32w+31; taddr carries the lane in bits 16-31).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

}  // namespace tc
}  // namespace mph
