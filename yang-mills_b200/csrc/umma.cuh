// umma.cuh -- fifth-generation tensor-core (tcgen05) building blocks for
// sm_100a: shared-memory matrix descriptors in the no-swizzle canonical
// layout, the kind::f16 instruction descriptor (BF16 operands, FP32
// accumulator), MMA issue and commit, tensor-memory allocation and loads,
// and an mbarrier wait with a time bound.
//
// Operand tiles in shared memory: 8x8 core matrices of 16-bit elements, each
// 8 rows of 16 contiguous bytes (128 bytes).  Element (r, c) of an R x C tile
// whose columns are the contiguous dimension lives at byte
//     (r / 8) * (C / 8) * 128 + (c / 8) * 128 + (r % 8) * 16 + (c % 8) * 2.
// Read as a K-major operand (rows = M or N, columns = K) the descriptor has
// leading byte offset 128 (next 8 columns) and stride byte offset
// (C / 8) * 128 (next 8 rows).  Read as an MN-major operand (rows = K,
// columns = M or N) the same bytes take stride byte offset 128 (next 8
// columns of M/N) and leading byte offset (C / 8) * 128 (next 8 rows of K).
// One kind::f16 MMA consumes K = 16, i.e. two core matrices along K.
#pragma once

#include <cstdint>

namespace ym {
namespace umma {

__device__ __forceinline__ uint32_t tile_offset(int r, int c, int cols) {
    return (uint32_t)((r >> 3) * (cols >> 3) * 128 + (c >> 3) * 128 + (r & 7) * 16 + (c & 7) * 2);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Matrix descriptor, no swizzle: start address, leading- and stride-dimension
// byte offsets (each stored >> 4), descriptor version 1 (bits 46-47), base
// offset 0, layout type 0.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: D format F32 (bits 4-5 = 1), A and B
// format BF16 (bits 7-9, 10-12 = 1), A/B major (bits 15, 16; 1 = MN-major),
// N >> 3 (bits 17-22), M >> 4 (bits 24-28).
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n, int a_mn_major, int b_mn_major) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn_major << 15) |
           ((uint32_t)b_mn_major << 16) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// D[tmem] (+)= A * B^T, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrive once on the mbarrier when every MMA this thread issued so far has
// completed.
__device__ __forceinline__ void commit(uint64_t *mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :
                 : "r"(smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Generic-proxy shared-memory writes visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_u32(mbar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for the phase with the given parity to complete; gives up after
// limit_ns nanoseconds and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, uint64_t limit_ns) {
    const uint32_t addr = smem_u32(mbar);
    const uint64_t t0 = global_ns();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
}

// Tensor-memory allocation (whole warp; ncols a power of two >= 32).
__device__ __forceinline__ void tmem_alloc(uint32_t *smem_slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(smem_slot)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive 32-bit columns of the warp's 32 lanes (lane = thread), with
// the wait for completion inside the same statement.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace umma
}  // namespace ym
