/* tcgen05 building blocks for the proposal network's BF16 GEMMs (sm_100a).

   D[128 x N] (FP32, in tensor memory) += A[128 x 16] * B[N x 16]^T per tcgen05.mma instruction,
   both operands in shared memory in the K-major, no-swizzle canonical layout: "core matrices"
   of 8 rows x 16 bytes (8 BF16 along K), rows 16 B apart, the two K halves of a 16-wide K step
   LBO = 128 B apart and consecutive 8-row groups SBO = 256 B apart.  Element (r, k) of a
   K-step tile of R rows therefore lives at byte
       (k / 16) * (R * 32) + (r / 8) * 256 + ((k % 16) / 8) * 128 + (r % 8) * 16 + (k % 8) * 2.
   Descriptor encodings follow the PTX ISA's tcgen05 matrix and instruction descriptors (the
   same bit layout as CUTLASS's UMMA::SmemDescriptor / UMMA::InstrDescriptor).

   Every wait on an mbarrier is bounded: after PT_TC_SPIN_LIMIT polls the caller records an error
   and leaves instead of hanging. */
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define PT_TC_SPIN_LIMIT (1u << 24)

namespace ptc {

/* Byte offset of (r, k) in a K-major no-swizzle tile of R rows (see above). */
__device__ __forceinline__ uint32_t kmajor_offset(int r, int k, int R) {
    return (uint32_t) ((k >> 4) * (R * 32) + (r >> 3) * 256 + ((k >> 3) & 1) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t) __cvta_generic_to_shared(p);
}

/* Shared-memory matrix descriptor: start >> 4 in [0,14), LBO >> 4 in [16,30), SBO >> 4 in
   [32,46), version 1 in [46,48), base offset 0, layout type 0 (no swizzle) in [61,64). */
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
    return (uint64_t) ((saddr & 0x3FFFF) >> 4) | ((uint64_t) (128 >> 4) << 16) | ((uint64_t) (256 >> 4) << 32) |
           ((uint64_t) 1 << 46);
}

/* Instruction descriptor, kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A and B (bits 7-9,
   10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 in [17,23), M >> 4 in [24,29). */
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t) (N >> 3) << 17) | ((uint32_t) (M >> 4) << 24);
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

/* Waits for the mbarrier phase `parity` to complete; false if the bound ran out. */
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
    uint32_t addr = smem_u32(bar);
    for (unsigned i = 0; i < PT_TC_SPIN_LIMIT; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done) : "r"(addr), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

/* Tensor-memory allocation by one full warp; the address is written to *slot. */
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

/* D (tensor memory) = A * B^T (+ D when accumulate), one 128 x N x 16 step; no output lane is
   disabled. */
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, int accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
        : "memory");
}

/* Arrives on `bar` once all previously issued tcgen05.mma of this thread have completed. */
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

/* 16 consecutive FP32 columns of this thread's tensor-memory lane. */
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

}  // namespace ptc
