/* BF16 tcgen05 GEMMs of the learned proposal network (training and inference).

   One kernel, D = A * B^T with A (M x K) and B (N x K) row-major BF16 in global memory and
   FP32 accumulation in tensor memory, covers every product the network needs:
     forward     Z = X W^T            (B = W, out x in)
     data grad   dH = dZ W            (B = W^T, stored transposed)
     weight grad dW = dZ^T X          (A = dZ^T, B = X^T: activations are also stored transposed)
   A CTA owns 128 rows of D and all N <= 256 columns.  K is consumed in chunks of 64: the 128
   threads stage the A and B chunks into shared memory in the canonical K-major layout
   (tc_gemm.cuh), one thread issues the four 128 x N x 16 tcgen05.mma of the chunk and commits
   them to an mbarrier, and all threads wait (bounded) before reusing the buffers.  The epilogue
   reads each thread's row from tensor memory 16 columns at a time (tcgen05.ld.32x32b) and applies
   one of the fused epilogues below. */
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "pt_internal.h"
#include "pt_kernels.h"
#include "tc_gemm.cuh"

namespace {

using bf16 = __nv_bfloat16;

}  // namespace

/* Epilogue of a GEMM, applied to D[r][c] (r < M, c < N). */
struct GemmEpi {
    enum Mode { STORE_F32 = 0, BIAS_RELU = 1, RELU_GRAD = 2, BIAS_F32 = 3 };
    int mode;
    float *c;                /* STORE_F32 / BIAS_F32 output, ldc */
    int ldc;
    const float *bias;       /* BIAS_RELU / BIAS_F32 */
    bf16 *h;                 /* BIAS_RELU / RELU_GRAD row-major BF16 output, ldh */
    int ldh;
    bf16 *ht;                /* optional transposed BF16 output [N x M], ldht */
    int ldht;
    const bf16 *mask;        /* RELU_GRAD: the layer's ReLU output; gradient passes where > 0 */
    int ldm;
    int *err;                /* set to 1 when a bounded wait gives up */
};

namespace {

template<int N>
__global__ void __launch_bounds__(128)
k_gemm(const bf16 *__restrict__ A, int lda, const bf16 *__restrict__ B, int ldb, int M, int K, GemmEpi epi) {
    constexpr int NCOLS = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
    constexpr uint32_t IDESC = ptc::idesc_bf16_f32(128, N);
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *sA = smem;                 /* 128 x 64 BF16 */
    unsigned char *sB = smem + 128 * 64 * 2;  /* N x 64 BF16 */
    __shared__ uint64_t mbar;
    __shared__ uint32_t tslot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * 128;
    if (warp == 0) ptc::tmem_alloc(&tslot, NCOLS);
    if (tid == 0) {
        ptc::mbar_init(&mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    ptc::tc_fence_before();
    __syncthreads();
    ptc::tc_fence_after();
    const uint32_t tmem = tslot;
    unsigned phase = 0;
    bool ok = true;
    for (int kc = 0; kc < K && ok; kc += 64) {
        const int kw = min(64, K - kc);
        const int nv = kw / 8;
        for (int i = tid; i < 128 * nv; i += 128) {
            int r = i / nv, k = (i % nv) * 8;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (m0 + r < M) v = *reinterpret_cast<const uint4 *>(A + (size_t) (m0 + r) * lda + kc + k);
            *reinterpret_cast<uint4 *>(sA + ptc::kmajor_offset(r, k, 128)) = v;
        }
        for (int i = tid; i < N * nv; i += 128) {
            int r = i / nv, k = (i % nv) * 8;
            *reinterpret_cast<uint4 *>(sB + ptc::kmajor_offset(r, k, N)) =
                *reinterpret_cast<const uint4 *>(B + (size_t) r * ldb + kc + k);
        }
        ptc::fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            ptc::tc_fence_after();
            const uint32_t a0 = ptc::smem_u32(sA), b0 = ptc::smem_u32(sB);
            for (int ks = 0; ks < kw / 16; ks++)
                ptc::mma_bf16(tmem, ptc::smem_desc(a0 + ks * 128 * 32), ptc::smem_desc(b0 + ks * N * 32), IDESC,
                              (kc > 0 || ks > 0) ? 1 : 0);
            ptc::mma_commit(&mbar);
        }
        /* the outcome must be uniform: the tensor-memory loads below are warp-collective */
        ok = __syncthreads_and(ptc::mbar_wait(&mbar, phase) ? 1 : 0) != 0;
        phase ^= 1u;
        ptc::tc_fence_after();
    }
    if (ok) {
        const int r = m0 + warp * 32 + lane;
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            ptc::tmem_ld16(tmem + ((uint32_t) (warp * 32) << 16) + (uint32_t) c0, v);
            if (r >= M) continue;
#pragma unroll
            for (int j = 0; j < 16; j++) {
                const int c = c0 + j;
                float x = v[j];
                switch (epi.mode) {
                    case GemmEpi::STORE_F32:
                        epi.c[(size_t) r * epi.ldc + c] = x;
                        break;
                    case GemmEpi::BIAS_F32:
                        epi.c[(size_t) r * epi.ldc + c] = x + epi.bias[c];
                        break;
                    case GemmEpi::BIAS_RELU: {
                        bf16 hv = __float2bfloat16_rn(fmaxf(x + epi.bias[c], 0.f));
                        epi.h[(size_t) r * epi.ldh + c] = hv;
                        if (epi.ht) epi.ht[(size_t) c * epi.ldht + r] = hv;
                        break;
                    }
                    case GemmEpi::RELU_GRAD: {
                        bool pass = __bfloat162float(epi.mask[(size_t) r * epi.ldm + c]) > 0.f;
                        bf16 g = __float2bfloat16_rn(pass ? x : 0.f);
                        epi.h[(size_t) r * epi.ldh + c] = g;
                        if (epi.ht) epi.ht[(size_t) c * epi.ldht + r] = g;
                        break;
                    }
                }
            }
        }
    } else if (tid == 0 && epi.err) {
        atomicExch(epi.err, 1);
    }
    if (!ok) ptc::mbar_wait(&mbar, phase ^ 1u);   /* one more bounded wait for work still in flight */
    ptc::tc_fence_before();
    __syncthreads();
    if (warp == 0) ptc::tmem_dealloc(tmem, NCOLS);
}

}  // namespace

/* D = A * B^T for A [M x K], B [N x K] row-major BF16 (lda, ldb multiples of 8, K a multiple
   of 16, N in {16, 32, 64, 128, 256}); the epilogue decides what is written. */
pt_status pt_gemm_bf16(const void *A, int lda, const void *B, int ldb, int M, int N, int K, const GemmEpi &epi,
                       cudaStream_t st) {
    if (M < 1 || K < 16 || K % 16 || lda % 8 || ldb % 8)
        return pt_fail(PT_BAD_ARG, "gemm: M=%d K=%d lda=%d ldb=%d", M, K, lda, ldb);
    dim3 grid((M + 127) / 128);
    const int smem = 128 * 64 * 2 + N * 64 * 2;
    const bf16 *a = (const bf16 *) A, *b = (const bf16 *) B;
#define PT_GEMM_CASE(NN) \
    case NN: \
        PT_CUDA(cudaFuncSetAttribute(k_gemm<NN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)); \
        k_gemm<NN><<<grid, 128, smem, st>>>(a, lda, b, ldb, M, K, epi); \
        break;
    switch (N) {
        PT_GEMM_CASE(16) PT_GEMM_CASE(32) PT_GEMM_CASE(64) PT_GEMM_CASE(128) PT_GEMM_CASE(256)
        default: return pt_fail(PT_UNSUPPORTED, "gemm: N=%d", N);
    }
#undef PT_GEMM_CASE
    PT_LAUNCHED();
    return PT_OK;
}

extern "C" {

/* Diagnostics (no reference counterpart): C = A * B^T in FP32 through the tcgen05 GEMM, device
   pointers; *err_flag (device int, may be NULL) is set when a bounded wait gave up. */
pt_status pt_tc_gemm_f32(const void *A, int lda, const void *B, int ldb, float *C, int ldc, int M, int N, int K,
                         int *err_flag, void *stream) {
    GemmEpi e;
    memset(&e, 0, sizeof(e));
    e.mode = GemmEpi::STORE_F32;
    e.c = C;
    e.ldc = ldc;
    e.err = err_flag;
    return pt_gemm_bf16(A, lda, B, ldb, M, N, K, e, (cudaStream_t) stream);
}

}  // extern "C"
