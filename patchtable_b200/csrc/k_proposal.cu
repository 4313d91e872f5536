/* Learned proposal network: features, labels, training and fused inference.

   The network maps a query patch's descriptor to a distribution over table cells and proposes the
   8 most probable cells; their stored b patches are then scored by the exact SSD like any other
   candidate.  Network: 16 inputs -> 128 -> ReLU -> 128 -> ReLU -> 32 logits, BF16 weights and
   activations, FP32 accumulation (tensor memory), FP32 master weights and Adam moments.

   Class space.  A softmax over the 1e8 cells of the table would need a 128 x 1e8 output layer, so
   the distribution is factorised over the table's grid dimensions: for each grid dimension d
   (at most 6) five logits score the bin of the match relative to the query patch's own bin,
   offset -2..+2; 6 x 5 = 30 logits (2 unused).  Offsets that leave the grid are masked out of the
   softmax.  A cell's probability is the product of its per-dimension probabilities; the 8 most
   probable cells (exact top-8 of the product, by beam search) are the proposals and the most
   probable cell's probability is the confidence.

   Inputs (per query patch, per grid dimension d): the descriptor value normalised to the table's
   range, (v - min) / range - 1/2, and its signed position inside its bin, (v - centre) / (distance
   to the bin boundary on that side); 12 values, 4 zeros pad the row to 16.

   Labels: the bin offsets, clamped to -2..+2, from the query patch's bin to the bin of the b patch
   the plain method matched it with.

   Training uses the tcgen05 GEMM of k_mlp.cu with fused epilogues (bias + ReLU with transposed
   copies for the weight gradients, ReLU masking of the data gradients).  Inference is one
   persistent kernel: per 128-patch tile it computes the features, runs the three layers on the
   tensor cores with the weights resident in shared memory and the accumulators in tensor memory,
   and ends with the masked softmax and top-8 search in registers. */
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "pt_bins.cuh"
#include "pt_internal.h"
#include "pt_kernels.h"
#include "tc_gemm.cuh"

using bf16 = __nv_bfloat16;

/* k_mlp.cu */
struct GemmEpi {
    enum Mode { STORE_F32 = 0, BIAS_RELU = 1, RELU_GRAD = 2, BIAS_F32 = 3 };
    int mode;
    float *c;
    int ldc;
    const float *bias;
    bf16 *h;
    int ldh;
    bf16 *ht;
    int ldht;
    const bf16 *mask;
    int ldm;
    int *err;
};
pt_status pt_gemm_bf16(const void *A, int lda, const void *B, int ldb, int M, int N, int K, const GemmEpi &epi,
                       cudaStream_t st);

namespace {

constexpr int NT = 256;
constexpr int PIN = PT_PROP_IN, PH = PT_PROP_HIDDEN, POUT = PT_PROP_OUT, PD = PT_PROP_DIMS, PC = PT_PROP_CLASSES,
              PK = PT_PROP_TOPK;

/* Offsets (floats) of the tensors in the parameter vector. */
constexpr int OFF_W1 = 0;                      /* PH x PIN */
constexpr int OFF_B1 = OFF_W1 + PH * PIN;      /* PH */
constexpr int OFF_W2 = OFF_B1 + PH;            /* PH x PH */
constexpr int OFF_B2 = OFF_W2 + PH * PH;       /* PH */
constexpr int OFF_W3 = OFF_B2 + PH;            /* POUT x PH */
constexpr int OFF_B3 = OFF_W3 + POUT * PH;     /* POUT */
constexpr int NPARAM = OFF_B3 + POUT;

/* Per-dimension bin parameters of the table the network works on. */
struct PropPlan {
    int G;
    int nslices[PD];
    long long stride[PD];
    float min_val[PD], range[PD];
    int pofs[PD];   /* dimension d: centres at part[pofs[d]], left sizes +nslices, right sizes +2 nslices */
};

/* Features and bins of one patch (descriptor v). */
__device__ __forceinline__ void prop_features(const PropPlan &pl, const float *__restrict__ part,
                                              const int *__restrict__ to_bin, const float *__restrict__ v, float *f,
                                              int *bin) {
#pragma unroll
    for (int d = 0; d < PD; d++) {
        f[d] = 0.f;
        f[PD + d] = 0.f;
        bin[d] = 0;
        if (d < pl.G) {
            const float x = v[d];
            const int b = pt_get_bin(pl.min_val[d], pl.range[d], to_bin + d * PT_NMAP, x);
            bin[d] = b;
            const float *P = part + pl.pofs[d];
            const int ns = pl.nslices[d];
            const float c = __ldg(P + b);
            const float s = x >= c ? __ldg(P + 2 * ns + b) : __ldg(P + ns + b);
            const float u = s > 0.f ? (x - c) / s : 0.f;
            f[PD + d] = fminf(fmaxf(u, -2.f), 2.f);
            const float r = pl.range[d] > 0.f ? (x - pl.min_val[d]) / pl.range[d] : 0.5f;
            f[d] = fminf(fmaxf(r, -0.5f), 1.5f) - 0.5f;
        }
    }
#pragma unroll
    for (int i = 2 * PD; i < PIN; i++) f[i] = 0.f;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

/* Training samples: features X [n x 16] BF16 and 8 label bytes per patch.  Byte d < 6 is
   offset | lo << 3 | hi << 5 (offset 0..4 stands for -2..+2; lo, hi = valid offsets below and above
   the patch's own bin, at most 2), 0xFF for unused dimensions or an invalid match; byte 6 is 1
   when every offset lay within -2..+2 before clamping. */
__global__ void k_prop_samples(const PropPlan pl, const float *__restrict__ part, const int *__restrict__ to_bin,
                               const float *__restrict__ qdesc, int ds, int n, const float *__restrict__ bdesc,
                               int bew, int beh, const double *__restrict__ ann, bf16 *X, unsigned char *lab) {
    const int p = blockIdx.x * NT + threadIdx.x;
    if (p >= n) return;
    float f[PIN];
    int ba[PD];
    prop_features(pl, part, to_bin, qdesc + (size_t) p * ds, f, ba);
    uint4 r0 = make_uint4(pack_bf16(f[0], f[1]), pack_bf16(f[2], f[3]), pack_bf16(f[4], f[5]), pack_bf16(f[6], f[7]));
    uint4 r1 = make_uint4(pack_bf16(f[8], f[9]), pack_bf16(f[10], f[11]), pack_bf16(f[12], f[13]), pack_bf16(f[14], f[15]));
    reinterpret_cast<uint4 *>(X)[2 * (size_t) p] = r0;
    reinterpret_cast<uint4 *>(X)[2 * (size_t) p + 1] = r1;
    const double ax = ann[3 * (size_t) p], ay = ann[3 * (size_t) p + 1];
    const bool valid = ax >= 0.0 && ay >= 0.0 && ax < (double) bew && ay < (double) beh;
    const int bx = valid ? (int) ax : 0, by = valid ? (int) ay : 0;
    unsigned char out[8];
    bool exact = valid;
#pragma unroll
    for (int d = 0; d < PD; d++) {
        out[d] = 0xFF;
        if (d < pl.G && valid) {
            const float vb = bdesc[((size_t) by * bew + bx) * ds + d];
            const int bb = pt_get_bin(pl.min_val[d], pl.range[d], to_bin + d * PT_NMAP, vb);
            int off = bb - ba[d];
            exact &= off >= -2 && off <= 2;
            off = off < -2 ? -2 : (off > 2 ? 2 : off);
            const int lo = min(2, ba[d]), hi = min(2, pl.nslices[d] - 1 - ba[d]);
            out[d] = (unsigned char) ((off + 2) | (lo << 3) | (hi << 5));
        }
    }
    out[6] = exact ? 1 : 0;
    out[7] = 0;
    uint2 w;
    memcpy(&w, out, 8);
    reinterpret_cast<uint2 *>(lab)[p] = w;
}

__global__ void k_to_bf16(const float *__restrict__ p, bf16 *w1, bf16 *w2, bf16 *w2t, bf16 *w3, bf16 *w3t) {
    const int i = blockIdx.x * NT + threadIdx.x;
    if (i < PH * PIN) w1[i] = __float2bfloat16_rn(p[OFF_W1 + i]);
    if (i < PH * PH) {
        const int o = i / PH, k = i % PH;
        const bf16 v = __float2bfloat16_rn(p[OFF_W2 + i]);
        w2[i] = v;
        w2t[k * PH + o] = v;
    }
    if (i < POUT * PH) {
        const int o = i / PH, k = i % PH;
        const bf16 v = __float2bfloat16_rn(p[OFF_W3 + i]);
        w3[i] = v;
        w3t[k * POUT + o] = v;
    }
}

/* X [B x 16] -> X^T [16 x B]. */
__global__ void k_transpose_x(const bf16 *__restrict__ X, int B, bf16 *Xt) {
    const int r = blockIdx.x * NT + threadIdx.x;
    if (r >= B) return;
#pragma unroll
    for (int c = 0; c < PIN; c++) Xt[(size_t) c * B + r] = X[(size_t) r * PIN + c];
}

/* Masked softmax cross-entropy per grid dimension.  dZ3 = (softmax - onehot) / B as BF16, row-major
   and transposed; the loss sum is accumulated in loss[0] (FP32). */
__global__ void k_ce(const float *__restrict__ logits, const unsigned char *__restrict__ labels, int B, bf16 *dz,
                     bf16 *dzt, float *loss) {
    const int r = blockIdx.x * NT + threadIdx.x;
    float l = 0.f;
    if (r < B) {
        const float *z = logits + (size_t) r * POUT;
        float g[POUT];
#pragma unroll
        for (int c = 0; c < POUT; c++) g[c] = 0.f;
#pragma unroll
        for (int d = 0; d < PD; d++) {
            const unsigned char b = labels[(size_t) r * 8 + d];
            if (b == 0xFF) continue;
            const int k0 = 2 - ((b >> 3) & 3), k1 = 2 + ((b >> 5) & 3), y = b & 7;
            float m = -3.0e38f;
#pragma unroll
            for (int k = 0; k < PC; k++)
                if (k >= k0 && k <= k1) m = fmaxf(m, z[d * PC + k]);
            float e[PC], s = 0.f;
#pragma unroll
            for (int k = 0; k < PC; k++) {
                e[k] = (k >= k0 && k <= k1) ? __expf(z[d * PC + k] - m) : 0.f;
                s += e[k];
            }
#pragma unroll
            for (int k = 0; k < PC; k++) g[d * PC + k] = (e[k] / s - (k == y ? 1.f : 0.f)) / (float) B;
            l += -(z[d * PC + y] - m - __logf(s));
        }
#pragma unroll
        for (int c = 0; c < POUT; c++) {
            const bf16 v = __float2bfloat16_rn(g[c]);
            dz[(size_t) r * POUT + c] = v;
            dzt[(size_t) c * B + r] = v;
        }
    }
    for (int o = 16; o; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && l != 0.f) atomicAdd(loss, l);
}

/* out[row] = sum of BF16 row `row` of a [rows x B] array (bias gradients). */
__global__ void k_rowsum(const bf16 *__restrict__ m, int B, float *out) {
    const int row = blockIdx.x;
    float s = 0.f;
    for (int i = threadIdx.x; i < B; i += NT) s += __bfloat162float(m[(size_t) row * B + i]);
    __shared__ float red[NT / 32];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int i = 0; i < NT / 32; i++) t += red[i];
        out[row] = t;
    }
}

/* Gathers the gradient pieces into one vector laid out like the parameters. */
__global__ void k_pack_grad(const float *gw1, const float *gb1, const float *gw2, const float *gb2, const float *gw3t,
                            const float *gb3, float *g) {
    const int i = blockIdx.x * NT + threadIdx.x;
    if (i < PH * PIN) g[OFF_W1 + i] = gw1[i];
    if (i < PH) { g[OFF_B1 + i] = gb1[i]; g[OFF_B2 + i] = gb2[i]; }
    if (i < PH * PH) g[OFF_W2 + i] = gw2[i];
    if (i < POUT * PH) { const int o = i / PH, k = i % PH; g[OFF_W3 + i] = gw3t[k * POUT + o]; }
    if (i < POUT) g[OFF_B3 + i] = gb3[i];
}

/* AdamW: decoupled weight decay wd on every parameter. */
__global__ void k_adam(float *p, const float *g, float *m, float *v, int n, float lr, float b1, float b2, float eps,
                       float wd, float c1, float c2) {
    const int i = blockIdx.x * NT + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * ((mi / c1) / (sqrtf(vi / c2) + eps) + wd * p[i]);
}

/* ---- fused inference ---- */

/* One CTA per SM, 4 groups of 128 threads; each group runs its own 128-patch tiles through the
   three layers.  The weights are shared; each group has its own input tile, hidden-activation
   tile, mbarrier and 128 tensor-memory columns (all three layers accumulate there in turn: a
   layer's accumulator is read completely before the next layer's MMAs are issued). */
constexpr int NGROUP = 4;
constexpr int SM_W1 = 0;                          /* PH x PIN BF16, K-major */
constexpr int SM_W2 = SM_W1 + PH * PIN * 2;       /* PH x PH */
constexpr int SM_W3 = SM_W2 + PH * PH * 2;        /* POUT x PH */
constexpr int SM_BIAS = SM_W3 + POUT * PH * 2;    /* b1, b2, b3 (FP32) */
constexpr int SM_GROUPS = ((SM_BIAS + (2 * PH + POUT) * 4 + 127) / 128) * 128;
constexpr int SM_GX = 0;                          /* per group: 128 x PIN input tile */
constexpr int SM_GH = 128 * PIN * 2;              /* per group: 128 x PH hidden tile */
constexpr int SM_GSIZE = SM_GH + 128 * PH * 2;
constexpr int SM_TOTAL = SM_GROUPS + NGROUP * SM_GSIZE;
constexpr int INFER_COLS = 128 * NGROUP;          /* all 512 tensor-memory columns of the SM */

/* Stages a rows x K row-major BF16 matrix into the K-major canonical layout. */
__device__ __forceinline__ void stage_kmajor(unsigned char *dst, const bf16 *__restrict__ src, int rows, int K) {
    const int nv = K / 8;
    for (int i = threadIdx.x; i < rows * nv; i += blockDim.x) {
        const int r = i / nv, k = (i % nv) * 8;
        *reinterpret_cast<uint4 *>(dst + ptc::kmajor_offset(r, k, rows)) =
            *reinterpret_cast<const uint4 *>(src + (size_t) r * K + k);
    }
}

/* Hidden-layer epilogue: this thread's row of the accumulator (128 columns at taddr) + bias, ReLU,
   BF16, written as row r of the next layer's A operand. */
__device__ __forceinline__ void epi_hidden(uint32_t taddr, const float *bias, unsigned char *sH, int r) {
#pragma unroll 1
    for (int c0 = 0; c0 < PH; c0 += 16) {
        float v[16];
        ptc::tmem_ld16(taddr + (uint32_t) c0, v);
        uint32_t pk[8];
#pragma unroll
        for (int j = 0; j < 8; j++)
            pk[j] = pack_bf16(fmaxf(v[2 * j] + bias[c0 + 2 * j], 0.f), fmaxf(v[2 * j + 1] + bias[c0 + 2 * j + 1], 0.f));
        *reinterpret_cast<uint4 *>(sH + ptc::kmajor_offset(r, c0, 128)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        *reinterpret_cast<uint4 *>(sH + ptc::kmajor_offset(r, c0 + 8, 128)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
    }
}

/* Barrier of one 128-thread group (named barrier 1 + g; 0 is __syncthreads). */
__device__ __forceinline__ void group_sync(int g) {
    asm volatile("bar.sync %0, 128;" ::"r"(1 + g) : "memory");
}

/* Group barrier returning whether `v` holds on every thread of the group. */
__device__ __forceinline__ bool group_and(int g, bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, %2, 128, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r) : "r"((uint32_t) v), "r"(1 + g) : "memory");
    return r != 0;
}

/* The group waits for the commit of the current phase; the outcome is uniform over the group. */
__device__ __forceinline__ bool group_wait(int g, uint64_t *mbar, unsigned &phase) {
    const bool ok = group_and(g, ptc::mbar_wait(mbar, phase));
    if (ok) phase ^= 1u;
    ptc::tc_fence_after();
    return ok;
}

/* Writes this thread's features as row r of the input tile. */
__device__ __forceinline__ void put_x(unsigned char *sX, int r, const float *f) {
    *reinterpret_cast<uint4 *>(sX + ptc::kmajor_offset(r, 0, 128)) =
        make_uint4(pack_bf16(f[0], f[1]), pack_bf16(f[2], f[3]), pack_bf16(f[4], f[5]), pack_bf16(f[6], f[7]));
    *reinterpret_cast<uint4 *>(sX + ptc::kmajor_offset(r, 8, 128)) =
        make_uint4(pack_bf16(f[8], f[9]), pack_bf16(f[10], f[11]), pack_bf16(f[12], f[13]), pack_bf16(f[14], f[15]));
}

__device__ __forceinline__ void tile_features(const PropPlan &pl, const float *part, const int *to_bin,
                                              const float *qdesc, int ds, int p, int n, float *f, int *bin) {
    if (p < n) {
        prop_features(pl, part, to_bin, qdesc + (size_t) p * ds, f, bin);
    } else {
#pragma unroll
        for (int i = 0; i < PIN; i++) f[i] = 0.f;
#pragma unroll
        for (int d = 0; d < PD; d++) bin[d] = 0;
    }
}

/* Keeps (a, ca) the larger of the two pairs. */
__device__ __forceinline__ void cmpx(float &a, int &ca, float &b, int &cb) {
    if (b > a) {
        const float t = a; a = b; b = t;
        const int u = ca; ca = cb; cb = u;
    }
}

/* Exact top-8 cells of the factorised distribution, in registers.  Per grid dimension the masked
   log-softmax of its 5 logits is sorted (descending, 9-comparator network); the beam of the best
   8 prefixes is extended by the pairs (prefix i, class rank k) with (i+1)(k+1) <= 8 -- any other
   pair is beaten by at least 8 of these, as both lists are sorted -- so the new beam is column
   k = 0 (already in order) with the other 9 pairs inserted.  bs: log-probabilities (-3.4e38 when
   fewer than 8 cells exist), bc: 3 bits of class per dimension. */
__device__ __forceinline__ void top_cells(const float *z, const int *bin, const PropPlan &pl, float *bs, int *bc) {
    constexpr float NEG = -3.4e38f;
#pragma unroll
    for (int j = 0; j < PK; j++) { bs[j] = NEG; bc[j] = 0; }
    bs[0] = 0.f;
#pragma unroll
    for (int d = 0; d < PD; d++) {
        if (d < pl.G) {
            const int k0 = 2 - min(2, bin[d]), k1 = 2 + min(2, pl.nslices[d] - 1 - bin[d]);
            float m = NEG;
#pragma unroll
            for (int k = 0; k < PC; k++)
                if (k >= k0 && k <= k1) m = fmaxf(m, z[d * PC + k]);
            float s = 0.f;
#pragma unroll
            for (int k = 0; k < PC; k++)
                if (k >= k0 && k <= k1) s += __expf(z[d * PC + k] - m);
            const float ls = m + __logf(s);
            float v[PC];
            int c[PC];
#pragma unroll
            for (int k = 0; k < PC; k++) {
                v[k] = (k >= k0 && k <= k1) ? z[d * PC + k] - ls : NEG;
                c[k] = k << (3 * d);
            }
            cmpx(v[0], c[0], v[3], c[3]); cmpx(v[1], c[1], v[4], c[4]);
            cmpx(v[0], c[0], v[2], c[2]); cmpx(v[1], c[1], v[3], c[3]);
            cmpx(v[0], c[0], v[1], c[1]); cmpx(v[2], c[2], v[4], c[4]);
            cmpx(v[1], c[1], v[2], c[2]); cmpx(v[3], c[3], v[4], c[4]);
            cmpx(v[2], c[2], v[3], c[3]);
            float nv[PK];
            int nc[PK];
#pragma unroll
            for (int i = 0; i < PK; i++) {
                nv[i] = bs[i] > NEG ? bs[i] + v[0] : NEG;
                nc[i] = bc[i] | c[0];
            }
#pragma unroll
            for (int k = 1; k < PC; k++) {
#pragma unroll
                for (int i = 0; i < PK; i++) {
                    if ((i + 1) * (k + 1) > PK) continue;
                    float sc = (bs[i] > NEG && v[k] > NEG) ? bs[i] + v[k] : NEG;
                    int cc = bc[i] | c[k];
                    if (sc > nv[PK - 1]) {
#pragma unroll
                        for (int j = 0; j < PK; j++) cmpx(nv[j], nc[j], sc, cc);
                    }
                }
            }
#pragma unroll
            for (int i = 0; i < PK; i++) { bs[i] = nv[i]; bc[i] = nc[i]; }
        }
    }
}

/* Persistent fused inference over n patches: cand[p*8 + j] = table entry of the j-th most probable
   cell (-1 past the last valid one), conf[p] = probability of the most probable cell; logits
   (optional) receives the 32 raw logits. */
__global__ void __launch_bounds__(128 * NGROUP, 1)
k_prop_infer(const PropPlan pl, const float *__restrict__ part, const int *__restrict__ to_bin,
             const float *__restrict__ qdesc, int ds, int n, const bf16 *__restrict__ w1, const bf16 *__restrict__ w2,
             const bf16 *__restrict__ w3, const float *__restrict__ params, const int *__restrict__ table, int *cand,
             float *conf, float *logits_out, int *err) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t mbar[NGROUP];
    __shared__ uint32_t tslot;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int g = warp >> 2;                 /* group */
    const int r = tid & 127;                 /* tile row = accumulator lane of this thread */
    float *sbias = reinterpret_cast<float *>(smem + SM_BIAS);
    unsigned char *sX = smem + SM_GROUPS + g * SM_GSIZE + SM_GX;
    unsigned char *sH = smem + SM_GROUPS + g * SM_GSIZE + SM_GH;
    if (warp == 0) ptc::tmem_alloc(&tslot, INFER_COLS);
    if (tid < NGROUP) {
        ptc::mbar_init(&mbar[tid], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    stage_kmajor(smem + SM_W1, w1, PH, PIN);
    stage_kmajor(smem + SM_W2, w2, PH, PH);
    stage_kmajor(smem + SM_W3, w3, POUT, PH);
    for (int i = tid; i < PH; i += blockDim.x) { sbias[i] = params[OFF_B1 + i]; sbias[PH + i] = params[OFF_B2 + i]; }
    for (int i = tid; i < POUT; i += blockDim.x) sbias[2 * PH + i] = params[OFF_B3 + i];
    ptc::fence_proxy_async();
    ptc::tc_fence_before();
    __syncthreads();
    ptc::tc_fence_after();
    /* group g owns columns [128 g, 128 g + 128); warp (4 g + j) reads lanes [32 j, 32 j + 32) */
    const uint32_t tcol = tslot + (uint32_t) (g * 128);
    const uint32_t trow = tcol + ((uint32_t) ((warp & 3) * 32) << 16);
    constexpr uint32_t ID1 = ptc::idesc_bf16_f32(128, PH), ID3 = ptc::idesc_bf16_f32(128, POUT);
    const uint32_t aW1 = ptc::smem_u32(smem + SM_W1), aW2 = ptc::smem_u32(smem + SM_W2),
                   aW3 = ptc::smem_u32(smem + SM_W3), aX = ptc::smem_u32(sX), aH = ptc::smem_u32(sH);
    const bool issuer = r == 0;
    uint64_t *bar = &mbar[g];
    unsigned phase = 0;
    bool ok = true;
    const int ntiles = (n + 127) / 128;
    const int gstride = gridDim.x * NGROUP;
    int tile = blockIdx.x * NGROUP + g;
    float f[PIN];
    int bin[PD];
    tile_features(pl, part, to_bin, qdesc, ds, tile * 128 + r, tile < ntiles ? n : 0, f, bin);
    for (; tile < ntiles; tile += gstride) {
        const int p = tile * 128 + r;
        const bool live = p < n;
        put_x(sX, r, f);
        ptc::fence_proxy_async();
        ptc::tc_fence_before();
        group_sync(g);
        if (issuer) {
            ptc::tc_fence_after();
            ptc::mma_bf16(tcol, ptc::smem_desc(aX), ptc::smem_desc(aW1), ID1, 0);
            ptc::mma_commit(bar);
        }
        /* the next tile's features, while the tensor cores work */
        const int nxt = tile + gstride;
        float fn[PIN];
        int binn[PD];
        tile_features(pl, part, to_bin, qdesc, ds, nxt * 128 + r, nxt < ntiles ? n : 0, fn, binn);
        if (!(ok = group_wait(g, bar, phase))) break;
        epi_hidden(trow, sbias, sH, r);
        ptc::fence_proxy_async();
        ptc::tc_fence_before();
        group_sync(g);
        if (issuer) {
            ptc::tc_fence_after();
#pragma unroll 1
            for (int ks = 0; ks < PH / 16; ks++)
                ptc::mma_bf16(tcol, ptc::smem_desc(aH + ks * 128 * 32), ptc::smem_desc(aW2 + ks * PH * 32), ID1, ks > 0);
            ptc::mma_commit(bar);
        }
        if (!(ok = group_wait(g, bar, phase))) break;
        epi_hidden(trow, sbias + PH, sH, r);
        ptc::fence_proxy_async();
        ptc::tc_fence_before();
        group_sync(g);
        if (issuer) {
            ptc::tc_fence_after();
#pragma unroll 1
            for (int ks = 0; ks < PH / 16; ks++)
                ptc::mma_bf16(tcol, ptc::smem_desc(aH + ks * 128 * 32), ptc::smem_desc(aW3 + ks * POUT * 32), ID3, ks > 0);
            ptc::mma_commit(bar);
        }
        if (!(ok = group_wait(g, bar, phase))) break;
        float z[POUT];
        ptc::tmem_ld16(trow, z);
        ptc::tmem_ld16(trow + 16, z + 16);
        ptc::tc_fence_before();
        if (live) {
#pragma unroll
            for (int c = 0; c < POUT; c++) z[c] += sbias[2 * PH + c];
            if (logits_out) {
                float4 *lo = reinterpret_cast<float4 *>(logits_out + (size_t) p * POUT);
#pragma unroll
                for (int c = 0; c < POUT / 4; c++) lo[c] = make_float4(z[4 * c], z[4 * c + 1], z[4 * c + 2], z[4 * c + 3]);
            }
            float bs[PK];
            int bc[PK];
            top_cells(z, bin, pl, bs, bc);
            int out[PK];
#pragma unroll
            for (int j = 0; j < PK; j++) {
                out[j] = -1;
                if (bs[j] > -3.0e38f) {
                    long long cell = 0;
#pragma unroll
                    for (int d = 0; d < PD; d++)
                        if (d < pl.G) cell += (long long) (bin[d] + ((bc[j] >> (3 * d)) & 7) - 2) * pl.stride[d];
                    out[j] = __ldg(table + cell);
                }
            }
            int4 *co = reinterpret_cast<int4 *>(cand + (size_t) p * PK);
            co[0] = make_int4(out[0], out[1], out[2], out[3]);
            co[1] = make_int4(out[4], out[5], out[6], out[7]);
            conf[p] = __expf(bs[0]);
        }
#pragma unroll
        for (int i = 0; i < PIN; i++) f[i] = fn[i];
#pragma unroll
        for (int d = 0; d < PD; d++) bin[d] = binn[d];
    }
    if (!ok) {
        if (issuer && err) atomicExch(err, 1);
        ptc::mbar_wait(bar, phase);   /* one more bounded wait for the tensor-core work in flight */
    }
    ptc::tc_fence_before();
    __syncthreads();
    if (warp == 0) ptc::tmem_dealloc(tslot, INFER_COLS);
}

PropPlan make_plan(const PtTableView &v) {
    PropPlan pl;
    memset(&pl, 0, sizeof(pl));
    pl.G = v.bins.G;
    for (int d = 0; d < pl.G && d < PD; d++) {
        pl.nslices[d] = v.nslices[d];
        pl.stride[d] = v.bins.stride[d];
        pl.min_val[d] = v.bins.min_val[d];
        pl.range[d] = v.bins.range[d];
        pl.pofs[d] = v.part_ofs[d];
    }
    return pl;
}

}  // namespace

struct pt_proposal {
    DevBuf<float> p, m, v, g;          /* FP32 master parameters, Adam moments, gradient */
    DevBuf<bf16> w1, w2, w2t, w3, w3t; /* BF16 copies for the GEMMs */
    int steps = 0;
    int B = 0;
    DevBuf<bf16> xt, h1, h1t, h2, h2t, dz3, dz3t, dz2, dz2t, dz1, dz1t;
    DevBuf<float> logits, gw1, gw2, gw3t, gb1, gb2, gb3, loss;
    DevBuf<int> err;
    float threshold = 0.5f;
    int kcoh_confident = 0;
    cudaStream_t st = nullptr;
    ~pt_proposal() {
        if (st) cudaStreamDestroy(st);
    }
};

namespace {

pt_status refresh_bf16(pt_proposal *q, cudaStream_t st) {
    k_to_bf16<<<(PH * PH + NT - 1) / NT, NT, 0, st>>>(q->p.p, q->w1.p, q->w2.p, q->w2t.p, q->w3.p, q->w3t.p);
    PT_LAUNCHED();
    return PT_OK;
}

pt_status ensure_batch(pt_proposal *q, int B) {
    if (B <= q->B) return PT_OK;
    PT_CUDA(q->xt.reserve((size_t) B * PIN));
    PT_CUDA(q->h1.reserve((size_t) B * PH));
    PT_CUDA(q->h1t.reserve((size_t) B * PH));
    PT_CUDA(q->h2.reserve((size_t) B * PH));
    PT_CUDA(q->h2t.reserve((size_t) B * PH));
    PT_CUDA(q->dz3.reserve((size_t) B * POUT));
    PT_CUDA(q->dz3t.reserve((size_t) B * POUT));
    PT_CUDA(q->dz2.reserve((size_t) B * PH));
    PT_CUDA(q->dz2t.reserve((size_t) B * PH));
    PT_CUDA(q->dz1.reserve((size_t) B * PH));
    PT_CUDA(q->dz1t.reserve((size_t) B * PH));
    PT_CUDA(q->logits.reserve((size_t) B * POUT));
    q->B = B;
    return PT_OK;
}

GemmEpi epi_of(pt_proposal *q, int mode) {
    GemmEpi e;
    memset(&e, 0, sizeof(e));
    e.mode = mode;
    e.err = q->err.p;
    return e;
}

/* Forward pass of B rows of X; with `train`, transposed activations are kept for the backward. */
pt_status forward(pt_proposal *q, const bf16 *X, int B, bool train, float *logits, cudaStream_t st) {
    GemmEpi e = epi_of(q, GemmEpi::BIAS_RELU);
    e.bias = q->p.p + OFF_B1;
    e.h = q->h1.p;
    e.ldh = PH;
    e.ht = train ? q->h1t.p : nullptr;
    e.ldht = B;
    PT_TRY(pt_gemm_bf16(X, PIN, q->w1.p, PIN, B, PH, PIN, e, st));
    e.bias = q->p.p + OFF_B2;
    e.h = q->h2.p;
    e.ht = train ? q->h2t.p : nullptr;
    PT_TRY(pt_gemm_bf16(q->h1.p, PH, q->w2.p, PH, B, PH, PH, e, st));
    GemmEpi f = epi_of(q, GemmEpi::BIAS_F32);
    f.bias = q->p.p + OFF_B3;
    f.c = logits;
    f.ldc = POUT;
    PT_TRY(pt_gemm_bf16(q->h2.p, PH, q->w3.p, PH, B, POUT, PH, f, st));
    return PT_OK;
}

/* Loss and parameter gradient of a batch (into q->g and q->loss), without updating. */
pt_status gradient(pt_proposal *q, const bf16 *X, const unsigned char *labels, int B, cudaStream_t st) {
    PT_TRY(ensure_batch(q, B));
    k_transpose_x<<<(B + NT - 1) / NT, NT, 0, st>>>(X, B, q->xt.p);
    PT_LAUNCHED();
    PT_TRY(forward(q, X, B, true, q->logits.p, st));
    PT_CUDA(cudaMemsetAsync(q->loss.p, 0, sizeof(float), st));
    k_ce<<<(B + NT - 1) / NT, NT, 0, st>>>(q->logits.p, labels, B, q->dz3.p, q->dz3t.p, q->loss.p);
    PT_LAUNCHED();
    /* dW3^T [PH x POUT] = H2^T dZ3 */
    GemmEpi e = epi_of(q, GemmEpi::STORE_F32);
    e.c = q->gw3t.p;
    e.ldc = POUT;
    PT_TRY(pt_gemm_bf16(q->h2t.p, B, q->dz3t.p, B, PH, POUT, B, e, st));
    /* dZ2 = (dZ3 W3) * [H2 > 0] */
    GemmEpi r = epi_of(q, GemmEpi::RELU_GRAD);
    r.mask = q->h2.p;
    r.ldm = PH;
    r.h = q->dz2.p;
    r.ldh = PH;
    r.ht = q->dz2t.p;
    r.ldht = B;
    PT_TRY(pt_gemm_bf16(q->dz3.p, POUT, q->w3t.p, POUT, B, PH, POUT, r, st));
    /* dW2 [PH x PH] = dZ2^T H1 */
    e.c = q->gw2.p;
    e.ldc = PH;
    PT_TRY(pt_gemm_bf16(q->dz2t.p, B, q->h1t.p, B, PH, PH, B, e, st));
    /* dZ1 = (dZ2 W2) * [H1 > 0] */
    r.mask = q->h1.p;
    r.h = q->dz1.p;
    r.ht = q->dz1t.p;
    PT_TRY(pt_gemm_bf16(q->dz2.p, PH, q->w2t.p, PH, B, PH, PH, r, st));
    /* dW1 [PH x PIN] = dZ1^T X */
    e.c = q->gw1.p;
    e.ldc = PIN;
    PT_TRY(pt_gemm_bf16(q->dz1t.p, B, q->xt.p, B, PH, PIN, B, e, st));
    k_rowsum<<<PH, NT, 0, st>>>(q->dz1t.p, B, q->gb1.p);
    PT_LAUNCHED();
    k_rowsum<<<PH, NT, 0, st>>>(q->dz2t.p, B, q->gb2.p);
    PT_LAUNCHED();
    k_rowsum<<<POUT, NT, 0, st>>>(q->dz3t.p, B, q->gb3.p);
    PT_LAUNCHED();
    k_pack_grad<<<(PH * PH + NT - 1) / NT, NT, 0, st>>>(q->gw1.p, q->gb1.p, q->gw2.p, q->gb2.p, q->gw3t.p, q->gb3.p, q->g.p);
    PT_LAUNCHED();
    return PT_OK;
}

pt_status check_err(pt_proposal *q, cudaStream_t st) {
    int e = 0;
    PT_CUDA(cudaMemcpyAsync(&e, q->err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    PT_CUDA(cudaStreamSynchronize(st));
    if (e) return pt_fail(PT_TIMEOUT, "a tensor-core wait of the proposal network gave up");
    return PT_OK;
}

pt_status check_batch(const pt_proposal *q, const void *X, const void *labels, int B) {
    if (!q || !X || !labels) return pt_fail(PT_BAD_ARG, "null argument");
    if (B < 64 || B % 64) return pt_fail(PT_BAD_ARG, "proposal batch %d: must be a positive multiple of 64", B);
    return PT_OK;
}

}  // namespace

/* ---- entry points used by pt_table.cu ---- */

pt_status pt_prop_check_table(const PtTableView &v) {
    if (v.bins.G < 1 || v.bins.G > PD)
        return pt_fail(PT_UNSUPPORTED, "the proposal network handles tables of 1..%d grid dimensions (this one has %d)",
                       PD, v.bins.G);
    if (!v.part) return pt_fail(PT_BAD_ARG, "table has no partition on the device");
    return PT_OK;
}

pt_status pt_launch_prop_samples(const PtTableView &v, const float *qdesc, int n, const double *ann, void *X,
                                 unsigned char *labels, cudaStream_t st) {
    PT_TRY(pt_prop_check_table(v));
    if (n <= 0) return PT_OK;
    k_prop_samples<<<(n + NT - 1) / NT, NT, 0, st>>>(make_plan(v), v.part, v.to_bin, qdesc, v.ds, n, v.b_desc, v.w - 7,
                                                     v.h - 7, ann, (bf16 *) X, labels);
    PT_LAUNCHED();
    return PT_OK;
}

pt_status pt_launch_prop_infer(const PtTableView &v, pt_proposal *q, const float *qdesc, int n, int *cand, float *conf,
                               float *logits, cudaStream_t st) {
    PT_TRY(pt_prop_check_table(v));
    if (!q) return pt_fail(PT_BAD_ARG, "null proposal network");
    if (n <= 0) return PT_OK;
    static int nsm = 0;
    if (!nsm) {
        int dev = 0;
        PT_CUDA(cudaGetDevice(&dev));
        PT_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    }
    PT_CUDA(cudaFuncSetAttribute(k_prop_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, SM_TOTAL));
    const int ntiles = (n + 127) / 128;
    /* one CTA per SM: its shared memory (SM_TOTAL) leaves no room for a second, so its allocation
       of all 512 tensor-memory columns never waits on another CTA of this kernel */
    const int groups = (ntiles + NGROUP - 1) / NGROUP;
    const int grid = groups < nsm ? groups : nsm;
    k_prop_infer<<<grid, 128 * NGROUP, SM_TOTAL, st>>>(make_plan(v), v.part, v.to_bin, qdesc, v.ds, n, q->w1.p, q->w2.p, q->w3.p,
                                              q->p.p, v.table, cand, conf, logits, q->err.p);
    PT_LAUNCHED();
    return PT_OK;
}

float pt_prop_threshold(const pt_proposal *q) { return q->threshold; }
int pt_prop_kcoh_confident(const pt_proposal *q) { return q->kcoh_confident; }
pt_status pt_prop_check_error(pt_proposal *q, cudaStream_t st) { return check_err(q, st); }

extern "C" {

pt_status pt_proposal_create(uint32_t seed, pt_proposal **out) {
    if (!out) return pt_fail(PT_BAD_ARG, "null output");
    *out = nullptr;
    pt_proposal *q = new pt_proposal();
    auto fail = [&](pt_status s) { delete q; return s; };
    if (cudaStreamCreateWithFlags(&q->st, cudaStreamNonBlocking) != cudaSuccess)
        return fail(pt_fail(PT_CUDA_ERR, "proposal network stream"));
    std::vector<float> h(NPARAM, 0.f);
    std::mt19937 rng(seed);
    auto init = [&](int off, int fan_out, int fan_in) {   /* He initialisation */
        std::normal_distribution<float> nd(0.f, std::sqrt(2.f / (float) fan_in));
        for (int i = 0; i < fan_out * fan_in; i++) h[off + i] = nd(rng);
    };
    init(OFF_W1, PH, 2 * PD);
    for (int o = 0; o < PH; o++)                   /* the 4 padding inputs are always zero */
        for (int k = 2 * PD; k < PIN; k++) h[OFF_W1 + o * PIN + k] = 0.f;
    init(OFF_W2, PH, PH);
    init(OFF_W3, POUT, PH);
    for (int i = 0; i < POUT * PH; i++) h[OFF_W3 + i] *= 0.1f;
    if (q->p.reserve(NPARAM) || q->m.reserve(NPARAM) || q->v.reserve(NPARAM) || q->g.reserve(NPARAM) ||
        q->w1.reserve(PH * PIN) || q->w2.reserve(PH * PH) || q->w2t.reserve(PH * PH) || q->w3.reserve(POUT * PH) ||
        q->w3t.reserve(POUT * PH) || q->gw1.reserve(PH * PIN) || q->gw2.reserve(PH * PH) || q->gw3t.reserve(PH * POUT) ||
        q->gb1.reserve(PH) || q->gb2.reserve(PH) || q->gb3.reserve(POUT) || q->loss.reserve(1) || q->err.reserve(1))
        return fail(pt_fail(PT_OOM, "proposal network buffers"));
    if (cudaMemcpyAsync(q->p.p, h.data(), sizeof(float) * NPARAM, cudaMemcpyHostToDevice, q->st) ||
        cudaMemsetAsync(q->m.p, 0, sizeof(float) * NPARAM, q->st) || cudaMemsetAsync(q->v.p, 0, sizeof(float) * NPARAM, q->st) ||
        cudaMemsetAsync(q->g.p, 0, sizeof(float) * NPARAM, q->st) || cudaMemsetAsync(q->err.p, 0, sizeof(int), q->st))
        return fail(pt_fail(PT_CUDA_ERR, "proposal network initialisation"));
    pt_status s = refresh_bf16(q, q->st);
    if (s != PT_OK) return fail(s);
    if (cudaStreamSynchronize(q->st) != cudaSuccess) return fail(pt_fail(PT_CUDA_ERR, "proposal network initialisation"));
    *out = q;
    return PT_OK;
}

void pt_proposal_free(pt_proposal *q) { delete q; }

int pt_proposal_num_params(void) { return NPARAM; }

pt_status pt_proposal_get_params(pt_proposal *q, float *host) {
    if (!q || !host) return pt_fail(PT_BAD_ARG, "null argument");
    PT_CUDA(cudaMemcpyAsync(host, q->p.p, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost, q->st));
    PT_CUDA(cudaStreamSynchronize(q->st));
    return PT_OK;
}

pt_status pt_proposal_set_params(pt_proposal *q, const float *host) {
    if (!q || !host) return pt_fail(PT_BAD_ARG, "null argument");
    PT_CUDA(cudaMemcpyAsync(q->p.p, host, sizeof(float) * NPARAM, cudaMemcpyHostToDevice, q->st));
    PT_CUDA(cudaMemsetAsync(q->m.p, 0, sizeof(float) * NPARAM, q->st));
    PT_CUDA(cudaMemsetAsync(q->v.p, 0, sizeof(float) * NPARAM, q->st));
    q->steps = 0;
    PT_TRY(refresh_bf16(q, q->st));
    PT_CUDA(cudaStreamSynchronize(q->st));
    return PT_OK;
}

pt_status pt_proposal_configure(pt_proposal *q, float threshold, int kcoh_confident) {
    if (!q) return pt_fail(PT_BAD_ARG, "null argument");
    if (!(threshold >= 0.f && threshold <= 1.f)) return pt_fail(PT_BAD_ARG, "threshold %g outside [0, 1]", threshold);
    q->threshold = threshold;
    q->kcoh_confident = kcoh_confident ? 1 : 0;
    return PT_OK;
}

pt_status pt_proposal_gradient(pt_proposal *q, const void *X, const uint8_t *labels, int B, float *loss,
                               float *grad_host, void *stream) {
    PT_TRY(check_batch(q, X, labels, B));
    cudaStream_t st = (cudaStream_t) stream;
    PT_TRY(gradient(q, (const bf16 *) X, labels, B, st));
    if (loss) PT_CUDA(cudaMemcpyAsync(loss, q->loss.p, sizeof(float), cudaMemcpyDeviceToHost, st));
    if (grad_host) PT_CUDA(cudaMemcpyAsync(grad_host, q->g.p, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost, st));
    PT_TRY(check_err(q, st));
    if (loss) *loss /= (float) B;
    return PT_OK;
}

pt_status pt_proposal_train_step(pt_proposal *q, const void *X, const uint8_t *labels, int B, float lr, float wd,
                                 float *loss, void *stream) {
    PT_TRY(check_batch(q, X, labels, B));
    cudaStream_t st = (cudaStream_t) stream;
    PT_TRY(gradient(q, (const bf16 *) X, labels, B, st));
    q->steps++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float) q->steps), c2 = 1.f - std::pow(b2, (float) q->steps);
    k_adam<<<(NPARAM + NT - 1) / NT, NT, 0, st>>>(q->p.p, q->g.p, q->m.p, q->v.p, NPARAM, lr, b1, b2, 1e-8f, wd, c1, c2);
    PT_LAUNCHED();
    PT_TRY(refresh_bf16(q, st));
    if (loss) {
        PT_CUDA(cudaMemcpyAsync(loss, q->loss.p, sizeof(float), cudaMemcpyDeviceToHost, st));
        PT_TRY(check_err(q, st));
        *loss /= (float) B;
    }
    return PT_OK;
}

pt_status pt_proposal_sync(pt_proposal *q, void *stream) {
    if (!q) return pt_fail(PT_BAD_ARG, "null argument");
    return check_err(q, (cudaStream_t) stream);
}

pt_status pt_proposal_forward(pt_proposal *q, const void *X, int B, float *logits, void *stream) {
    if (!q || !X || !logits) return pt_fail(PT_BAD_ARG, "null argument");
    if (B < 1) return pt_fail(PT_BAD_ARG, "batch %d", B);
    cudaStream_t st = (cudaStream_t) stream;
    PT_TRY(ensure_batch(q, B));
    PT_TRY(forward(q, (const bf16 *) X, B, false, logits, st));
    return check_err(q, st);
}

}  // extern "C"
