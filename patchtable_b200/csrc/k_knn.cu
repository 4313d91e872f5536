/* Exact k-nearest-neighbour search in descriptor space for the k-coherence step.

   Ranking (shared with the CPU oracle): squared L2 in float, dimensions summed in index order,
   each product and sum rounded (no fused operations); ties by the smaller point index.

   Structure: train points are sorted by a Morton code of their quantised descriptor, cut into
   buckets of 32 consecutive points, and a complete binary tree of axis-aligned bounding boxes is
   built over the buckets (implicit heap layout, one launch per level).  Each query
   descends the tree depth first, nearer child first, and skips a subtree only when the box's
   lower bound exceeds the current k-th distance by more than the float rounding of a distance
   could account for -- so the result equals an exhaustive search.  Queries are processed in
   Morton order and each warp walks the tree together (k_knn_warp). */
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include "pt_internal.h"
#include "pt_kernels.h"

namespace {

constexpr int NT = 128;
constexpr int BUCKET = 32;

__global__ void k_range(const float *__restrict__ pts, int N, int nd, float *mn, float *mx) {
    __shared__ float smin[PT_DESC_MAX][NT], smax[PT_DESC_MAX][NT];
    float a[PT_DESC_MAX], b[PT_DESC_MAX];
    for (int d = 0; d < nd; d++) { a[d] = __int_as_float(0x7f800000); b[d] = -__int_as_float(0x7f800000); }
    for (int i = blockIdx.x * NT + threadIdx.x; i < N; i += gridDim.x * NT)
        for (int d = 0; d < nd; d++) { float v = pts[(size_t) i * nd + d]; a[d] = fminf(a[d], v); b[d] = fmaxf(b[d], v); }
    for (int d = 0; d < nd; d++) { smin[d][threadIdx.x] = a[d]; smax[d][threadIdx.x] = b[d]; }
    __syncthreads();
    if (threadIdx.x < nd) {
        int d = threadIdx.x;
        float u = smin[d][0], v = smax[d][0];
        for (int i = 1; i < NT; i++) { u = fminf(u, smin[d][i]); v = fmaxf(v, smax[d][i]); }
        mn[blockIdx.x * PT_DESC_MAX + d] = u;
        mx[blockIdx.x * PT_DESC_MAX + d] = v;
    }
}

struct Quant {
    int nd, bits;
    float mn[PT_DESC_MAX], scale[PT_DESC_MAX];
};

__global__ void k_morton(const Quant qz, const float *__restrict__ pts, int N, unsigned long long *codes, int *idx) {
    int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= N) return;
    unsigned q[PT_DESC_MAX];
    const unsigned top = (1u << qz.bits) - 1;
    for (int d = 0; d < qz.nd; d++) {
        float t = (pts[(size_t) i * qz.nd + d] - qz.mn[d]) * qz.scale[d];
        t = fminf(fmaxf(t, 0.f), (float) top);
        q[d] = (unsigned) t;
    }
    unsigned long long c = 0;
    for (int b = qz.bits - 1; b >= 0; b--)
        for (int d = 0; d < qz.nd; d++) c = (c << 1) | ((q[d] >> b) & 1u);
    codes[i] = c;
    idx[i] = i;
}

__global__ void k_reorder(const float *__restrict__ pts, int N, int nd, const int *__restrict__ perm, float *sp) {
    long long t = blockIdx.x * 256ll + threadIdx.x;
    if (t >= (long long) N * nd) return;
    int i = (int) (t / nd), d = (int) (t % nd);
    sp[t] = pts[(size_t) perm[i] * nd + d];
}

/* Leaf boxes (heap nodes L .. 2L-1); empty leaves get an inverted box. */
__global__ void k_leaf_box(const float *__restrict__ sp, int N, int nd, int L, float *lo, float *hi) {
    int j = blockIdx.x * 256 + threadIdx.x;
    if (j >= L) return;
    int node = L + j;
    for (int d = 0; d < nd; d++) {
        float a = __int_as_float(0x7f800000), b = -__int_as_float(0x7f800000);
        for (int i = j * BUCKET; i < min(N, (j + 1) * BUCKET); i++) { float v = sp[(size_t) i * nd + d]; a = fminf(a, v); b = fmaxf(b, v); }
        lo[(size_t) node * nd + d] = a;
        hi[(size_t) node * nd + d] = b;
    }
}

__global__ void k_inner_box(int first, int count, int nd, float *lo, float *hi) {
    int j = blockIdx.x * 256 + threadIdx.x;
    if (j >= count) return;
    int node = first + j;
    for (int d = 0; d < nd; d++) {
        lo[(size_t) node * nd + d] = fminf(lo[(size_t) (2 * node) * nd + d], lo[(size_t) (2 * node + 1) * nd + d]);
        hi[(size_t) node * nd + d] = fmaxf(hi[(size_t) (2 * node) * nd + d], hi[(size_t) (2 * node + 1) * nd + d]);
    }
}

/* Squared distance from q to a box, rounded down enough to be a lower bound of the squared distance. */
__device__ __forceinline__ float box_lb(const float (&q)[PT_DESC_MAX], const float *lo, const float *hi, int nd) {
    float s = 0.f;
#pragma unroll
    for (int d = 0; d < PT_DESC_MAX; d++) {          /* unrolled: q stays in registers */
        if (d < nd) {
            float e = fmaxf(fmaxf(lo[d] - q[d], q[d] - hi[d]), 0.f);
            s += e * e;
        }
    }
    return s * (1.0f - 1e-5f);
}

__device__ __forceinline__ bool before(float d, int i, float d2, int i2) { return d < d2 || (d == d2 && i < i2); }

/* The search, with the 32 queries of a warp walking the tree together: a node is opened
   when any lane's lower bound admits it, the traversal stack is shared by the warp, and a
   leaf's points are staged once in shared memory and read back by every lane as broadcasts.
   The lanes' paths through the tree are nearly the same (queries in Morton order), so the warp
   does the union of its lanes' work without divergence.  Lanes score only leaves their own bound
   admits, with the same rounding and tie rule, so the result equals the per-thread search. */
constexpr int KNN_STACK = 64;
constexpr int PSTRIDE = PT_DESC_MAX + 1;            /* staged point stride (odd: no bank conflicts) */

template<int K, int NV>
__global__ void __launch_bounds__(NT)
k_knn_warp(const float *__restrict__ sp, const int *__restrict__ sidx, int N, int nd, int L,
           const float *__restrict__ lo, const float *__restrict__ hi, const float *__restrict__ qdesc,
           const int *__restrict__ qorder, int Q, int *out) {
    __shared__ int stk_s[NT / 32][KNN_STACK];
    __shared__ float4 pts_s[NT / 32][BUCKET * NV];       /* a leaf's points, NV float4 each (zero-padded) */
    __shared__ int pid_s[NT / 32][BUCKET];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int t = blockIdx.x * NT + threadIdx.x;
    const bool active = t < Q;
    const int q = active ? qorder[t] : 0;
    float qv[PT_DESC_MAX];
#pragma unroll
    for (int d = 0; d < PT_DESC_MAX; d++) qv[d] = (active && d < nd) ? qdesc[(size_t) q * nd + d] : 0.f;
    float kd[K];
    int ki[K];
#pragma unroll
    for (int j = 0; j < K; j++) { kd[j] = __int_as_float(0x7f800000); ki[j] = 0x7fffffff; }
    int *stk = stk_s[wid];
    float4 *pts = pts_s[wid];
    int *pid = pid_s[wid];
    if (lane == 0) stk[0] = 1;
    __syncwarp();
    int top = 1;
    while (top > 0) {
        const int node = stk[--top];
        __syncwarp();
        const float lb = active ? box_lb(qv, lo + (size_t) node * nd, hi + (size_t) node * nd, nd) : 0.f;
        const bool want = active && !(lb > kd[K - 1]);
        if (!__any_sync(FULL, want)) continue;
        if (node >= L) {
            const int base = (node - L) * BUCKET;
            const int cnt = min(BUCKET, N - base);
            if (lane < cnt) {
                const float *src = sp + (size_t) (base + lane) * nd;
                float v[4 * NV];
#pragma unroll
                for (int d = 0; d < 4 * NV; d++) v[d] = d < nd ? src[d] : 0.f;
#pragma unroll
                for (int u = 0; u < NV; u++) pts[lane * NV + u] = make_float4(v[4 * u], v[4 * u + 1], v[4 * u + 2], v[4 * u + 3]);
                pid[lane] = sidx[base + lane];
            }
            __syncwarp();
            if (want) {
                for (int m = 0; m < cnt; m++) {
                    /* every lane reads the same point: 16-byte broadcasts; the partial sum after
                       the first four dimensions already rejects most points (it only grows) */
                    float dsum = 0.f;
#pragma unroll
                    for (int u = 0; u < NV; u++) {
                        const float4 pv = pts[m * NV + u];
                        const float pc[4] = {pv.x, pv.y, pv.z, pv.w};
#pragma unroll
                        for (int c = 0; c < 4; c++) {
                            if (4 * u + c < nd) {
                                const float e = __fsub_rn(qv[4 * u + c], pc[c]);
                                dsum = __fadd_rn(dsum, __fmul_rn(e, e));
                            }
                        }
                        if (u == 0 && dsum > kd[K - 1]) break;
                    }
                    if (dsum > kd[K - 1]) continue;
                    const int id = pid[m];
                    if (!before(dsum, id, kd[K - 1], ki[K - 1])) continue;
#pragma unroll
                    for (int s2 = K - 1; s2 >= 0; s2--) {
                        if (before(dsum, id, kd[s2], ki[s2])) {
                            if (s2 > 0 && before(dsum, id, kd[s2 - 1], ki[s2 - 1])) { kd[s2] = kd[s2 - 1]; ki[s2] = ki[s2 - 1]; }
                            else { kd[s2] = dsum; ki[s2] = id; }
                        }
                    }
                }
            }
            __syncwarp();                        /* the next leaf restages the points */
            continue;
        }
        const int c0 = 2 * node, c1 = 2 * node + 1;
        float l0 = 0.f, l1 = 0.f;
        if (want) {
            l0 = box_lb(qv, lo + (size_t) c0 * nd, hi + (size_t) c0 * nd, nd);
            l1 = box_lb(qv, lo + (size_t) c1 * nd, hi + (size_t) c1 * nd, nd);
        }
        float s0 = l0, s1 = l1;                   /* nearer child (for the warp) first */
#pragma unroll
        for (int o = 16; o; o >>= 1) { s0 += __shfl_xor_sync(FULL, s0, o); s1 += __shfl_xor_sync(FULL, s1, o); }
        if (top + 2 > KNN_STACK) continue;        /* cannot happen: depth <= 31 */
        if (lane == 0) {
            if (s0 <= s1) { stk[top] = c1; stk[top + 1] = c0; }
            else { stk[top] = c0; stk[top + 1] = c1; }
        }
        __syncwarp();
        top += 2;
    }
    if (active)
        for (int j = 0; j < K; j++) out[(size_t) q * K + j] = ki[j] == 0x7fffffff ? -1 : ki[j];
}

/* The same search for K = 128 .. 1024 (sets that need that many neighbours: thin images, or
   narrow flat regions where the nearest descriptors all lie within kcoherence_min_dist).  The
   sorted list lives in global memory (wd: distances, out: indices, K per query); a leaf's
   admissible points are first sorted in a 32-entry buffer and then merged into the list from the
   back in one pass, keeping the K smallest.  Traversal, rounding and tie rule are those of
   k_knn_warp, so its first 64 entries equal that kernel's result. */
__global__ void __launch_bounds__(NT)
k_knn_wide(const float *__restrict__ sp, const int *__restrict__ sidx, int N, int nd, int L,
           const float *__restrict__ lo, const float *__restrict__ hi, const float *__restrict__ qdesc,
           const int *__restrict__ qorder, int Q, int K, float *wd, int *out) {
    __shared__ int stk_s[NT / 32][KNN_STACK];
    __shared__ float pts_s[NT / 32][BUCKET * PSTRIDE];
    __shared__ int pid_s[NT / 32][BUCKET];
    const unsigned FULL = 0xffffffffu;
    const float INF = __int_as_float(0x7f800000);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int t = blockIdx.x * NT + threadIdx.x;
    const bool active = t < Q;
    const int q = active ? qorder[t] : 0;
    float qv[PT_DESC_MAX];
#pragma unroll
    for (int d = 0; d < PT_DESC_MAX; d++) qv[d] = (active && d < nd) ? qdesc[(size_t) q * nd + d] : 0.f;
    float *ld = wd + (size_t) q * K;
    int *li = out + (size_t) q * K;
    if (active)
        for (int j = 0; j < K; j++) { ld[j] = INF; li[j] = 0x7fffffff; }
    float worst_d = INF;
    int worst_i = 0x7fffffff;
    int *stk = stk_s[wid];
    float *pts = pts_s[wid];
    int *pid = pid_s[wid];
    if (lane == 0) stk[0] = 1;
    __syncwarp();
    int top = 1;
    while (top > 0) {
        const int node = stk[--top];
        __syncwarp();
        const float lb = active ? box_lb(qv, lo + (size_t) node * nd, hi + (size_t) node * nd, nd) : 0.f;
        const bool want = active && !(lb > worst_d);
        if (!__any_sync(FULL, want)) continue;
        if (node >= L) {
            const int base = (node - L) * BUCKET;
            const int cnt = min(BUCKET, N - base);
            if (lane < cnt) {
                const float *src = sp + (size_t) (base + lane) * nd;
                for (int d = 0; d < nd; d++) pts[lane * PSTRIDE + d] = src[d];
                pid[lane] = sidx[base + lane];
            }
            __syncwarp();
            if (want) {
                float bd[BUCKET];
                int bi[BUCKET];
                int nb = 0;
                for (int m = 0; m < cnt; m++) {
                    const float *pv = pts + m * PSTRIDE;
                    float dsum = 0.f;
#pragma unroll
                    for (int d = 0; d < PT_DESC_MAX; d++) {
                        if (d < nd) {
                            const float e = __fsub_rn(qv[d], pv[d]);
                            dsum = __fadd_rn(dsum, __fmul_rn(e, e));
                        }
                    }
                    const int id = pid[m];
                    if (!before(dsum, id, worst_d, worst_i)) continue;
                    int s2 = nb++;
                    while (s2 > 0 && before(dsum, id, bd[s2 - 1], bi[s2 - 1])) { bd[s2] = bd[s2 - 1]; bi[s2] = bi[s2 - 1]; s2--; }
                    bd[s2] = dsum;
                    bi[s2] = id;
                }
                if (nb > 0) {
                    /* backward merge: the union's largest go to virtual slots K .. K+nb-1 and drop out */
                    int ia = K - 1, ib = nb - 1;
                    for (int p = K + nb - 1; ib >= 0; p--) {
                        if (ia < 0 || before(ld[ia], li[ia], bd[ib], bi[ib])) {
                            if (p < K) { ld[p] = bd[ib]; li[p] = bi[ib]; }
                            ib--;
                        } else {
                            if (p < K) { ld[p] = ld[ia]; li[p] = li[ia]; }
                            ia--;
                        }
                    }
                    worst_d = ld[K - 1];
                    worst_i = li[K - 1];
                }
            }
            __syncwarp();                        /* the next leaf restages the points */
            continue;
        }
        const int c0 = 2 * node, c1 = 2 * node + 1;
        float l0 = 0.f, l1 = 0.f;
        if (want) {
            l0 = box_lb(qv, lo + (size_t) c0 * nd, hi + (size_t) c0 * nd, nd);
            l1 = box_lb(qv, lo + (size_t) c1 * nd, hi + (size_t) c1 * nd, nd);
        }
        float s0 = l0, s1 = l1;
#pragma unroll
        for (int o = 16; o; o >>= 1) { s0 += __shfl_xor_sync(FULL, s0, o); s1 += __shfl_xor_sync(FULL, s1, o); }
        if (top + 2 > KNN_STACK) continue;        /* cannot happen: depth <= 31 */
        if (lane == 0) {
            if (s0 <= s1) { stk[top] = c1; stk[top + 1] = c0; }
            else { stk[top] = c0; stk[top + 1] = c1; }
        }
        __syncwarp();
        top += 2;
    }
    if (active)
        for (int j = 0; j < K; j++)
            if (li[j] == 0x7fffffff) li[j] = -1;
}

}  // namespace

/* Exact top-K (K in {12, 16, 24, 32, 48, 64}, or a power of two up to PT_KNN_WIDE_MAX) train
   indices of every query, ascending (dist, index). */
pt_status pt_launch_knn(const float *train, int N, int nd, const float *qdesc, int Q, int K, int *out, cudaStream_t st) {
    if (N < 1 || Q < 1) return PT_OK;
    if (nd < 1 || nd > PT_DESC_MAX) return pt_fail(PT_UNSUPPORTED, "knn: %d dims", nd);
    /* range of the train points */
    const int NB = 148;
    DevBuf<float> pmn, pmx;
    PT_CUDA(pmn.reserve(NB * PT_DESC_MAX));
    PT_CUDA(pmx.reserve(NB * PT_DESC_MAX));
    k_range<<<NB, NT, 0, st>>>(train, N, nd, pmn.p, pmx.p);
    PT_LAUNCHED();
    std::vector<float> a(NB * PT_DESC_MAX), b(NB * PT_DESC_MAX);
    PT_CUDA(cudaMemcpyAsync(a.data(), pmn.p, sizeof(float) * a.size(), cudaMemcpyDeviceToHost, st));
    PT_CUDA(cudaMemcpyAsync(b.data(), pmx.p, sizeof(float) * b.size(), cudaMemcpyDeviceToHost, st));
    PT_CUDA(cudaStreamSynchronize(st));
    Quant qz;
    memset(&qz, 0, sizeof(qz));
    qz.nd = nd;
    qz.bits = std::min(10, 63 / nd);
    /* One scale for every dimension (that of the widest range): the Morton order then splits the
       dimensions in proportion to their spread, so a bucket's box is about as wide in every
       dimension in distance units, which is what the Euclidean lower bounds prune with.  (The
       search is exact whatever the order; only its pruning depends on the boxes.) */
    float rmax = 0.f;
    for (int d = 0; d < nd; d++) {
        float mn = a[d], mx = b[d];
        for (int i = 1; i < NB; i++) { mn = std::min(mn, a[i * PT_DESC_MAX + d]); mx = std::max(mx, b[i * PT_DESC_MAX + d]); }
        qz.mn[d] = mn;
        rmax = std::max(rmax, mx - mn);
    }
    for (int d = 0; d < nd; d++) qz.scale[d] = rmax > 0.f ? (float) ((1u << qz.bits) - 1) / rmax : 0.f;
    /* sort train points and queries by Morton code */
    DevBuf<unsigned long long> codes, codes2;
    DevBuf<int> idx, perm, qidx, qorder, sidx;
    DevBuf<float> sp;
    PT_CUDA(codes.reserve(std::max(N, Q)));
    PT_CUDA(codes2.reserve(std::max(N, Q)));
    PT_CUDA(idx.reserve(std::max(N, Q)));
    PT_CUDA(perm.reserve(N));
    PT_CUDA(qorder.reserve(Q));
    PT_CUDA(sp.reserve((size_t) N * nd));
    size_t tb = 0;
    PT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, codes.p, codes2.p, idx.p, perm.p, std::max(N, Q), 0, 64, st));
    DevBuf<unsigned char> tmp;
    PT_CUDA(tmp.reserve(tb));
    k_morton<<<(N + 255) / 256, 256, 0, st>>>(qz, train, N, codes.p, idx.p);
    PT_LAUNCHED();
    PT_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, codes.p, codes2.p, idx.p, perm.p, N, 0, 64, st));
    pt_count_launches(4);
    k_morton<<<(Q + 255) / 256, 256, 0, st>>>(qz, qdesc, Q, codes.p, idx.p);
    PT_LAUNCHED();
    PT_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, codes.p, codes2.p, idx.p, qorder.p, Q, 0, 64, st));
    pt_count_launches(4);
    k_reorder<<<(unsigned) (((long long) N * nd + 255) / 256), 256, 0, st>>>(train, N, nd, perm.p, sp.p);
    PT_LAUNCHED();
    /* bucket boxes and the tree above them */
    int nbk = (N + BUCKET - 1) / BUCKET;
    int L = 1;
    while (L < nbk) L <<= 1;
    DevBuf<float> lo, hi;
    PT_CUDA(lo.reserve((size_t) 2 * L * nd));
    PT_CUDA(hi.reserve((size_t) 2 * L * nd));
    k_leaf_box<<<(L + 255) / 256, 256, 0, st>>>(sp.p, N, nd, L, lo.p, hi.p);
    PT_LAUNCHED();
    for (int first = L / 2; first >= 1; first /= 2) {
        k_inner_box<<<(first + 255) / 256, 256, 0, st>>>(first, first, nd, lo.p, hi.p);
        PT_LAUNCHED();
    }
    dim3 grid((Q + NT - 1) / NT);
    if (K > 64) {
        if (K > PT_KNN_WIDE_MAX || (K & (K - 1))) return pt_fail(PT_UNSUPPORTED, "knn K=%d", K);
        DevBuf<float> wd;
        PT_CUDA(wd.reserve((size_t) Q * K));
        k_knn_wide<<<grid, NT, 0, st>>>(sp.p, perm.p, N, nd, L, lo.p, hi.p, qdesc, qorder.p, Q, K, wd.p, out);
        PT_LAUNCHED();
        PT_CUDA(cudaStreamSynchronize(st));
        return PT_OK;
    }
#define PT_KNN_K(KK) case KK: if (nd <= 8) k_knn_warp<KK, 2><<<grid, NT, 0, st>>>(sp.p, perm.p, N, nd, L, lo.p, hi.p, qdesc, qorder.p, Q, out); \
        else k_knn_warp<KK, 4><<<grid, NT, 0, st>>>(sp.p, perm.p, N, nd, L, lo.p, hi.p, qdesc, qorder.p, Q, out); break;
    switch (K) {
        PT_KNN_K(12) PT_KNN_K(16) PT_KNN_K(24) PT_KNN_K(32) PT_KNN_K(48) PT_KNN_K(64)
        default: return pt_fail(PT_UNSUPPORTED, "knn K=%d", K);
    }
#undef PT_KNN_K
    PT_LAUNCHED();
    PT_CUDA(cudaStreamSynchronize(st));
    return PT_OK;
}
