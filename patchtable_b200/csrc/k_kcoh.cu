/* k-coherence set of the table image (patchtable/patchtable.h:2653-2869, FLANN path with
   TABLE_KCOHERENCE_TRIANGLE).

   For every query patch of b the reference asks for its knn nearest patches in descriptor space,
   marks a neighbour valid when it lies at least kcoherence_min_dist pixels away, doubles knn until
   `kcoherence` valid neighbours exist, re-sorts the knn matches by exact 8x8x3 distance and keeps
   the first `kcoherence` valid ones.  Two details of that loop carry state from patch to patch:
     * knn starts from the previous patch's final knn unless x is a multiple of flann_reset_step
       (patchtable.h:2714), so knn is a running maximum over segments of the raster order;
     * the validity loop stops at the kcoherence-th valid match, so the flags past that point keep
       the values the previous patch left in the vector (after its exact-distance sort), and those
       stale flags take part in the final selection (patchtable.h:2793-2856).
   The kernels below reproduce both: one thread walks each segment in order, carrying the flag
   vector; the only state that crosses a segment boundary is one flag bit, which is resolved by a
   scan over segments after each segment has been evaluated for both values of that bit.

   The nearest-neighbour search (k_knn.cu) is exact, ranked by (float squared L2 summed in
   dimension order without fused operations, point index); FLANN's approximate tree is not
   reproduced.  Lists of up to 64 neighbours keep their validity flags in one 64-bit word; longer
   ones (up to PT_KNN_WIDE_MAX, reached when most of a patch's nearest descriptors lie within
   kcoherence_min_dist, e.g. inside a flat region) use the *_wide kernels with multi-word flags. */
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <vector>

#include "pt_internal.h"
#include "pt_descdist.cuh"
#include "pt_kernels.h"

namespace {

/* Copies descriptor rows (ds-strided records) of the listed patches into a compact n x nd array. */
__global__ void k_gather_rows(const float *__restrict__ desc, int ds, int nd, const int *__restrict__ rows, int n,
                              float *out) {
    long long t = blockIdx.x * 256ll + threadIdx.x;
    if (t >= (long long) n * nd) return;
    int i = (int) (t / nd), d = (int) (t % nd);
    out[t] = desc[(size_t) rows[i] * ds + d];
}

/* Validity bits of each query's sorted neighbour list (Kc entries per query) and m = the smallest
   knn0 * 2^j <= klim whose prefix holds `kc` valid neighbours (0 when none does). */
__global__ void k_kc_valid(const int *__restrict__ nbr, int Kc, int klim, int Q, const int *__restrict__ qpos,
                           const int *__restrict__ tpos, int min_dist2, int kc, int knn0,
                           unsigned long long *valid, int *m_out) {
    int q = blockIdx.x * 256 + threadIdx.x;
    if (q >= Q) return;
    int qx = pt_x(qpos[q]), qy = pt_y(qpos[q]);
    unsigned long long bits = 0;
    for (int j = 0; j < Kc && j < 64; j++) {
        int v = tpos[nbr[(size_t) q * Kc + j]];
        int dx = pt_x(v) - qx, dy = pt_y(v) - qy;
        if (dx * dx + dy * dy >= min_dist2) bits |= 1ull << j;
    }
    valid[q] = bits;
    int m = 0;
    for (int k = knn0; k <= klim; k *= 2) {
        unsigned long long mask = k >= 64 ? ~0ull : ((1ull << k) - 1);
        if (__popcll(bits & mask) >= kc) { m = k; break; }
    }
    m_out[q] = m;
}

/* Final knn of every query: running maximum of m over each segment, restarting at knn0. */
__global__ void k_kc_chain(const int *__restrict__ seg_start, int nseg, int Q, const int *__restrict__ m,
                           int knn0, int Kc, int *knn, int *overflow) {
    int s = blockIdx.x * 256 + threadIdx.x;
    if (s >= nseg) return;
    int q0 = seg_start[s], q1 = (s + 1 < nseg) ? seg_start[s + 1] : Q;
    int cur = knn0;
    for (int q = q0; q < q1; q++) {
        int mq = m[q];
        if (mq == 0) { atomicExch(overflow, 1); mq = Kc; }
        cur = max(cur, mq);
        if (cur > Kc) atomicExch(overflow, 1);
        knn[q] = min(cur, Kc);
    }
}

/* patch_dist_exact<float,8,3> (patchtable.h:330-373): four lane sums over 8 rows of 24
   interleaved RGB floats, lane q taking float indices q, q+4, ..., q+20 of each row in order,
   lanes added 0+1+2+3 at the end.  Inputs are RGBA images. */
__device__ __forceinline__ float ssd_exact(const float4 *__restrict__ A, int aw, int ax, int ay,
                                           const float4 *__restrict__ B, int bw, int bx, int by) {
    float l0 = 0.f, l1 = 0.f, l2 = 0.f, l3 = 0.f;
#pragma unroll 2
    for (int dy = 0; dy < 8; dy++) {
        const float4 *ar = A + (size_t) (ay + dy) * aw + ax;
        const float4 *br = B + (size_t) (by + dy) * bw + bx;
        float e[24];
#pragma unroll
        for (int p = 0; p < 8; p++) {
            float4 a = __ldg(ar + p), b = __ldg(br + p);
            float t0 = __fsub_rn(a.x, b.x), t1 = __fsub_rn(a.y, b.y), t2 = __fsub_rn(a.z, b.z);
            e[3 * p] = __fmul_rn(t0, t0); e[3 * p + 1] = __fmul_rn(t1, t1); e[3 * p + 2] = __fmul_rn(t2, t2);
        }
#pragma unroll
        for (int n = 0; n < 6; n++) {
            l0 = __fadd_rn(l0, e[4 * n]); l1 = __fadd_rn(l1, e[4 * n + 1]);
            l2 = __fadd_rn(l2, e[4 * n + 2]); l3 = __fadd_rn(l3, e[4 * n + 3]);
        }
    }
    return __fadd_rn(__fadd_rn(__fadd_rn(l0, l1), l2), l3);
}

/* Exact distance from each query patch to its first knn neighbours. */
__global__ void k_kc_ssd(const float4 *__restrict__ b, int bw, const int *__restrict__ nbr, int Kc, int Q,
                         const int *__restrict__ qpos, const int *__restrict__ tpos, const int *__restrict__ knn,
                         float *ssd) {
    long long t = blockIdx.x * 256ll + threadIdx.x;
    int q = (int) (t / Kc), j = (int) (t % Kc);
    if (q >= Q || j >= knn[q]) return;
    int v = tpos[nbr[(size_t) q * Kc + j]];
    ssd[(size_t) q * Kc + j] = ssd_exact(b, bw, pt_x(qpos[q]), pt_y(qpos[q]), b, bw, pt_x(v), pt_y(v));
}

/* Descriptor mode: patch_dist_approx of the two patches' descriptor store entries
   (TABLE_LOOKUP_PATCH_DIST with is_descriptor, patchtable.h:310-320). */
__global__ void k_kc_desc(const float4 *__restrict__ bdesc, int ds4, int nd, int ew, const int *__restrict__ nbr, int Kc,
                          int Q, const int *__restrict__ qpos, const int *__restrict__ tpos, const int *__restrict__ knn,
                          float *ssd) {
    long long t = blockIdx.x * 256ll + threadIdx.x;
    int q = (int) (t / Kc), j = (int) (t % Kc);
    if (q >= Q || j >= knn[q]) return;
    int v = tpos[nbr[(size_t) q * Kc + j]];
    float4 a[4];
    pt_desc_load(bdesc + ((size_t) pt_y(qpos[q]) * ew + pt_x(qpos[q])) * ds4, 4 * ds4, a);
    ssd[(size_t) q * Kc + j] = pt_desc_dist(a, bdesc + ((size_t) pt_y(v) * ew + pt_x(v)) * ds4, nd);
}

/* The sequential selection of one segment with incoming stale bit `bin` (the flag at index
   kc after the knn0 truncation).  Writes the kept (position, distance) pairs; returns the
   outgoing bit. */
__device__ int select_segment(int q0, int q1, int bin, int kc, int knn0, int Kc, const int *__restrict__ nbr,
                              const int *__restrict__ tpos, const unsigned long long *__restrict__ valid,
                              const int *__restrict__ knn, const float *__restrict__ ssd, int2 *outp) {
    unsigned long long F = bin ? (1ull << kc) : 0ull;   /* flags entering the first patch */
    int S = knn0;
    float sd[64];
    int sp[64], so[64];
    for (int q = q0; q < q1; q++) {
        int kq = knn[q];
        unsigned long long vb = valid[q];
        /* fresh flags up to and including the kc-th valid neighbour */
        int r = 0, nv = 0;
        while (r < kq) { if ((vb >> r) & 1ull) nv++; r++; if (nv >= kc) break; }
        unsigned long long fresh = r >= 64 ? vb : (vb & ((1ull << r) - 1));
        unsigned long long keep = (S >= 64) ? ~0ull : ((1ull << S) - 1);
        unsigned long long stale = F & keep & ~(r >= 64 ? ~0ull : ((1ull << r) - 1));
        unsigned long long flags = fresh | stale;
        /* sort (ssd, pos, flag) ascending; positions are distinct */
        for (int j = 0; j < kq; j++) {
            float d = ssd[(size_t) q * Kc + j];
            int p = tpos[nbr[(size_t) q * Kc + j]];
            int t = j;
            while (t > 0 && (sd[t - 1] > d || (sd[t - 1] == d && sp[t - 1] > p))) {
                sd[t] = sd[t - 1]; sp[t] = sp[t - 1]; so[t] = so[t - 1]; t--;
            }
            sd[t] = d; sp[t] = p; so[t] = j;
        }
        unsigned long long nf = 0;
        int cv = 0;
        for (int t = 0; t < kq; t++) {
            int f = (int) ((flags >> so[t]) & 1ull);
            if (f) nf |= 1ull << t;
            if (f && cv < kc) { outp[(size_t) q * kc + cv] = make_int2(sp[t], __float_as_int(sd[t])); cv++; }
        }
        F = nf;
        S = kq;
    }
    (void) Kc;
    return (int) ((F >> kc) & 1ull);
}

__global__ void k_kc_select(const int *__restrict__ seg_start, int nseg, int Q, int kc, int knn0, int Kc,
                            const int *__restrict__ nbr, const int *__restrict__ tpos,
                            const unsigned long long *__restrict__ valid, const int *__restrict__ knn,
                            const float *__restrict__ ssd, int2 *out0, int2 *out1, unsigned char *fn) {
    int s = blockIdx.x * 64 + threadIdx.x;
    if (s >= nseg) return;
    int q0 = seg_start[s], q1 = (s + 1 < nseg) ? seg_start[s + 1] : Q;
    int b0 = select_segment(q0, q1, 0, kc, knn0, Kc, nbr, tpos, valid, knn, ssd, out0);
    int b1 = select_segment(q0, q1, 1, kc, knn0, Kc, nbr, tpos, valid, knn, ssd, out1);
    fn[s] = (unsigned char) (b0 | (b1 << 1));   /* the segment's map of the carried bit */
}

/* Lists longer than 64 (Kc = 128 .. PT_KNN_WIDE_MAX): the same validity bits and selection with
   the flags held in W = Kc / 64 words and the per-patch sort in global scratch. */
constexpr int KW_WORDS = PT_KNN_WIDE_MAX / 64;

__device__ __forceinline__ unsigned long long below(int n, int w) {     /* bits [64w, n) of word w */
    const int lo = 64 * w;
    return n >= lo + 64 ? ~0ull : (n <= lo ? 0ull : ((1ull << (n - lo)) - 1));
}

__global__ void k_kc_valid_wide(const int *__restrict__ nbr, int Kc, int Q, const int *__restrict__ qpos,
                                const int *__restrict__ tpos, int min_dist2, int kc, int knn0,
                                unsigned long long *valid, int *m_out) {
    int q = blockIdx.x * 256 + threadIdx.x;
    if (q >= Q) return;
    const int W = Kc / 64;
    int qx = pt_x(qpos[q]), qy = pt_y(qpos[q]);
    unsigned long long *vq = valid + (size_t) q * W;
    for (int w = 0; w < W; w++) {
        unsigned long long bits = 0;
        for (int b = 0; b < 64; b++) {
            int v = tpos[nbr[(size_t) q * Kc + 64 * w + b]];
            int dx = pt_x(v) - qx, dy = pt_y(v) - qy;
            if (dx * dx + dy * dy >= min_dist2) bits |= 1ull << b;
        }
        vq[w] = bits;
    }
    int m = 0;
    for (int k = knn0; k <= Kc; k *= 2) {
        int c = 0;
        for (int w = 0; w < W; w++) c += __popcll(vq[w] & below(k, w));
        if (c >= kc) { m = k; break; }
    }
    m_out[q] = m;
}

__device__ int select_segment_wide(int q0, int q1, int bin, int kc, int knn0, int Kc, const int *__restrict__ nbr,
                                   const int *__restrict__ tpos, const unsigned long long *__restrict__ valid,
                                   const int *__restrict__ knn, const float *__restrict__ ssd, int2 *outp,
                                   float *sd, int *sp, int *so) {
    const int W = Kc / 64;
    unsigned long long F[KW_WORDS];
    for (int w = 0; w < KW_WORDS; w++) F[w] = 0ull;
    if (bin) F[kc >> 6] |= 1ull << (kc & 63);
    int S = knn0;
    for (int q = q0; q < q1; q++) {
        const int kq = knn[q];
        const unsigned long long *vb = valid + (size_t) q * W;
        int r = 0, nv = 0;
        while (r < kq) { if ((vb[r >> 6] >> (r & 63)) & 1ull) nv++; r++; if (nv >= kc) break; }
        unsigned long long flags[KW_WORDS];
        for (int w = 0; w < W; w++) flags[w] = (vb[w] & below(r, w)) | (F[w] & below(S, w) & ~below(r, w));
        for (int j = 0; j < kq; j++) {
            float d = ssd[(size_t) q * Kc + j];
            int p = tpos[nbr[(size_t) q * Kc + j]];
            int t = j;
            while (t > 0 && (sd[t - 1] > d || (sd[t - 1] == d && sp[t - 1] > p))) {
                sd[t] = sd[t - 1]; sp[t] = sp[t - 1]; so[t] = so[t - 1]; t--;
            }
            sd[t] = d; sp[t] = p; so[t] = j;
        }
        for (int w = 0; w < KW_WORDS; w++) F[w] = 0ull;
        int cv = 0;
        for (int t = 0; t < kq; t++) {
            const int o = so[t];
            const int f = (int) ((flags[o >> 6] >> (o & 63)) & 1ull);
            if (f) F[t >> 6] |= 1ull << (t & 63);
            if (f && cv < kc) { outp[(size_t) q * kc + cv] = make_int2(sp[t], __float_as_int(sd[t])); cv++; }
        }
        S = kq;
    }
    return (int) ((F[kc >> 6] >> (kc & 63)) & 1ull);
}

__global__ void k_kc_select_wide(const int *__restrict__ seg_start, int nseg, int Q, int kc, int knn0, int Kc,
                                 const int *__restrict__ nbr, const int *__restrict__ tpos,
                                 const unsigned long long *__restrict__ valid, const int *__restrict__ knn,
                                 const float *__restrict__ ssd, int2 *out0, int2 *out1, unsigned char *fn,
                                 float *sd, int *sp, int *so) {
    int s = blockIdx.x * 64 + threadIdx.x;
    if (s >= nseg) return;
    int q0 = seg_start[s], q1 = (s + 1 < nseg) ? seg_start[s + 1] : Q;
    const size_t o = (size_t) s * Kc;
    int b0 = select_segment_wide(q0, q1, 0, kc, knn0, Kc, nbr, tpos, valid, knn, ssd, out0, sd + o, sp + o, so + o);
    int b1 = select_segment_wide(q0, q1, 1, kc, knn0, Kc, nbr, tpos, valid, knn, ssd, out1, sd + o, sp + o, so + o);
    fn[s] = (unsigned char) (b0 | (b1 << 1));
}

/* Composition of bit maps f encoded as (f(0) | f(1) << 1): apply a, then b. */
struct ComposeOp {
    __device__ unsigned char operator()(unsigned char a, unsigned char b) const {
        int a0 = a & 1, a1 = (a >> 1) & 1;
        int r0 = (b >> a0) & 1, r1 = (b >> a1) & 1;
        return (unsigned char) (r0 | (r1 << 1));
    }
};

/* Picks each segment's scenario given the carried bit (the composed map of all earlier segments
   applied to the initial 0) and writes the k-coherence set. */
__global__ void k_kc_finish(const int *__restrict__ seg_start, int nseg, int Q, int kc,
                            const unsigned char *__restrict__ prefix, const int2 *__restrict__ out0,
                            const int2 *__restrict__ out1, const int *__restrict__ qcell, int2 *kcoh) {
    int s = blockIdx.x * 256 + threadIdx.x;
    if (s >= nseg) return;
    int bin = s == 0 ? 0 : (prefix[s - 1] & 1);
    const int2 *src = bin ? out1 : out0;
    int q0 = seg_start[s], q1 = (s + 1 < nseg) ? seg_start[s + 1] : Q;
    for (int q = q0; q < q1; q++)
        for (int k = 0; k < kc; k++) kcoh[(size_t) qcell[q] * kc + k] = src[(size_t) q * kc + k];
}

}  // namespace

/* train: N x nd compact descriptors (row order = FLANN index order); tpos: packed positions
   (patch coords) of the train points.  Queries are train rows qrow[q] at positions qpos[q], in
   the reference's loop order, with output cell qcell[q] (index into the beh x bew grid).
   seg_start: first query of each segment.  kcoh receives beh x bew x kc (pos, dist bits). */
namespace {

/* The k-coherence index lists of a build without an allowed mask (build_kcoherence's loops):
   train point i = patch (tx * fbs, ty * fbs) in raster order; query i = patch (qx * ks, qy * ks)
   with its output cell; segment j starts at query row j / ncols, column cols[j % ncols]. */
__global__ void k_kc_lists(int ew, int fbs, int ks, int ntx, int nqx, int N, int Q, int ncols, int nseg,
                           const int *__restrict__ cols, int *trows, int *tpos, int *qrows, int *qpos, int *qcell, int *seg) {
    const long long i = blockIdx.x * 256ll + threadIdx.x;
    if (i < N) {
        const int y = (int) (i / ntx) * fbs, x = (int) (i % ntx) * fbs;
        trows[i] = y * ew + x;
        tpos[i] = pt_xy(x, y);
    }
    if (i < Q) {
        const int py = (int) (i / nqx) * ks, px = (int) (i % nqx) * ks;
        qrows[i] = py * ew + px;
        qpos[i] = pt_xy(px, py);
        qcell[i] = (py / ks) * ew + px / ks;
    }
    if (i < nseg) seg[i] = (int) (i / ncols) * nqx + cols[i % ncols];
}

/* Masked lists, step 1: which train and query grid points are allowed patches. */
__global__ void k_kc_flags(const int *__restrict__ allowed, int idx, int ew, int fbs, int ks, int ntx, int N0, int nqx,
                           int Q0, int *tflag, int *qflag) {
    const long long i = blockIdx.x * 256ll + threadIdx.x;
    if (i < N0) {
        const int y = (int) (i / ntx) * fbs, x = (int) (i % ntx) * fbs;
        tflag[i] = __ldg(allowed + (size_t) y * ew + x) == idx;
    }
    if (i < Q0) {
        const int py = (int) (i / nqx) * ks, px = (int) (i % nqx) * ks;
        qflag[i] = __ldg(allowed + (size_t) py * ew + px) == idx;
    }
}

/* Step 2: an allowed query opens a segment when it is the first allowed query or its column
   satisfies the reset rule ((x / ks) % reset == 0, x in padded coordinates). */
__global__ void k_kc_segflags(int ks, int reset, int nqx, int Q0, const int *__restrict__ qflag,
                              const int *__restrict__ qinc, int *gflag) {
    const long long i = blockIdx.x * 256ll + threadIdx.x;
    if (i >= Q0) return;
    const int px = (int) (i % nqx) * ks;
    gflag[i] = qflag[i] && (qinc[i] == 1 || ((px + 7) / ks) % reset == 0);
}

/* Step 3: allowed points go to their ranks among the allowed ones (inclusive scans - 1), so the
   lists keep the raster order of the unmasked loops with the disallowed points left out. */
__global__ void k_kc_scatter(int ew, int fbs, int ks, int ntx, int N0, int nqx, int Q0, const int *__restrict__ tflag,
                             const int *__restrict__ tinc, const int *__restrict__ qflag, const int *__restrict__ qinc,
                             const int *__restrict__ gflag, const int *__restrict__ ginc, int *trows, int *tpos,
                             int *qrows, int *qpos, int *qcell, int *seg) {
    const long long i = blockIdx.x * 256ll + threadIdx.x;
    if (i < N0 && tflag[i]) {
        const int y = (int) (i / ntx) * fbs, x = (int) (i % ntx) * fbs, o = tinc[i] - 1;
        trows[o] = y * ew + x;
        tpos[o] = pt_xy(x, y);
    }
    if (i < Q0 && qflag[i]) {
        const int py = (int) (i / nqx) * ks, px = (int) (i % nqx) * ks, o = qinc[i] - 1;
        qrows[o] = py * ew + px;
        qpos[o] = pt_xy(px, py);
        qcell[o] = (py / ks) * ew + px / ks;
        if (gflag[i]) seg[ginc[i] - 1] = o;
    }
}

}  // namespace

pt_status pt_kc_lists_masked(int ew, int eh, int fbs, int ks, int reset, const int *allowed, int allowed_index,
                             int *trows, int *tpos, int *qrows, int *qpos, int *qcell, int *seg, int *n_out, int *q_out,
                             int *nseg_out, cudaStream_t st) {
    const int ntx = (ew + fbs - 1) / fbs, nty = (eh + fbs - 1) / fbs;
    const int nqx = (ew + ks - 1) / ks, nqy = (eh + ks - 1) / ks;
    const long long N0 = (long long) ntx * nty, Q0 = (long long) nqx * nqy;
    if (Q0 >= (1ll << 31) || N0 >= (1ll << 31) || reset < 1)
        return pt_fail(PT_UNSUPPORTED, "k-coherence index lists");    /* callers use the general path */
    const long long M = std::max(N0, Q0);
    DevBuf<int> tflag, tinc, qflag, qinc, gflag, ginc, tot;
    PT_CUDA(tflag.reserve(N0)); PT_CUDA(tinc.reserve(N0));
    PT_CUDA(qflag.reserve(Q0)); PT_CUDA(qinc.reserve(Q0));
    PT_CUDA(gflag.reserve(Q0)); PT_CUDA(ginc.reserve(Q0));
    PT_CUDA(tot.reserve(3));
    size_t tmp_bytes = 0;
    PT_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, tflag.p, tinc.p, (int) M, st));
    DevBuf<unsigned char> tmp;
    PT_CUDA(tmp.reserve(tmp_bytes));
    const unsigned blocks = (unsigned) ((M + 255) / 256);
    k_kc_flags<<<blocks, 256, 0, st>>>(allowed, allowed_index, ew, fbs, ks, ntx, (int) N0, nqx, (int) Q0, tflag.p, qflag.p);
    PT_LAUNCHED();
    size_t b = tmp_bytes;
    PT_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, b, tflag.p, tinc.p, (int) N0, st));
    b = tmp_bytes;
    PT_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, b, qflag.p, qinc.p, (int) Q0, st));
    k_kc_segflags<<<(unsigned) ((Q0 + 255) / 256), 256, 0, st>>>(ks, reset, nqx, (int) Q0, qflag.p, qinc.p, gflag.p);
    PT_LAUNCHED();
    b = tmp_bytes;
    PT_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, b, gflag.p, ginc.p, (int) Q0, st));
    k_kc_scatter<<<blocks, 256, 0, st>>>(ew, fbs, ks, ntx, (int) N0, nqx, (int) Q0, tflag.p, tinc.p, qflag.p, qinc.p,
                                         gflag.p, ginc.p, trows, tpos, qrows, qpos, qcell, seg);
    PT_LAUNCHED();
    PT_CUDA(cudaMemcpyAsync(tot.p, tinc.p + N0 - 1, sizeof(int), cudaMemcpyDeviceToDevice, st));
    PT_CUDA(cudaMemcpyAsync(tot.p + 1, qinc.p + Q0 - 1, sizeof(int), cudaMemcpyDeviceToDevice, st));
    PT_CUDA(cudaMemcpyAsync(tot.p + 2, ginc.p + Q0 - 1, sizeof(int), cudaMemcpyDeviceToDevice, st));
    int h_tot[3] = {0, 0, 0};
    PT_CUDA(cudaMemcpyAsync(h_tot, tot.p, sizeof(h_tot), cudaMemcpyDeviceToHost, st));
    PT_CUDA(cudaStreamSynchronize(st));           /* the scratch goes out of scope */
    *n_out = h_tot[0];
    *q_out = h_tot[1];
    *nseg_out = h_tot[2];
    return PT_OK;
}

pt_status pt_kc_lists(int ew, int eh, int fbs, int ks, int reset, int *trows, int *tpos, int *qrows, int *qpos,
                      int *qcell, int *seg, int *n_out, int *q_out, int *nseg_out, cudaStream_t st) {
    const int ntx = (ew + fbs - 1) / fbs, nty = (eh + fbs - 1) / fbs;
    const int nqx = (ew + ks - 1) / ks, nqy = (eh + ks - 1) / ks;
    const long long N = (long long) ntx * nty, Q = (long long) nqx * nqy;
    /* the columns where a segment starts: (x / ks) % reset == 0 with x = px + 7 in padded
       coordinates (patchtable.h:2714); the first query always starts one */
    std::vector<int> cols;
    for (int qx = 0; qx < nqx; qx++)
        if (((qx * ks + 7) / ks) % reset == 0) cols.push_back(qx);
    if (cols.empty() || Q >= (1ll << 31) || N >= (1ll << 31))
        return pt_fail(PT_UNSUPPORTED, "k-coherence index lists");    /* callers use the general path */
    const bool first = cols[0] != 0;                                   /* query 0 opens a segment of its own */
    const long long nseg = (long long) nqy * (long long) cols.size();
    DevBuf<int> d_cols;
    PT_CUDA(d_cols.reserve(cols.size()));
    PT_CUDA(cudaMemcpyAsync(d_cols.p, cols.data(), sizeof(int) * cols.size(), cudaMemcpyHostToDevice, st));
    const long long tot = std::max(std::max(N, Q), nseg);
    k_kc_lists<<<(unsigned) ((tot + 255) / 256), 256, 0, st>>>(ew, fbs, ks, ntx, nqx, (int) N, (int) Q, (int) cols.size(),
                                                           (int) nseg, d_cols.p, trows, tpos, qrows, qpos, qcell,
                                                           seg + (first ? 1 : 0));
    PT_LAUNCHED();
    if (first) PT_CUDA(cudaMemsetAsync(seg, 0, sizeof(int), st));
    PT_CUDA(cudaStreamSynchronize(st));           /* d_cols goes out of scope */
    *n_out = (int) N;
    *q_out = (int) Q;
    *nseg_out = (int) nseg + (first ? 1 : 0);
    return PT_OK;
}

pt_status pt_gather_rows(const float *desc, int ds, int nd, const int *rows, int n, float *out, cudaStream_t st) {
    long long tot = (long long) n * nd;
    k_gather_rows<<<(unsigned) ((tot + 255) / 256), 256, 0, st>>>(desc, ds, nd, rows, n, out);
    PT_LAUNCHED();
    return PT_OK;
}

pt_status pt_kcoherence(const float4 *b_rgba, int bw, const float *bdesc, int ds, int ew, const float *train, int N, int nd, const int *tpos,
                        const float *qdesc, const int *qpos, const int *qcell, int Q, const int *seg_start, int nseg,
                        int kc, int min_dist, int2 *kcoh, int *max_knn_out, cudaStream_t st) {
    if (kc < 1 || kc >= 32) return pt_fail(PT_UNSUPPORTED, "kcoherence must be in 1..31");
    int knn0 = kc + 1;
    int Kcap = 16;
    while (Kcap < 2 * knn0) Kcap *= 2;
    for (;;) {
        if (Kcap > PT_KNN_WIDE_MAX)
            return pt_fail(PT_UNSUPPORTED, "k-coherence needs more than %d neighbours for some patch", PT_KNN_WIDE_MAX);
        const bool wide = Kcap > 64;
        /* The knn chain only takes the values knn0 * 2^j: with a capacity of Kcap neighbours the
           longest list any patch can use is klim, the largest of them within Kcap, so the search
           asks for the smallest supported width Kc >= klim (fewer neighbours to keep sorted and a
           tighter pruning bound); the first klim entries are the same as in a wider search. */
        int klim = knn0;
        while (2 * klim <= Kcap) klim *= 2;
        int Kc = Kcap;
        if (!wide) {
            static const int widths[] = {12, 16, 24, 32, 48, 64};
            for (int wv : widths)
                if (wv >= klim) { Kc = wv; break; }
        } else {
            klim = Kcap;
        }
        const int W = wide ? Kc / 64 : 1;
        if (Kc > N) return pt_fail(PT_BAD_ARG, "k-coherence: image has too few patches (%d)", N);
        DevBuf<int> nbr, mm, knn, ovf;
        DevBuf<unsigned long long> valid;
        DevBuf<float> ssd;
        PT_CUDA(nbr.reserve((size_t) Q * Kc));
        PT_CUDA(mm.reserve(Q));
        PT_CUDA(knn.reserve(Q));
        PT_CUDA(ovf.reserve(1));
        PT_CUDA(valid.reserve((size_t) Q * W));
        PT_CUDA(ssd.reserve((size_t) Q * Kc));
        PT_TRY(pt_launch_knn(train, N, nd, qdesc, Q, Kc, nbr.p, st));
        if (wide)
            k_kc_valid_wide<<<(Q + 255) / 256, 256, 0, st>>>(nbr.p, Kc, Q, qpos, tpos, min_dist * min_dist, kc, knn0, valid.p,
                                                             mm.p);
        else
            k_kc_valid<<<(Q + 255) / 256, 256, 0, st>>>(nbr.p, Kc, klim, Q, qpos, tpos, min_dist * min_dist, kc, knn0,
                                                        valid.p, mm.p);
        PT_LAUNCHED();
        PT_CUDA(cudaMemsetAsync(ovf.p, 0, sizeof(int), st));
        k_kc_chain<<<(nseg + 255) / 256, 256, 0, st>>>(seg_start, nseg, Q, mm.p, knn0, klim, knn.p, ovf.p);
        PT_LAUNCHED();
        int overflow = 0;
        PT_CUDA(cudaMemcpyAsync(&overflow, ovf.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        PT_CUDA(cudaStreamSynchronize(st));
        if (overflow) { Kcap *= 2; continue; }
        long long tot = (long long) Q * Kc;
        if (bdesc)
            k_kc_desc<<<(unsigned) ((tot + 255) / 256), 256, 0, st>>>(reinterpret_cast<const float4 *>(bdesc), ds / 4, nd, ew,
                                                                      nbr.p, Kc, Q, qpos, tpos, knn.p, ssd.p);
        else
            k_kc_ssd<<<(unsigned) ((tot + 255) / 256), 256, 0, st>>>(b_rgba, bw, nbr.p, Kc, Q, qpos, tpos, knn.p, ssd.p);
        PT_LAUNCHED();
        DevBuf<int2> o0, o1;
        DevBuf<unsigned char> fn, pre;
        PT_CUDA(o0.reserve((size_t) Q * kc));
        PT_CUDA(o1.reserve((size_t) Q * kc));
        PT_CUDA(fn.reserve(nseg));
        PT_CUDA(pre.reserve(nseg));
        DevBuf<float> wsd;
        DevBuf<int> wsp, wso;
        if (wide) {
            PT_CUDA(wsd.reserve((size_t) nseg * Kc));
            PT_CUDA(wsp.reserve((size_t) nseg * Kc));
            PT_CUDA(wso.reserve((size_t) nseg * Kc));
            k_kc_select_wide<<<(nseg + 63) / 64, 64, 0, st>>>(seg_start, nseg, Q, kc, knn0, Kc, nbr.p, tpos, valid.p, knn.p,
                                                             ssd.p, o0.p, o1.p, fn.p, wsd.p, wsp.p, wso.p);
        } else {
            k_kc_select<<<(nseg + 63) / 64, 64, 0, st>>>(seg_start, nseg, Q, kc, knn0, Kc, nbr.p, tpos, valid.p, knn.p,
                                                        ssd.p, o0.p, o1.p, fn.p);
        }
        PT_LAUNCHED();
        size_t tb = 0;
        PT_CUDA(cub::DeviceScan::InclusiveScan(nullptr, tb, fn.p, pre.p, ComposeOp(), nseg, st));
        DevBuf<unsigned char> tmp;
        PT_CUDA(tmp.reserve(tb));
        PT_CUDA(cub::DeviceScan::InclusiveScan(tmp.p, tb, fn.p, pre.p, ComposeOp(), nseg, st));
        pt_count_launches(1);
        k_kc_finish<<<(nseg + 255) / 256, 256, 0, st>>>(seg_start, nseg, Q, kc, pre.p, o0.p, o1.p, qcell, kcoh);
        PT_LAUNCHED();
        if (max_knn_out) *max_knn_out = klim;
        PT_CUDA(cudaStreamSynchronize(st));
        return PT_OK;
    }
}
