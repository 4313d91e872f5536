/* Query kernels: nearest-neighbour field from image a to the table image b.

   Replaces lookup_templated<0,0> (patchtable/patchtable.h:3468-4217).  The reference sweeps the
   patches in scanline order (reversed on odd iterations); at each patch it
     1. starts from the stored match with its distance scaled by prop_scale = 1/(1+coherence_spatial),
     2. tries the table cell of the patch's descriptor on the first iteration (:3641-3709),
     3. tries the k-coherence neighbours of the current best, stopping once the stored
        distance of a neighbour reaches triangle_factor * best (:3750-3851),
     4. pushes the chosen offset to the 3x3 neighbourhood, replacing a neighbour's match when the
        pushed patch is closer (summed-area-table propagation, :3908-4145).
   Here every patch runs steps 1-3 at once ("choose"), then every patch takes the best of the
   offsets its neighbours chose ("pull", the mirror image of the push), and the pair of phases
   repeats for a fixed number of passes.  All distances are the reference's patch_dist_exact
   (patchtable.h:330-373) evaluated in the same float order, so every returned NNF_DIST is that
   function's value for the returned match; a candidate's sum stops early once its partial sum
   already reaches the value it must beat (the partial sum can only grow). */
#include <cuda_runtime.h>

#include <cstring>

#include "pt_internal.h"
#include "pt_kernels.h"

namespace {

constexpr int NT = 256;

struct QPlan {
    int aw, ah;              /* a image size (pixels) */
    int ew, eh;              /* a patches */
    int bw, bh;              /* b image size */
    int bew, beh;            /* b patches */
    double prop_scale;
    double triangle;
    int kc, ks;              /* kcoherence, kcoherence_step */
    int radius;              /* query_step + prop_dist */
    int do_kcoh;
    int step;                /* neighbour spacing of this pull pass (jump flooding) */
};

__device__ __forceinline__ float finf() { return __int_as_float(0x7f800000); }

/* Adds per-thread counts to counters[0..1] with one atomic per warp (profiling only). */
__device__ __forceinline__ void count_work(unsigned long long *counters, unsigned cand, unsigned rows) {
    if (!counters) return;
    unsigned c = __reduce_add_sync(0xffffffffu, cand), r = __reduce_add_sync(0xffffffffu, rows);
    if ((threadIdx.x & 31) == 0) { atomicAdd(counters, (unsigned long long) c); atomicAdd(counters + 1, (unsigned long long) r); }
}

constexpr int TW = 256;                   /* query patches per CTA row segment */
constexpr int ATW = TW + 7;               /* pixels per staged a row */

/* Stages the 8 pixel rows under a CTA's row segment of query patches in shared memory. */
__device__ __forceinline__ void stage_a(float4 *atile, const float4 *__restrict__ a, int aw, int ah, int x0, int y) {
    for (int i = threadIdx.x; i < 8 * ATW; i += TW) {
        int r = i / ATW, c = i - r * ATW;
        int gx = x0 + c, gy = y + r;
        atile[i] = (gx < aw && gy < ah) ? __ldg(a + (size_t) gy * aw + gx) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

/* patch_dist_exact with the query patch in shared memory, streamed pixel by pixel into the four
   SSE lanes (interleaved RGB float e = 3p + c goes to lane e & 3, in increasing e per lane, as
   patchtable.h:349-356 sums it); abandons the sum once a row's partial total reaches `bound`. */
__device__ __forceinline__ float ssd_tile(const float4 *atile, int tx, const float4 *__restrict__ B, int bw,
                                          int bx, int by, float bound, unsigned &rows) {
    float l0 = 0.f, l1 = 0.f, l2 = 0.f, l3 = 0.f;
#pragma unroll 1
    for (int dy = 0; dy < 8; dy++) {
        rows++;
        const float4 *ar = atile + dy * ATW + tx;
        const float4 *br = B + (size_t) (by + dy) * bw + bx;
#pragma unroll
        for (int p = 0; p < 8; p++) {
            float4 av = ar[p], bv = __ldg(br + p);
            float t0 = __fsub_rn(av.x, bv.x), t1 = __fsub_rn(av.y, bv.y), t2 = __fsub_rn(av.z, bv.z);
            float q0 = __fmul_rn(t0, t0), q1 = __fmul_rn(t1, t1), q2 = __fmul_rn(t2, t2);
            /* e = 3p, 3p+1, 3p+2 -> lanes (3p) & 3, (3p+1) & 3, (3p+2) & 3 */
            const int e0 = (3 * p) & 3, e1 = (3 * p + 1) & 3, e2 = (3 * p + 2) & 3;
            if (e0 == 0) l0 = __fadd_rn(l0, q0); else if (e0 == 1) l1 = __fadd_rn(l1, q0); else if (e0 == 2) l2 = __fadd_rn(l2, q0); else l3 = __fadd_rn(l3, q0);
            if (e1 == 0) l0 = __fadd_rn(l0, q1); else if (e1 == 1) l1 = __fadd_rn(l1, q1); else if (e1 == 2) l2 = __fadd_rn(l2, q1); else l3 = __fadd_rn(l3, q1);
            if (e2 == 0) l0 = __fadd_rn(l0, q2); else if (e2 == 1) l1 = __fadd_rn(l1, q2); else if (e2 == 2) l2 = __fadd_rn(l2, q2); else l3 = __fadd_rn(l3, q2);
        }
        if (dy < 7 && __fadd_rn(__fadd_rn(__fadd_rn(l0, l1), l2), l3) >= bound) return finf();
    }
    return __fadd_rn(__fadd_rn(__fadd_rn(l0, l1), l2), l3);
}

/* Up to G candidates' sums advanced together row by row, so each query row is read from shared
   memory once per group; each candidate's sum keeps the reference's lane order and stops once its
   partial total reaches `bound`.  Returns the candidates' full sums (+inf when stopped). */
template<int G>
__device__ __forceinline__ void ssd_group(const float4 *atile, int tx, const float4 *__restrict__ B, int bw,
                                          const int *cand, int nc, float bound, float *out, unsigned &rows) {
    float l[G][4];
    bool live[G];
#pragma unroll
    for (int g = 0; g < G; g++) { l[g][0] = l[g][1] = l[g][2] = l[g][3] = 0.f; live[g] = g < nc; }
#pragma unroll 1
    for (int dy = 0; dy < 8; dy++) {
        bool any = false;
#pragma unroll
        for (int g = 0; g < G; g++) any |= live[g];
        if (!any) break;
        float4 av[8];
#pragma unroll
        for (int p = 0; p < 8; p++) av[p] = atile[dy * ATW + tx + p];
#pragma unroll
        for (int g = 0; g < G; g++) {
            if (!live[g]) continue;
            rows++;
            const float4 *br = B + (size_t) (pt_y(cand[g]) + dy) * bw + pt_x(cand[g]);
#pragma unroll
            for (int p = 0; p < 8; p++) {
                float4 bv = __ldg(br + p);
                float t0 = __fsub_rn(av[p].x, bv.x), t1 = __fsub_rn(av[p].y, bv.y), t2 = __fsub_rn(av[p].z, bv.z);
                float q[3] = {__fmul_rn(t0, t0), __fmul_rn(t1, t1), __fmul_rn(t2, t2)};
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const int e = (3 * p + c) & 3;   /* SSE lane of interleaved float 3p + c */
                    l[g][e] = __fadd_rn(l[g][e], q[c]);
                }
            }
            if (dy < 7 && __fadd_rn(__fadd_rn(__fadd_rn(l[g][0], l[g][1]), l[g][2]), l[g][3]) >= bound) live[g] = false;
        }
    }
#pragma unroll
    for (int g = 0; g < G; g++)
        out[g] = live[g] ? __fadd_rn(__fadd_rn(__fadd_rn(l[g][0], l[g][1]), l[g][2]), l[g][3]) : finf();
}

/* Proposals of the learned network for one patch (LEARNED instantiation of k_choose_tile). */
struct LearnedArgs {
    const int *cand;          /* n x 8 table entries, -1 = none; NULL on passes without proposals */
    const float *conf;        /* n: probability of the best proposed cell */
    float threshold;          /* patches below it keep the plain candidates */
    int kcoh_confident;       /* confident patches also try k-coherence */
    unsigned long long *counters;   /* [confident patches, proposals scored] or NULL */
};

/* Steps 1-3 for every patch ("choose"): returns the chosen match and its exact distance.  One CTA
   per 256-patch row segment, with the segment's query rows staged in shared memory.  The LEARNED
   instantiation replaces, for patches whose proposal confidence reaches the threshold, the table
   candidate by the network's proposals (scored best-first in groups of three) and, unless
   configured otherwise, skips k-coherence for them. */
template<bool LEARNED>
__global__ void __launch_bounds__(TW)
k_choose_tile(const QPlan c_q, const float4 *__restrict__ a, const float4 *__restrict__ b, const int *__restrict__ cur_pos,
              const float *__restrict__ cur_d, const int *__restrict__ tcand, const int2 *__restrict__ kcoh, int do_table,
              int *ch_pos, float *ch_d, int *kc_done, int use_done, unsigned long long *counters, const LearnedArgs la) {
    extern __shared__ float4 atile[];
    const int x0 = blockIdx.x * TW, y = blockIdx.y;
    stage_a(atile, a, c_q.aw, c_q.ah, x0, y);
    __syncthreads();
    const int x = x0 + threadIdx.x;
    const bool live = x < c_q.ew;
    unsigned ne = 0, rows = 0, n_conf = 0, n_prop = 0;
    if (live) {
        const int p = y * c_q.ew + x;
        int pos = cur_pos[p];
        float dstore = cur_d[p];
        int xb = pt_x(pos), yb = pt_y(pos);
        float dbest = (float) ((double) dstore * c_q.prop_scale);
        float dch = dstore;
        bool confident = false;
        if (LEARNED) confident = la.conf[p] >= la.threshold;
        if (LEARNED && confident && do_table && la.cand) {
            int cand[PT_PROP_TOPK];
            int nc = 0;
            const int4 *cp = reinterpret_cast<const int4 *>(la.cand + (size_t) p * PT_PROP_TOPK);
            const int4 c0 = cp[0], c1 = cp[1];
            const int raw[PT_PROP_TOPK] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
#pragma unroll
            for (int j = 0; j < PT_PROP_TOPK; j++) {
                if (raw[j] < 0) continue;
                const int c = pt_xy(pt_x(raw[j]) - 7, pt_y(raw[j]) - 7);
                bool dup = c == pt_xy(xb, yb);
                for (int t = 0; t < nc; t++) dup |= cand[t] == c;
                if (!dup) cand[nc++] = c;
            }
            constexpr int G = 3;
            for (int g0 = 0; g0 < nc; g0 += G) {
                float d[G];
                ssd_group<G>(atile, threadIdx.x, b, c_q.bw, cand + g0, nc - g0, dbest, d, rows);
#pragma unroll
                for (int g = 0; g < G; g++)
                    if (g0 + g < nc && d[g] < dbest) { dbest = d[g]; dch = d[g]; xb = pt_x(cand[g0 + g]); yb = pt_y(cand[g0 + g]); }
            }
            ne += nc;
            n_conf = 1;
            n_prop = nc;
        } else if (do_table) {
            int v = tcand[p];
            int xs = pt_x(v) - 7, ys = pt_y(v) - 7;
            if (xs != xb || ys != yb) {
                float dc = ssd_tile(atile, threadIdx.x, b, c_q.bw, xs, ys, dbest, rows);
                ne++;
                if (dc < dbest) { dbest = dc; dch = dc; xb = xs; yb = ys; }
            }
        }
        const int kc_src = pt_xy(xb, yb);
        const bool repeat = use_done && kc_done[p] == kc_src;
        bool accepted = false;
        const bool kc_here = !LEARNED || !confident || la.kcoh_confident;
        if (c_q.do_kcoh && kc_here && !repeat && xb < c_q.bew && yb < c_q.beh) {
            int ks = c_q.ks;
            const int2 *kp = kcoh + ((size_t) (yb / ks) * c_q.bew + (xb / ks)) * c_q.kc;
            int kdx = ks > 1 ? xb % ks : 0, kdy = ks > 1 ? yb % ks : 0;
            for (int k = 0; k < c_q.kc; k++) {
                int2 e = kp[k];
                float kd = __int_as_float(e.y);
                if ((double) kd >= c_q.triangle * (double) dbest) break;
                int xs = pt_x(e.x) + kdx, ys = pt_y(e.x) + kdy;
                if (xs >= c_q.bew) xs = c_q.bew - 1;
                if (ys >= c_q.beh) ys = c_q.beh - 1;
                float dc = ssd_tile(atile, threadIdx.x, b, c_q.bw, xs, ys, dbest, rows);
                ne++;
                if (dc < dbest) { dbest = dc; dch = dc; xb = xs; yb = ys; accepted = true; }
            }
        }
        if (c_q.do_kcoh) kc_done[p] = (repeat || !accepted) ? kc_src : -1;
        ch_pos[p] = pt_xy(xb, yb);
        ch_d[p] = dch;
    }
    count_work(counters, ne, rows);
    if (LEARNED && la.counters) {
        unsigned c = __reduce_add_sync(0xffffffffu, n_conf), q = __reduce_add_sync(0xffffffffu, n_prop);
        if ((threadIdx.x & 31) == 0) { atomicAdd(la.counters, (unsigned long long) c); atomicAdd(la.counters + 1, (unsigned long long) q); }
    }
}

/* Step 4 as a pull: the best of the stored match and every neighbour's chosen offset applied to
   this patch.  The patch's own choice comes first; the distinct neighbour candidates follow in
   increasing order of the distance their neighbour achieved with them (the likeliest good ones
   first, so the running best -- the early-exit bound -- tightens soonest), three at a time.
   Neighbours sit `step` patches apart; passes with decreasing steps (jump flooding) carry an
   offset across a region in a logarithmic number of passes, where the reference's sequential
   sweep carries it along a whole row in one sweep. */
template<int R>
__global__ void __launch_bounds__(TW)
k_pull_tile(const QPlan c_q, const float4 *__restrict__ a, const float4 *__restrict__ b, const int *__restrict__ cur_pos,
            const float *__restrict__ cur_d, const int *__restrict__ ch_pos, const float *__restrict__ ch_d,
            int *nxt_pos, float *nxt_d, unsigned long long *counters) {
    extern __shared__ float4 atile[];
    const int x0 = blockIdx.x * TW, y = blockIdx.y;
    stage_a(atile, a, c_q.aw, c_q.ah, x0, y);
    __syncthreads();
    const int x = x0 + threadIdx.x;
    const bool live = x < c_q.ew;
    unsigned ne = 0, rows = 0;
    if (live) {
        const int p = y * c_q.ew + x;
        int bpos = cur_pos[p];
        float bd = cur_d[p];
        {
            int cp = ch_pos[p];
            if (pt_x(cp) < c_q.bew && pt_y(cp) < c_q.beh && cp != bpos && ch_d[p] < bd) { bd = ch_d[p]; bpos = cp; }
        }
        constexpr int MAXC = (2 * R + 1) * (2 * R + 1) - 1;
        int cand[MAXC];
        float key[MAXC];
        int nc = 0;
        const int S = c_q.step;
#pragma unroll
        for (int dy = -R; dy <= R; dy++) {
#pragma unroll
            for (int dx = -R; dx <= R; dx++) {
                if (dx == 0 && dy == 0) continue;
                int ny = y + S * dy, nx = x + S * dx;
                if (ny < 0 || ny >= c_q.eh || nx < 0 || nx >= c_q.ew) continue;
                int q = ny * c_q.ew + nx;
                int cp = ch_pos[q];
                int xs = pt_x(cp) - S * dx, ys = pt_y(cp) - S * dy;
                if (xs < 0 || ys < 0 || xs >= c_q.bew || ys >= c_q.beh) continue;
                int c = pt_xy(xs, ys);
                bool dup = c == bpos;
                for (int t = 0; t < nc; t++) dup |= cand[t] == c;
                if (dup) continue;
                /* insertion by the neighbour's own distance (ties keep neighbour order) */
                float k = ch_d[q];
                int t = nc++;
                while (t > 0 && key[t - 1] > k) { key[t] = key[t - 1]; cand[t] = cand[t - 1]; t--; }
                key[t] = k;
                cand[t] = c;
            }
        }
        constexpr int G = 3;
        for (int c0 = 0; c0 < nc; c0 += G) {
            float d[G];
            ssd_group<G>(atile, threadIdx.x, b, c_q.bw, cand + c0, nc - c0, bd, d, rows);
#pragma unroll
            for (int g = 0; g < G; g++)
                if (c0 + g < nc && d[g] < bd) { bd = d[g]; bpos = cand[c0 + g]; }
        }
        ne += nc;
        nxt_pos[p] = bpos;
        nxt_d[p] = bd;
    }
    count_work(counters, ne, rows);
}

__global__ void k_init(int n, int pos, float d, int *cur_pos, float *cur_d) {
    int p = blockIdx.x * NT + threadIdx.x;
    if (p < n) { cur_pos[p] = pos; cur_d[p] = d; }
}

__global__ void k_output(int n, const int *__restrict__ pos, const float *__restrict__ d, double *ann) {
    int p = blockIdx.x * NT + threadIdx.x;
    if (p >= n) return;
    int v = pos[p];
    ann[3 * (size_t) p + 0] = pt_x(v);
    ann[3 * (size_t) p + 1] = pt_y(v);
    ann[3 * (size_t) p + 2] = d[p];
}

}  // namespace

static pt_status make_qplan(const QuerySetup &s, QPlan &q) {
    memset(&q, 0, sizeof(q));
    q.aw = s.aw; q.ah = s.ah; q.ew = s.aw - 7; q.eh = s.ah - 7;
    q.bw = s.bw; q.bh = s.bh; q.bew = s.bw - 7; q.beh = s.bh - 7;
    q.prop_scale = s.prop_scale;
    q.triangle = s.triangle_factor;
    q.kc = s.kcoherence;
    q.ks = s.kcoherence_step;
    q.radius = s.radius;
    q.do_kcoh = s.kcoherence > 0;
    q.step = s.step < 1 ? 1 : s.step;
    if (q.radius > 2) return pt_fail(PT_UNSUPPORTED, "propagation radius %d > 2 on the GPU path", q.radius);
    return PT_OK;
}

pt_status pt_launch_init(int n, int pos, float d, int *cur_pos, float *cur_d, cudaStream_t st) {
    k_init<<<(n + NT - 1) / NT, NT, 0, st>>>(n, pos, d, cur_pos, cur_d);
    PT_LAUNCHED();
    return PT_OK;
}

pt_status pt_launch_choose(const QuerySetup &s, int n, const float4 *a, const float4 *b, const int *cur_pos, const float *cur_d,
                           const int *tcand, const int2 *kcoh, int do_table, int *ch_pos,
                           float *ch_d, int *kc_done, int use_done, unsigned long long *evals, cudaStream_t st) {
    QPlan q;
    PT_TRY(make_qplan(s, q));
    (void) n;
    dim3 grid((q.ew + TW - 1) / TW, q.eh);
    LearnedArgs none;
    memset(&none, 0, sizeof(none));
    k_choose_tile<false><<<grid, TW, sizeof(float4) * 8 * ATW, st>>>(q, a, b, cur_pos, cur_d, tcand, kcoh, do_table, ch_pos,
                                                                   ch_d, kc_done, use_done, evals, none);
    PT_LAUNCHED();
    return PT_OK;
}

pt_status pt_launch_choose_learned(const QuerySetup &s, const float4 *a, const float4 *b, const int *cur_pos,
                                   const float *cur_d, const int *tcand, const int2 *kcoh, int do_table, int *ch_pos,
                                   float *ch_d, int *kc_done, int use_done, const int *lcand, const float *lconf,
                                   float threshold, int kcoh_confident, unsigned long long *evals,
                                   unsigned long long *lcounters, cudaStream_t st) {
    QPlan q;
    PT_TRY(make_qplan(s, q));
    if (!lconf) return pt_fail(PT_BAD_ARG, "learned choose without confidences");
    LearnedArgs la;
    la.cand = lcand;
    la.conf = lconf;
    la.threshold = threshold;
    la.kcoh_confident = kcoh_confident;
    la.counters = lcounters;
    dim3 grid((q.ew + TW - 1) / TW, q.eh);
    k_choose_tile<true><<<grid, TW, sizeof(float4) * 8 * ATW, st>>>(q, a, b, cur_pos, cur_d, tcand, kcoh, do_table, ch_pos,
                                                                  ch_d, kc_done, use_done, evals, la);
    PT_LAUNCHED();
    return PT_OK;
}

pt_status pt_launch_pull(const QuerySetup &s, int n, const float4 *a, const float4 *b, const int *cur_pos, const float *cur_d,
                         const int *ch_pos, const float *ch_d, int *nxt_pos, float *nxt_d,
                         unsigned long long *evals, cudaStream_t st) {
    QPlan q;
    PT_TRY(make_qplan(s, q));
    (void) n;
    dim3 grid((q.ew + TW - 1) / TW, q.eh);
    if (q.radius <= 1)
        k_pull_tile<1><<<grid, TW, sizeof(float4) * 8 * ATW, st>>>(q, a, b, cur_pos, cur_d, ch_pos, ch_d, nxt_pos, nxt_d, evals);
    else
        k_pull_tile<2><<<grid, TW, sizeof(float4) * 8 * ATW, st>>>(q, a, b, cur_pos, cur_d, ch_pos, ch_d, nxt_pos, nxt_d, evals);
    PT_LAUNCHED();
    return PT_OK;
}

pt_status pt_launch_output(int n, const int *pos, const float *d, double *ann, cudaStream_t st) {
    k_output<<<(n + NT - 1) / NT, NT, 0, st>>>(n, pos, d, ann);
    PT_LAUNCHED();
    return PT_OK;
}
