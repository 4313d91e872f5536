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

/* patch_dist_exact in the reference's order, abandoning the sum (returning +inf) as soon as the
   running total reaches `bound`. */
__device__ __forceinline__ float ssd_bounded(const float4 *__restrict__ A, int aw, int ax, int ay,
                                             const float4 *__restrict__ B, int bw, int bx, int by, float bound,
                                             unsigned &rows) {
    float l0 = 0.f, l1 = 0.f, l2 = 0.f, l3 = 0.f;
    for (int dy = 0; dy < 8; dy++) {
        rows++;
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
        if (dy < 7 && __fadd_rn(__fadd_rn(__fadd_rn(l0, l1), l2), l3) >= bound) return finf();
    }
    return __fadd_rn(__fadd_rn(__fadd_rn(l0, l1), l2), l3);
}

/* Adds per-thread counts to counters[0..1] with one atomic per warp (profiling only). */
__device__ __forceinline__ void count_work(unsigned long long *counters, unsigned cand, unsigned rows) {
    if (!counters) return;
    unsigned c = __reduce_add_sync(0xffffffffu, cand), r = __reduce_add_sync(0xffffffffu, rows);
    if ((threadIdx.x & 31) == 0) { atomicAdd(counters, (unsigned long long) c); atomicAdd(counters + 1, (unsigned long long) r); }
}

/* Steps 1-3 for every patch: returns the chosen match and its exact distance. */
__global__ void __launch_bounds__(NT)
k_choose(const QPlan c_q, const float4 *__restrict__ a, const float4 *__restrict__ b, const int *__restrict__ cur_pos,
         const float *__restrict__ cur_d, const int *__restrict__ tcand, const int2 *__restrict__ kcoh, int do_table,
         int *ch_pos, float *ch_d, int *kc_done, int use_done, unsigned long long *counters) {
    int p = blockIdx.x * NT + threadIdx.x;
    const bool live = p < c_q.ew * c_q.eh;
    unsigned ne = 0, rows = 0;
    if (live) {
    int x = p % c_q.ew, y = p / c_q.ew;
    int pos = cur_pos[p];
    float dstore = cur_d[p];
    int xb = pt_x(pos), yb = pt_y(pos);
    float dbest = (float) ((double) dstore * c_q.prop_scale);
    float dch = dstore;          /* exact distance of the chosen match */
    if (do_table) {
        int v = tcand[p];
        int xs = pt_x(v) - 7, ys = pt_y(v) - 7;
        if (xs != xb || ys != yb) {
            float dc = ssd_bounded(a, c_q.aw, x, y, b, c_q.bw, xs, ys, dbest, rows);
            ne++;
            if (dc < dbest) { dbest = dc; dch = dc; xb = xs; yb = ys; }
        }
    }
    /* kc_done[p] holds a position whose k-coherence set was already tried by this patch without
       any acceptance; with the same position the stored distance, the bound and therefore every
       outcome would repeat, so the set is skipped (an exact shortcut). */
    const int kc_src = pt_xy(xb, yb);
    const bool repeat = use_done && kc_done[p] == kc_src;
    bool accepted = false;
    if (c_q.do_kcoh && !repeat && xb < c_q.bew && yb < c_q.beh) {
        int ks = c_q.ks;
        /* kcoherence_set is beh x bew x kc even when ks > 1 (patchtable.h:2659, 3758). */
        const int2 *kp = kcoh + ((size_t) (yb / ks) * c_q.bew + (xb / ks)) * c_q.kc;
        int kdx = ks > 1 ? xb % ks : 0, kdy = ks > 1 ? yb % ks : 0;
        for (int k = 0; k < c_q.kc; k++) {
            int2 e = kp[k];
            float kd = __int_as_float(e.y);
            if ((double) kd >= c_q.triangle * (double) dbest) break;
            int xs = pt_x(e.x) + kdx, ys = pt_y(e.x) + kdy;
            if (xs >= c_q.bew) xs = c_q.bew - 1;
            if (ys >= c_q.beh) ys = c_q.beh - 1;
            float dc = ssd_bounded(a, c_q.aw, x, y, b, c_q.bw, xs, ys, dbest, rows);
            ne++;
            if (dc < dbest) { dbest = dc; dch = dc; xb = xs; yb = ys; accepted = true; }
        }
    }
    if (c_q.do_kcoh) kc_done[p] = (repeat || !accepted) ? kc_src : -1;
    ch_pos[p] = pt_xy(xb, yb);
    ch_d[p] = dch;
    }
    count_work(counters, ne, rows);
}

/* Step 4 as a pull: the best of the stored match and every neighbour's chosen offset applied
   to this patch.  Neighbours sit `step` patches apart; passes with decreasing steps (jump
   flooding) carry an offset across a region in a logarithmic number of passes, where the
   reference's sequential sweep carries it along a whole row in one sweep.  The patch's own choice is taken first (its exact distance is known), then the
   distinct neighbour candidates are evaluated row by row together, so each row of the query
   patch is loaded once for all of them.  Every candidate's sum keeps the reference's order, and
   candidates are accepted in neighbour order with a strict comparison, as a sequential loop
   would; a candidate stops as soon as its partial sum reaches the best distance known before
   the rows start. */
template<int R>
__device__ __forceinline__ void pull_patch(const QPlan &c_q, const float4 *__restrict__ a, const float4 *__restrict__ b,
                                           int x, int y, int &bpos, float &bd, const int *__restrict__ ch_pos,
                                           const float *__restrict__ ch_d, unsigned &ne, unsigned &rows) {
    constexpr int MAXC = (2 * R + 1) * (2 * R + 1) - 1;
    const int S = c_q.step;
    {
        int q = y * c_q.ew + x;
        int cp = ch_pos[q];
        if (pt_x(cp) < c_q.bew && pt_y(cp) < c_q.beh && cp != bpos && ch_d[q] < bd) { bd = ch_d[q]; bpos = cp; }
    }
    int cand[MAXC];
    int nc = 0;
#pragma unroll
    for (int dy = -R; dy <= R; dy++) {
#pragma unroll
        for (int dx = -R; dx <= R; dx++) {
            if (dx == 0 && dy == 0) continue;
            int ny = y + S * dy, nx = x + S * dx;
            if (ny < 0 || ny >= c_q.eh || nx < 0 || nx >= c_q.ew) continue;
            int cp = ch_pos[ny * c_q.ew + nx];
            int xs = pt_x(cp) - S * dx, ys = pt_y(cp) - S * dy;
            if (xs < 0 || ys < 0 || xs >= c_q.bew || ys >= c_q.beh) continue;
            int c = pt_xy(xs, ys);
            bool dup = c == bpos;
            for (int t = 0; t < nc; t++) dup |= cand[t] == c;
            if (!dup) cand[nc++] = c;
        }
    }
    if (nc == 0) return;
    ne += nc;
    float l[MAXC][4];
#pragma unroll
    for (int c = 0; c < MAXC; c++) { l[c][0] = l[c][1] = l[c][2] = l[c][3] = 0.f; }
    unsigned active = (1u << nc) - 1u;
    const float bound = bd;
    for (int dy = 0; dy < 8 && active; dy++) {
        const float4 *ar = a + (size_t) (y + dy) * c_q.aw + x;
        float4 av[8];
#pragma unroll
        for (int p = 0; p < 8; p++) av[p] = __ldg(ar + p);
#pragma unroll
        for (int c = 0; c < MAXC; c++) {
            if (!((active >> c) & 1u)) continue;
            rows++;
            const float4 *br = b + (size_t) (pt_y(cand[c]) + dy) * c_q.bw + pt_x(cand[c]);
            float e[24];
#pragma unroll
            for (int p = 0; p < 8; p++) {
                float4 bv = __ldg(br + p);
                float t0 = __fsub_rn(av[p].x, bv.x), t1 = __fsub_rn(av[p].y, bv.y), t2 = __fsub_rn(av[p].z, bv.z);
                e[3 * p] = __fmul_rn(t0, t0); e[3 * p + 1] = __fmul_rn(t1, t1); e[3 * p + 2] = __fmul_rn(t2, t2);
            }
#pragma unroll
            for (int n = 0; n < 6; n++) {
                l[c][0] = __fadd_rn(l[c][0], e[4 * n]); l[c][1] = __fadd_rn(l[c][1], e[4 * n + 1]);
                l[c][2] = __fadd_rn(l[c][2], e[4 * n + 2]); l[c][3] = __fadd_rn(l[c][3], e[4 * n + 3]);
            }
            if (dy < 7 && __fadd_rn(__fadd_rn(__fadd_rn(l[c][0], l[c][1]), l[c][2]), l[c][3]) >= bound) active &= ~(1u << c);
        }
    }
#pragma unroll
    for (int c = 0; c < MAXC; c++) {
        if (!((active >> c) & 1u)) continue;
        float d = __fadd_rn(__fadd_rn(__fadd_rn(l[c][0], l[c][1]), l[c][2]), l[c][3]);
        if (d < bd) { bd = d; bpos = cand[c]; }
    }
}

__global__ void __launch_bounds__(NT)
k_pull(const QPlan c_q, const float4 *__restrict__ a, const float4 *__restrict__ b, const int *__restrict__ cur_pos,
       const float *__restrict__ cur_d, const int *__restrict__ ch_pos, const float *__restrict__ ch_d,
       int *nxt_pos, float *nxt_d, unsigned long long *counters) {
    int p = blockIdx.x * NT + threadIdx.x;
    const bool live = p < c_q.ew * c_q.eh;
    unsigned ne = 0, rows = 0;
    if (live) {
        int x = p % c_q.ew, y = p / c_q.ew;
        int bpos = cur_pos[p];
        float bd = cur_d[p];
        if (c_q.radius <= 1) pull_patch<1>(c_q, a, b, x, y, bpos, bd, ch_pos, ch_d, ne, rows);
        else pull_patch<2>(c_q, a, b, x, y, bpos, bd, ch_pos, ch_d, ne, rows);
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
    k_choose<<<(n + NT - 1) / NT, NT, 0, st>>>(q, a, b, cur_pos, cur_d, tcand, kcoh, do_table, ch_pos, ch_d, kc_done, use_done, evals);
    PT_LAUNCHED();
    return PT_OK;
}

pt_status pt_launch_pull(const QuerySetup &s, int n, const float4 *a, const float4 *b, const int *cur_pos, const float *cur_d,
                         const int *ch_pos, const float *ch_d, int *nxt_pos, float *nxt_d,
                         unsigned long long *evals, cudaStream_t st) {
    QPlan q;
    PT_TRY(make_qplan(s, q));
    k_pull<<<(n + NT - 1) / NT, NT, 0, st>>>(q, a, b, cur_pos, cur_d, ch_pos, ch_d, nxt_pos, nxt_d, evals);
    PT_LAUNCHED();
    return PT_OK;
}

pt_status pt_launch_output(int n, const int *pos, const float *d, double *ann, cudaStream_t st) {
    k_output<<<(n + NT - 1) / NT, NT, 0, st>>>(n, pos, d, ann);
    PT_LAUNCHED();
    return PT_OK;
}
