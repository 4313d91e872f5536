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

#include <atomic>
#include <cstring>

#include "pt_internal.h"
#include "pt_descdist.cuh"
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
    int kc, ks;              /* kcoherence (entries per cell), kcoherence_step */
    int kc_try;              /* entries tried per patch (<= kc) */
    int radius;              /* query_step + prop_dist */
    int do_kcoh;
    int step;                /* neighbour spacing of this pull pass (jump flooding) */
    int pull_max;            /* most neighbour candidates scored per patch */
    int tile;                /* query patches per CTA (single-image launches) */
    int row0, rows;          /* patch rows of a single-image launch */
    const float4 *b1;        /* b shifted by one pixel: b1[i] = b[i + 1] */
    const int *allowed;      /* b patches that may be matched (allowed[p] == allowed_index), or NULL */
    int allowed_index;
    const float4 *adesc;     /* descriptor mode: query descriptor store (ds4 float4 per patch), or NULL */
    const float4 *bdesc;     /* descriptor mode: table descriptor store */
    int ds4, nd;             /* float4 per store entry, descriptor dimensions */
    const int *tcand_more;   /* further tables' entries, [table][patch] (ntables > 1), or NULL */
    int ntc;
    int spatial, do_rs, pass; /* spatial search radius, random search, pass index (its seed) */
    double *ann;             /* last pull: the float64 NNF written directly, or NULL */
};

/* lowbias32 integer hash (C. Wellons' published constants): the random search's choice of
   neighbour for a patch in a pass, in place of the reference's sequential rand() stream. */
__device__ __forceinline__ unsigned mix32(unsigned x) {
    x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
    return x;
}

__device__ __forceinline__ float finf() { return __int_as_float(0x7f800000); }

/* Adds per-thread counts to counters[0..1] with one atomic per warp (profiling only). */
__device__ __forceinline__ void count_work(unsigned long long *counters, unsigned cand, unsigned rows) {
    if (!counters) return;
    unsigned c = __reduce_add_sync(0xffffffffu, cand), r = __reduce_add_sync(0xffffffffu, rows);
    if ((threadIdx.x & 31) == 0) { atomicAdd(counters, (unsigned long long) c); atomicAdd(counters + 1, (unsigned long long) r); }
}

constexpr int TWD = 32;                   /* query patches per CTA row segment when none is chosen */
/* Threads per SM the register caps of the lean choose and the one-candidate pull leave room for.
   Both compile to 56 registers under these caps; tighter caps (20 x 64 or 24 x 64 threads per
   SM: 48 or 40 registers, no spills) measured 1-3 % slower at 1080p. */
constexpr int CHOOSE_LEAN_LANES = 12 * 64;
constexpr int PULL_ONE_LANES = 16 * 64;
constexpr int TWD_DESC = 64;              /* query patches per CTA in descriptor mode */

/* Stages the 8 pixel rows under a CTA's row segment of TW query patches in shared memory
   (TW + 7 pixels per row) as packed RGB, 3 floats per pixel: a lane reading channel c of its 8
   pixels touches word 3 * pixel + c, so each warp-wide 4-byte load hits 32 distinct banks in one
   wavefront, and a row costs 24 wavefronts instead of the 32 of 16-byte RGBA loads. */
template<int TW>
__device__ __forceinline__ void stage_a(float4 *atile, const float4 *__restrict__ a, int aw, int ah, int x0, int y) {
    constexpr int ATW = TW + 7;
    float *at = reinterpret_cast<float *>(atile);
    for (int i = threadIdx.x; i < 8 * ATW; i += TW) {
        int r = i / ATW, c = i - r * ATW;
        int gx = x0 + c, gy = y + r;
        const float4 v = (gx < aw && gy < ah) ? __ldg(a + (size_t) gy * aw + gx) : make_float4(0.f, 0.f, 0.f, 0.f);
        at[3 * i] = v.x;
        at[3 * i + 1] = v.y;
        at[3 * i + 2] = v.z;
    }
}

/* Shared-memory bytes of a staged query tile of TW patches. */
constexpr size_t atile_bytes(int TW) { return sizeof(float) * 3 * 8 * (TW + 7); }

/* Query row dy of the patch at tile column tx. */
template<int TW>
__device__ __forceinline__ void load_arow(const float4 *atile, int dy, int tx, float4 (&av)[8]) {
    const float *at = reinterpret_cast<const float *>(atile) + 3 * (dy * (TW + 7) + tx);
#pragma unroll
    for (int p = 0; p < 8; p++) av[p] = make_float4(at[3 * p], at[3 * p + 1], at[3 * p + 2], 0.f);
}

/* One 32-byte read-only load: pixels p[0], p[1]. */
__device__ __forceinline__ void ld_px2(const float4 *p, float4 &u, float4 &v) {
    asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(u.x), "=f"(u.y), "=f"(u.z), "=f"(u.w), "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
        : "l"(p));
}

/* The 8 pixels (x..x+7, y) of b with four 32-byte loads: pixel index i = y*bw + x is read from b
   when even and from the shifted copy b1 (b1[i-1] = b[i]) when odd, so every load starts on a
   32-byte boundary (both arrays are 256-byte aligned). */
__device__ __forceinline__ void load_brow(const QPlan &q, const float4 *__restrict__ B, int x, int y, float4 (&bv)[8]) {
    const size_t i = (size_t) y * q.bw + x;
    const float4 *src = (i & 1) ? q.b1 + (i - 1) : B + i;
#pragma unroll
    for (int j = 0; j < 4; j++) ld_px2(src + 2 * j, bv[2 * j], bv[2 * j + 1]);
}

/* Adds one patch row to the four SSE-lane sums of patch_dist_exact (patchtable.h:349-356): the
   interleaved RGB float e = 3p + c goes to lane e & 3, in increasing e per lane. */
__device__ __forceinline__ void row_lanes(const float4 (&av)[8], const float4 (&bv)[8], float (&l)[4]) {
#pragma unroll
    for (int p = 0; p < 8; p++) {
        const float t0 = __fsub_rn(av[p].x, bv[p].x), t1 = __fsub_rn(av[p].y, bv[p].y), t2 = __fsub_rn(av[p].z, bv[p].z);
        const float qd[3] = {__fmul_rn(t0, t0), __fmul_rn(t1, t1), __fmul_rn(t2, t2)};
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const int e = (3 * p + c) & 3;
            l[e] = __fadd_rn(l[e], qd[c]);
        }
    }
}

__device__ __forceinline__ float lane_total(const float (&l)[4]) {
    return __fadd_rn(__fadd_rn(__fadd_rn(l[0], l[1]), l[2]), l[3]);
}

/* patch_dist_exact with the query patch in shared memory; abandons the sum once a row's partial
   total reaches `bound` (+inf returned). */
template<int TW>
__device__ __forceinline__ float ssd_tile(const float4 *atile, int tx, const QPlan &q, const float4 *__restrict__ B,
                                          int bx, int by, float bound, unsigned &rows) {
    float l[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 1
    for (int dy = 0; dy < 8; dy++) {
        rows++;
        float4 av[8], bv[8];
        load_brow(q, B, bx, by + dy, bv);
        load_arow<TW>(atile, dy, tx, av);
        row_lanes(av, bv, l);
        if (dy < 7 && lane_total(l) >= bound) return finf();
    }
    return lane_total(l);
}

/* Up to G candidates' sums advanced together row by row, so each query row is read from shared
   memory once per group; candidate g takes part when bit g of `valid` is set.  Each sum keeps the
   reference's lane order and stops once its partial total reaches `bound`.  out[g] = the full sum,
   or +inf when stopped or not taking part. */
template<int TW, int G>
__device__ __forceinline__ void ssd_group(const float4 *atile, int tx, const QPlan &q, const float4 *__restrict__ B,
                                          const int (&cand)[G], unsigned valid, float bound, float (&out)[G],
                                          unsigned &rows) {
    float l[G][4];
    bool live[G];
#pragma unroll
    for (int g = 0; g < G; g++) { l[g][0] = l[g][1] = l[g][2] = l[g][3] = 0.f; live[g] = (valid >> g) & 1; }
#pragma unroll 1
    for (int dy = 0; dy < 8; dy++) {
        bool any = false;
#pragma unroll
        for (int g = 0; g < G; g++) any |= live[g];
        if (!any) break;
        float4 av[8];
        load_arow<TW>(atile, dy, tx, av);
#pragma unroll
        for (int g = 0; g < G; g++) {
            if (!live[g]) continue;
            rows++;
            float4 bv[8];
            load_brow(q, B, pt_x(cand[g]), pt_y(cand[g]) + dy, bv);
            row_lanes(av, bv, l[g]);
            if (dy < 7 && lane_total(l[g]) >= bound) live[g] = false;
        }
    }
#pragma unroll
    for (int g = 0; g < G; g++) out[g] = live[g] ? lane_total(l[g]) : finf();
}

/* The query patch a distance is taken from: its RGB rows staged in shared memory (image mode) or
   its descriptor in registers (descriptor mode, DESC instantiations). */
struct AQuery {
    const float4 *atile;
    int tx;
    float4 v[4];
};

/* One candidate's distance: patch_dist_exact (image mode, abandoned at `bound`) or
   patch_dist_approx of the descriptors (descriptor mode, always complete: a complete sum at or
   above the bound is rejected by the caller exactly as an abandoned one). */
template<int TW, bool DESC>
__device__ __forceinline__ float dist1(const AQuery &aq, const QPlan &q, const float4 *__restrict__ B, int bx, int by,
                                       float bound, unsigned &rows) {
    if constexpr (DESC) {
        rows++;
        return pt_desc_dist(aq.v, q.bdesc + ((size_t) by * q.bew + bx) * q.ds4, q.nd);
    } else {
        return ssd_tile<TW>(aq.atile, aq.tx, q, B, bx, by, bound, rows);
    }
}

template<int TW, int G, bool DESC>
__device__ __forceinline__ void dist_group(const AQuery &aq, const QPlan &q, const float4 *__restrict__ B,
                                           const int (&cand)[G], unsigned valid, float bound, float (&out)[G],
                                           unsigned &rows) {
    if constexpr (DESC) {
#pragma unroll
        for (int g = 0; g < G; g++) {
            out[g] = finf();
            if ((valid >> g) & 1) {
                rows++;
                out[g] = pt_desc_dist(aq.v, q.bdesc + ((size_t) pt_y(cand[g]) * q.bew + pt_x(cand[g])) * q.ds4, q.nd);
            }
        }
    } else {
        ssd_group<TW, G>(aq.atile, aq.tx, q, B, cand, valid, bound, out, rows);
    }
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
/* LEAN: the table step only (no further tables, k-coherence, spatial or random search), so the
   registers those steps need are not reserved. */
template<int TW, bool LEARNED, bool DESC, bool LEAN = false>
__device__ __forceinline__ void
choose_seg(const QPlan &c_q, float4 *atile, const float4 *__restrict__ a, const float4 *__restrict__ b,
           const int *__restrict__ cur_pos, const float *__restrict__ cur_d, const int *__restrict__ tcand,
           const int2 *__restrict__ kcoh, int do_table, int *ch_pos, float *ch_d, int *kc_done, int use_done,
           unsigned long long *counters, const LearnedArgs &la, int x0, int y) {
    if constexpr (!DESC) {
        stage_a<TW>(atile, a, c_q.aw, c_q.ah, x0, y);
        __syncthreads();
    }
    const int x = x0 + threadIdx.x;
    const bool live = x < c_q.ew;
    unsigned ne = 0, rows = 0, n_conf = 0, n_prop = 0;
    if (live) {
        const int p = y * c_q.ew + x;
        AQuery aq;
        aq.atile = atile;
        aq.tx = threadIdx.x;
        if constexpr (DESC) pt_desc_load(c_q.adesc + (size_t) p * c_q.ds4, 4 * c_q.ds4, aq.v);
        /* no state arrays: the initial field, x = b's ew + 1 and DIST_INFINITY (patchtable.h:3538-3547) */
        int pos = cur_pos ? cur_pos[p] : pt_xy(c_q.bew + 1, 0);
        float dstore = cur_d ? cur_d[p] : (float) PT_DIST_INF;
        int xb = pt_x(pos), yb = pt_y(pos);
        float dbest = (float) ((double) dstore * c_q.prop_scale);
        float dch = dstore;
        bool confident = false;
        if (LEARNED) confident = la.conf[p] >= la.threshold;
        if (LEARNED && confident && do_table && la.cand) {
            /* the proposals in the network's order, repeats dropped, three at a time */
            const int4 *cp = reinterpret_cast<const int4 *>(la.cand + (size_t) p * PT_PROP_TOPK);
            const int4 c0 = cp[0], c1 = cp[1];
            const int raw[PT_PROP_TOPK] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
            int cand[PT_PROP_TOPK + 1];
            unsigned keep = 0;
            const int own = pt_xy(xb, yb);
#pragma unroll
            for (int j = 0; j < PT_PROP_TOPK; j++) {
                const int px = pt_x(raw[j]) - 7, py = pt_y(raw[j]) - 7;
                const bool in_b = raw[j] >= 0 && px >= 0 && py >= 0 && px < c_q.bew && py < c_q.beh;
                cand[j] = in_b ? pt_xy(px, py) : -1;
                bool dup = !in_b || cand[j] == own;
#pragma unroll
                for (int t = 0; t < j; t++) dup |= ((keep >> t) & 1) && cand[t] == cand[j];
                if (!dup) keep |= 1u << j;
            }
            cand[PT_PROP_TOPK] = -1;
            constexpr int G = 3;
#pragma unroll
            for (int g0 = 0; g0 < PT_PROP_TOPK; g0 += G) {
                const unsigned m = (keep >> g0) & ((1u << G) - 1);
                if (!m) continue;
                const int cg[G] = {cand[g0], cand[g0 + 1], g0 + 2 <= PT_PROP_TOPK ? cand[g0 + 2] : -1};
                float d[G];
                dist_group<TW, G, DESC>(aq, c_q, b, cg, m, dbest, d, rows);
#pragma unroll
                for (int g = 0; g < G; g++)
                    if (((m >> g) & 1) && d[g] < dbest) { dbest = d[g]; dch = d[g]; xb = pt_x(cg[g]); yb = pt_y(cg[g]); }
            }
            n_prop = __popc(keep);
            ne += n_prop;
            n_conf = 1;
        } else if (do_table) {
            int v = tcand[p];
            int xs = pt_x(v) - 7, ys = pt_y(v) - 7;
            /* a table built here only holds patches of b; the range test guards against a corrupt
               table file or entry array, which must not make the kernel read outside b */
            const bool in_b = xs >= 0 && ys >= 0 && xs < c_q.bew && ys < c_q.beh;
            if (in_b && (xs != xb || ys != yb)) {
                float dc = dist1<TW, DESC>(aq, c_q, b, xs, ys, dbest, rows);
                ne++;
                if (dc < dbest) { dbest = dc; dch = dc; xb = xs; yb = ys; }
            }
            /* Further tables (patchtable.h:3711-3735): each entry is scored unless it equals the
               best so far or the previous table's entry. */
            const size_t np = (size_t) c_q.ew * c_q.eh;
            for (int k = 0; k < (LEAN ? 0 : c_q.ntc); k++) {
                const int v1 = c_q.tcand_more[(size_t) k * np + p];
                const int xs1 = pt_x(v1) - 7, ys1 = pt_y(v1) - 7;
                const bool in_b1 = xs1 >= 0 && ys1 >= 0 && xs1 < c_q.bew && ys1 < c_q.beh;
                if (in_b1 && (xs1 != xb || ys1 != yb) && (xs1 != xs || ys1 != ys)) {
                    float dc = dist1<TW, DESC>(aq, c_q, b, xs1, ys1, dbest, rows);
                    ne++;
                    if (dc < dbest) { dbest = dc; dch = dc; xb = xs1; yb = ys1; }
                }
                xs = xs1;
                ys = ys1;
            }
        }
        const int kc_src = pt_xy(xb, yb);
        const bool repeat = use_done && kc_done[p] == kc_src;
        bool accepted = false;
        const bool kc_here = !LEARNED || !confident || la.kcoh_confident;
        if (!LEAN && c_q.do_kcoh && kc_here && !repeat && xb < c_q.bew && yb < c_q.beh) {
            /* The reference tries the list in order and stops at the first neighbour whose stored
               distance reaches triangle * best.  Here two neighbours are scored together with the
               best known before the group as the early-exit bound, then the sequential decisions
               are replayed: a sum cut short by that looser bound could not have been accepted, and
               one that completes is exact, so the outcome equals the one-by-one loop. */
            const int ks = c_q.ks;
            const int2 *kp = kcoh + ((size_t) (yb / ks) * c_q.bew + (xb / ks)) * c_q.kc;
            const int kdx = ks > 1 ? xb % ks : 0, kdy = ks > 1 ? yb % ks : 0;
            constexpr int G = 2;             /* -speed presets list 2 to 20 neighbours; pairs keep registers low */
            bool done = false;
            for (int k = 0; k < c_q.kc_try && !done; k += G) {
                int cg[G];
                float kdg[G];
                unsigned m = 0;
#pragma unroll
                for (int j = 0; j < G; j++) {
                    cg[j] = 0;
                    kdg[j] = 0.f;
                    if (m == (1u << j) - 1 && k + j < c_q.kc_try) {
                        const int2 e = kp[k + j];
                        const float kd = __int_as_float(e.y);
                        if ((double) kd < c_q.triangle * (double) dbest) {
                            int xs = pt_x(e.x) + kdx, ys = pt_y(e.x) + kdy;
                            if (xs >= c_q.bew) xs = c_q.bew - 1;
                            if (ys >= c_q.beh) ys = c_q.beh - 1;
                            cg[j] = pt_xy(xs, ys);
                            kdg[j] = kd;
                            m |= 1u << j;
                        }
                    }
                }
                if (m != (1u << G) - 1) done = true;     /* the list ends or stops inside this group */
                if (!m) break;
                float d[G];
                dist_group<TW, G, DESC>(aq, c_q, b, cg, m, dbest, d, rows);
                ne += __popc(m);
#pragma unroll
                for (int j = 0; j < G; j++) {
                    if (!((m >> j) & 1)) continue;
                    if ((double) kdg[j] >= c_q.triangle * (double) dbest) { done = true; break; }
                    if (d[j] < dbest) { dbest = d[j]; dch = d[j]; xb = pt_x(cg[j]); yb = pt_y(cg[j]); accepted = true; }
                }
            }
        }
        if (!LEAN && c_q.do_kcoh) kc_done[p] = (repeat || !accepted) ? kc_src : -1;
        const bool have = xb < c_q.bew && yb < c_q.beh;
        if (!LEAN && c_q.spatial > 0 && have) {
            /* Spatial search (patchtable.h:3855-3873): every other patch of the (2s+1)^2 window
               around the best match, rows then columns, scored in pairs and replayed in order. */
            const int S = c_q.spatial, xb0 = xb, yb0 = yb;
            int symin = yb0 - S, symax = yb0 + S + 1, sxmin = xb0 - S, sxmax = xb0 + S + 1;
            if (symin < 0) symin = 0; else if (symax > c_q.beh) symax = c_q.beh;
            if (sxmin < 0) sxmin = 0; else if (sxmax > c_q.bew) sxmax = c_q.bew;
            if (symax > c_q.beh) symax = c_q.beh;          /* windows wider than b */
            if (sxmax > c_q.bew) sxmax = c_q.bew;
            const int swd = sxmax - sxmin, nwin = (symax - symin) * swd;
            constexpr int G = 2;
            for (int i0 = 0; i0 < nwin; i0 += G) {
                int cg[G];
                unsigned m = 0;
#pragma unroll
                for (int j = 0; j < G; j++) {
                    cg[j] = 0;
                    const int i = i0 + j;
                    if (i >= nwin) continue;
                    const int ys = symin + i / swd, xs = sxmin + i % swd;
                    if (xs == xb0 && ys == yb0) continue;
                    if (c_q.allowed && __ldg(c_q.allowed + (size_t) ys * c_q.bew + xs) != c_q.allowed_index) continue;
                    cg[j] = pt_xy(xs, ys);
                    m |= 1u << j;
                }
                if (!m) continue;
                float d[G];
                dist_group<TW, G, DESC>(aq, c_q, b, cg, m, dbest, d, rows);
                ne += __popc(m);
#pragma unroll
                for (int j = 0; j < G; j++)
                    if (((m >> j) & 1) && d[j] < dbest) { dbest = d[j]; dch = d[j]; xb = pt_x(cg[j]); yb = pt_y(cg[j]); }
            }
        } else if (!LEAN && c_q.do_rs && have) {
            /* Random search (patchtable.h:3874-3903): one of the 8 neighbours of the best match.
               dx, dy + 1 for r = 0..7 are packed two bits each: {-1,0,1,-1,1,-1,0,1},
               {-1,-1,-1,0,0,1,1,1}. */
            const unsigned r = mix32((unsigned) p * 2654435761u + (unsigned) c_q.pass * 0x9e3779b9u + 0x6a09e667u) & 7u;
            const int xs = xb + (int) ((37412u >> (2 * r)) & 3u) - 1, ys = yb + (int) ((43328u >> (2 * r)) & 3u) - 1;
            if (xs >= 0 && xs < c_q.bew && ys >= 0 && ys < c_q.beh &&
                (!c_q.allowed || __ldg(c_q.allowed + (size_t) ys * c_q.bew + xs) == c_q.allowed_index)) {
                const float dc = dist1<TW, DESC>(aq, c_q, b, xs, ys, dbest, rows);
                ne++;
                if (dc < dbest) { dbest = dc; dch = dc; xb = xs; yb = ys; }
            }
        }
        ch_pos[p] = pt_xy(xb, yb);
        ch_d[p] = dch;
    }
    count_work(counters, ne, rows);
    if (LEARNED && la.counters) {
        unsigned c = __reduce_add_sync(0xffffffffu, n_conf), q = __reduce_add_sync(0xffffffffu, n_prop);
        if ((threadIdx.x & 31) == 0) { atomicAdd(la.counters, (unsigned long long) c); atomicAdd(la.counters + 1, (unsigned long long) q); }
    }
}

/* At least 10 x 64 threads' worth of CTAs per SM: the register budget this leaves keeps the gather
   latency hidden without the spills of tighter caps (measured at 1080p, 64 patches per CTA:
   choose 0.70 ms unrestricted, 0.611 at 10 x 64, 0.619 at 12 x 64, 0.625 at 16 x 64). */
template<int TW, bool LEARNED, bool DESC, bool LEAN = false>
__global__ void __launch_bounds__(TW, (LEAN ? CHOOSE_LEAN_LANES : 10 * 64) / TW)
k_choose_tile(const QPlan c_q, const float4 *__restrict__ a, const float4 *__restrict__ b, const int *__restrict__ cur_pos,
              const float *__restrict__ cur_d, const int *__restrict__ tcand, const int2 *__restrict__ kcoh, int do_table,
              int *ch_pos, float *ch_d, int *kc_done, int use_done, unsigned long long *counters, const LearnedArgs la) {
    extern __shared__ float4 atile[];
    choose_seg<TW, LEARNED, DESC, LEAN>(c_q, atile, a, b, cur_pos, cur_d, tcand, kcoh, do_table, ch_pos, ch_d, kc_done,
                                        use_done, counters, la, blockIdx.x * TW, blockIdx.y + c_q.row0);
}

/* Step 4 as a pull: the best of the stored match and every neighbour's chosen offset applied to
   this patch.  The patch's own choice comes first; the distinct neighbour candidates follow in
   increasing order of the distance their neighbour achieved with them (the likeliest good ones
   first, so the running best -- the early-exit bound -- tightens soonest), three at a time.
   Neighbours sit `step` patches apart; passes with decreasing steps (jump flooding) carry an
   offset across a region in a logarithmic number of passes, where the reference's sequential
   sweep carries it along a whole row in one sweep. */
/* ONE: a single neighbour candidate per patch (pull_max 1).  The candidate is the one the
   general path would sort first -- among distinct candidates keyed by their first occurrence, the
   smallest key, the earliest on ties -- found in one streaming pass, and it is scored alone. */
template<int TW, int R, bool DESC, bool ONE = false>
__device__ __forceinline__ void
pull_seg(const QPlan &c_q, float4 *atile, const float4 *__restrict__ a, const float4 *__restrict__ b,
         const int *__restrict__ cur_pos, const float *__restrict__ cur_d, const int *__restrict__ ch_pos,
         const float *__restrict__ ch_d, int *nxt_pos, float *nxt_d, unsigned long long *counters, int x0, int y) {
    if constexpr (!DESC) {
        stage_a<TW>(atile, a, c_q.aw, c_q.ah, x0, y);
        __syncthreads();
    }
    const int x = x0 + threadIdx.x;
    const bool live = x < c_q.ew;
    unsigned ne = 0, rows = 0;
    if (live) {
        const int p = y * c_q.ew + x;
        AQuery aq;
        aq.atile = atile;
        aq.tx = threadIdx.x;
        if constexpr (DESC) pt_desc_load(c_q.adesc + (size_t) p * c_q.ds4, 4 * c_q.ds4, aq.v);
        int bpos = cur_pos ? cur_pos[p] : pt_xy(c_q.bew + 1, 0);      /* null: the initial field */
        float bd = cur_d ? cur_d[p] : (float) PT_DIST_INF;
        {
            int cp = ch_pos[p];
            if (pt_x(cp) < c_q.bew && pt_y(cp) < c_q.beh && cp != bpos && ch_d[p] < bd) { bd = ch_d[p]; bpos = cp; }
        }
        constexpr int MAXC = (2 * R + 1) * (2 * R + 1) - 1;
        const int S = c_q.step;
        int nc = 0;
        if constexpr (ONE) {
            /* the distinct candidates seen so far, newest first (fixed register slots) */
            int seen[MAXC];
#pragma unroll
            for (int t = 0; t < MAXC; t++) seen[t] = -1;
            int best = -1;
            float bestk = finf();
#pragma unroll
            for (int dy = -R; dy <= R; dy++) {
#pragma unroll
                for (int dx = -R; dx <= R; dx++) {
                    if (dx == 0 && dy == 0) continue;
                    const int ny = y + S * dy, nx = x + S * dx;
                    if (ny < 0 || ny >= c_q.eh || nx < 0 || nx >= c_q.ew) continue;
                    const int q = ny * c_q.ew + nx;
                    const int cp = ch_pos[q];
                    const int xs = pt_x(cp) - S * dx, ys = pt_y(cp) - S * dy;
                    if (xs < 0 || ys < 0 || xs >= c_q.bew || ys >= c_q.beh) continue;
                    if (c_q.allowed && __ldg(c_q.allowed + (size_t) ys * c_q.bew + xs) != c_q.allowed_index) continue;
                    const int c = pt_xy(xs, ys);
                    bool dup = c == bpos;
#pragma unroll
                    for (int t = 0; t < MAXC; t++) dup |= seen[t] == c;
                    if (dup) continue;
#pragma unroll
                    for (int t = MAXC - 1; t > 0; t--) seen[t] = seen[t - 1];
                    seen[0] = c;
                    const float k = ch_d[q];
                    if (k < bestk) { bestk = k; best = c; }   /* the general sort's insertion rule */
                    nc++;
                }
            }
            nc = best >= 0 ? 1 : 0;
            if (nc) {
                const float d = dist1<TW, DESC>(aq, c_q, b, pt_x(best), pt_y(best), bd, rows);
                if (d < bd) { bd = d; bpos = best; }
            }
        } else {
        /* distinct neighbour candidates sorted by the neighbour's own distance (ties keep the
           neighbour order), kept in registers: every slot index is known at compile time */
        int cand[MAXC];
        float key[MAXC];
#pragma unroll
        for (int t = 0; t < MAXC; t++) { cand[t] = -1; key[t] = finf(); }
#pragma unroll
        for (int dy = -R; dy <= R; dy++) {
#pragma unroll
            for (int dx = -R; dx <= R; dx++) {
                if (dx == 0 && dy == 0) continue;
                const int ny = y + S * dy, nx = x + S * dx;
                if (ny < 0 || ny >= c_q.eh || nx < 0 || nx >= c_q.ew) continue;
                const int q = ny * c_q.ew + nx;
                const int cp = ch_pos[q];
                const int xs = pt_x(cp) - S * dx, ys = pt_y(cp) - S * dy;
                if (xs < 0 || ys < 0 || xs >= c_q.bew || ys >= c_q.beh) continue;
                if (c_q.allowed && __ldg(c_q.allowed + (size_t) ys * c_q.bew + xs) != c_q.allowed_index) continue;
                int c = pt_xy(xs, ys);
                bool dup = c == bpos;
#pragma unroll
                for (int t = 0; t < MAXC; t++) dup |= cand[t] == c;
                if (dup) continue;
                float k = ch_d[q];
#pragma unroll
                for (int t = 0; t < MAXC; t++) {
                    if (k < key[t]) {
                        const float tk = key[t]; key[t] = k; k = tk;
                        const int tc = cand[t]; cand[t] = c; c = tc;
                    }
                }
                nc++;
            }
        }
        if (nc > c_q.pull_max) nc = c_q.pull_max;   /* the best-first prefix of the list */
        constexpr int G = 3;
#pragma unroll
        for (int g0 = 0; g0 < MAXC; g0 += G) {
            if (g0 < nc) {
                const int cg[G] = {cand[g0], g0 + 1 < MAXC ? cand[g0 + 1] : -1, g0 + 2 < MAXC ? cand[g0 + 2] : -1};
                const int left = nc - g0;
                const unsigned m = left >= G ? (1u << G) - 1 : (1u << left) - 1;
                float d[G];
                dist_group<TW, G, DESC>(aq, c_q, b, cg, m, bd, d, rows);
#pragma unroll
                for (int g = 0; g < G; g++)
                    if (((m >> g) & 1) && d[g] < bd) { bd = d[g]; bpos = cg[g]; }
            }
        }
        }
        ne += nc;
        if (c_q.ann) {                          /* k_output fused: x, y, dist of the final field */
            double *o = c_q.ann + 3 * (size_t) p;
            o[0] = pt_x(bpos);
            o[1] = pt_y(bpos);
            o[2] = bd;
        } else {
            nxt_pos[p] = bpos;
            nxt_d[p] = bd;
        }
    }
    count_work(counters, ne, rows);
}

/* At most 14 x 64 threads' worth of CTAs per SM (73 registers, 10 bytes of spills): the pull is
   latency-bound, and the extra resident warps hide the gathers (measured at 1080p with one
   candidate per patch: 0.341 -> 0.286 ms; at 16 x 64 the spills grow to 200 bytes and it slows). */
template<int TW, int R, bool DESC, bool ONE = false>
__global__ void __launch_bounds__(TW, (ONE ? PULL_ONE_LANES : 14 * 64) / TW)
k_pull_tile(const QPlan c_q, const float4 *__restrict__ a, const float4 *__restrict__ b, const int *__restrict__ cur_pos,
            const float *__restrict__ cur_d, const int *__restrict__ ch_pos, const float *__restrict__ ch_d,
            int *nxt_pos, float *nxt_d, unsigned long long *counters) {
    extern __shared__ float4 atile[];
    pull_seg<TW, R, DESC, ONE>(c_q, atile, a, b, cur_pos, cur_d, ch_pos, ch_d, nxt_pos, nxt_d, counters, blockIdx.x * TW,
                               blockIdx.y + c_q.row0);
}

/* ---- batched queries: many images, one launch per phase over a flattened segment list ---- */

/* Index of the image that owns flattened segment s (segs[i] = first segment of image i). */
__device__ __forceinline__ int owner(const PtBatchImage *__restrict__ imgs, int n, long long s, int twi) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&imgs[mid].seg_off[twi]) <= s) lo = mid; else hi = mid - 1;
    }
    return lo;
}

/* Runs body(s) for the row segments this CTA takes from the launch's work counter (zeroed before
   the launch): segments go out in order, one at a time, to whichever CTA is free, so uneven
   segment costs cannot leave some CTAs with a longer share.  A CTA claims its next segment when it
   starts the current one and reads the claim only after it, so the counter's round trip overlaps
   the work. */
template<class Body>
__device__ __forceinline__ void for_each_segment(unsigned long long *work, long long nseg, Body &&body) {
    __shared__ long long s_next;
    if (threadIdx.x == 0) s_next = (long long) atomicAdd(work, 1ull);
    __syncthreads();
    long long s = s_next;
    while (s < nseg) {
        long long claim = 0;
        if (threadIdx.x == 0) claim = (long long) atomicAdd(work, 1ull);
        body(s);
        __syncthreads();                       /* every thread is done with s_next and the staged tile */
        if (threadIdx.x == 0) s_next = claim;
        __syncthreads();
        s = s_next;
    }
}

/* Persistent choose over every row segment of every image, handed out by a work counter. */
template<int TW, bool LEAN = false>
__global__ void __launch_bounds__(TW, (LEAN ? CHOOSE_LEAN_LANES : 10 * 64) / TW)
k_choose_batch(const QPlan base, const PtBatchImage *__restrict__ imgs, int n, long long nseg, int twi,
               const float4 *__restrict__ a, const float4 *__restrict__ b, const int *__restrict__ cur_pos,
               const float *__restrict__ cur_d, const int *__restrict__ tcand, const int2 *__restrict__ kcoh, int do_table,
               int *ch_pos, float *ch_d, int *kc_done, int use_done, unsigned long long *counters,
               unsigned long long *work) {
    extern __shared__ float4 atile[];
    LearnedArgs none;
    none.cand = nullptr; none.conf = nullptr; none.threshold = 0.f; none.kcoh_confident = 0; none.counters = nullptr;
    for_each_segment(work, nseg, [&](long long s) {
        const int i = owner(imgs, n, s, twi);
        const PtBatchImage &g = imgs[i];
        const long long ls = s - g.seg_off[twi];
        const int spr = (g.ew + TW - 1) / TW;
        const int y = (int) (ls / spr), x0 = (int) (ls % spr) * TW;
        QPlan q = base;
        q.aw = g.w; q.ah = g.h; q.ew = g.ew; q.eh = g.eh;
        const long long o = g.patch_off;
        choose_seg<TW, false, false, LEAN>(q, atile, a + g.pix_off, b, cur_pos ? cur_pos + o : nullptr,
                                           cur_d ? cur_d + o : nullptr, tcand + o, kcoh, do_table, ch_pos + o, ch_d + o,
                                           kc_done + o, use_done, counters, none, x0, y);
    });
}

template<int TW, int R, bool ONE = false>
__global__ void __launch_bounds__(TW, (ONE ? PULL_ONE_LANES : 14 * 64) / TW)
k_pull_batch(const QPlan base, const PtBatchImage *__restrict__ imgs, int n, long long nseg, int twi,
             const float4 *__restrict__ a, const float4 *__restrict__ b, const int *__restrict__ cur_pos,
             const float *__restrict__ cur_d, const int *__restrict__ ch_pos, const float *__restrict__ ch_d,
             int *nxt_pos, float *nxt_d, unsigned long long *counters, unsigned long long *work) {
    extern __shared__ float4 atile[];
    for_each_segment(work, nseg, [&](long long s) {
        const int i = owner(imgs, n, s, twi);
        const PtBatchImage &g = imgs[i];
        const long long ls = s - g.seg_off[twi];
        const int spr = (g.ew + TW - 1) / TW;
        const int y = (int) (ls / spr), x0 = (int) (ls % spr) * TW;
        QPlan q = base;
        q.aw = g.w; q.ah = g.h; q.ew = g.ew; q.eh = g.eh;
        const long long o = g.patch_off;
        if (base.ann) q.ann = base.ann + 3 * o;        /* last pass: this image's NNF records */
        pull_seg<TW, R, false, ONE>(q, atile, a + g.pix_off, b, cur_pos ? cur_pos + o : nullptr,
                                    cur_d ? cur_d + o : nullptr, ch_pos + o, ch_d + o, nxt_pos + o, nxt_d + o, counters, x0, y);
    });
}

/* patch_dist_exact of a patch of a (RGBA rows in global memory) and a patch of b, in the
   reference's lane order, without an early exit. */
__device__ __forceinline__ float ssd_global(const QPlan &q, const float4 *__restrict__ a, int ax, int ay,
                                           const float4 *__restrict__ B, int bx, int by) {
    float l[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 1
    for (int dy = 0; dy < 8; dy++) {
        float4 av[8], bv[8];
        load_brow(q, B, bx, by + dy, bv);
#pragma unroll
        for (int p = 0; p < 8; p++) av[p] = __ldg(a + (size_t) (ay + dy) * q.aw + ax + p);
        row_lanes(av, bv, l);
    }
    return lane_total(l);
}

/* Initial field from the previous frame's NNF (patchtable.h:3548-3585): its matches (clamped to
   the table image when sanitize is set) with either their distance recomputed and scaled by
   scale_sv[p] (when given) or temporal_scale, or the previous distance times temporal_scale.
   orig[p] keeps what the end of the lookup restores for a patch that kept this match and this
   distance (patchtable.h:4178-4193): the scaled distance divided by temporal_scale. */
__global__ void k_init_temporal(const QPlan q, const double *__restrict__ prev, const float *__restrict__ scale_sv,
                                int recalc, int sanitize, double temporal_scale, const float4 *__restrict__ a,
                                const float4 *__restrict__ B, int *cur_pos, float *cur_d, double *orig, int *bad) {
    const int p = blockIdx.x * NT + threadIdx.x;
    if (p >= q.ew * q.eh) return;
    const int x = p % q.ew, y = p / q.ew;
    int xs = (int) prev[3 * (size_t) p], ys = (int) prev[3 * (size_t) p + 1];
    if (xs < 0 || ys < 0 || xs >= q.bew || ys >= q.beh) {
        if (!sanitize) atomicExch(bad, 1);
        xs = min(max(xs, 0), q.bew - 1);
        ys = min(max(ys, 0), q.beh - 1);
    }
    double scaled;
    if (recalc) {
        float dcur;
        if (q.adesc) {
            float4 v[4];
            pt_desc_load(q.adesc + (size_t) p * q.ds4, 4 * q.ds4, v);
            dcur = pt_desc_dist(v, q.bdesc + ((size_t) ys * q.bew + xs) * q.ds4, q.nd);
        } else {
            dcur = ssd_global(q, a, x, y, B, xs, ys);
        }
        scaled = (double) dcur * (scale_sv ? (double) scale_sv[p] : temporal_scale);
    } else {
        scaled = prev[3 * (size_t) p + 2] * temporal_scale;
    }
    cur_pos[p] = pt_xy(xs, ys);
    cur_d[p] = (float) scaled;
    orig[p] = scaled / temporal_scale;
}

/* init_random (patchtable.h:3522-3537): a random match per patch with its distance; the match
   comes from a hash of the patch index instead of two rand() calls. */
__global__ void k_init_random(const QPlan q, const float4 *__restrict__ a, const float4 *__restrict__ B, int *cur_pos,
                              float *cur_d) {
    const int p = blockIdx.x * NT + threadIdx.x;
    if (p >= q.ew * q.eh) return;
    const int x = p % q.ew, y = p / q.ew;
    unsigned hsh = mix32((unsigned) p * 0x9e3779b1u + 0x85ebca6bu);
    const int xs = (int) (hsh % (unsigned) q.bew);
    hsh = mix32(hsh ^ 0x27d4eb2fu);
    const int ys = (int) (hsh % (unsigned) q.beh);
    float d;
    if (q.adesc) {
        float4 v[4];
        pt_desc_load(q.adesc + (size_t) p * q.ds4, 4 * q.ds4, v);
        d = pt_desc_dist(v, q.bdesc + ((size_t) ys * q.bew + xs) * q.ds4, q.nd);
    } else {
        d = ssd_global(q, a, x, y, B, xs, ys);
    }
    cur_pos[p] = pt_xy(xs, ys);
    cur_d[p] = d;
}

/* The float64 NNF; a patch whose match and distance are still the initial temporal ones gets the
   unscaled distance back (patchtable.h:4178-4193). */
__global__ void k_output_temporal(int n, const int *__restrict__ pos, const float *__restrict__ d,
                                  const int *__restrict__ pos0, const float *__restrict__ d0,
                                  const double *__restrict__ orig, double *ann) {
    const int p = blockIdx.x * NT + threadIdx.x;
    if (p >= n) return;
    const int v = pos[p];
    ann[3 * (size_t) p + 0] = pt_x(v);
    ann[3 * (size_t) p + 1] = pt_y(v);
    ann[3 * (size_t) p + 2] = (v == pos0[p] && d[p] == d0[p]) ? orig[p] : (double) d[p];
}

__global__ void k_init(int n, int pos, float d, int *cur_pos, float *cur_d) {
    int p = blockIdx.x * NT + threadIdx.x;
    if (p < n) { cur_pos[p] = pos; cur_d[p] = d; }
}

/* The packed form of a float64 NNF whose distances are float values (every lookup but the
   temporal one): position x | y << 16 and the float distance, both exact. */
__global__ void k_pack_nnf(long long n, const double *__restrict__ ann, int *pos, float *d) {
    const long long p = blockIdx.x * (long long) NT + threadIdx.x;
    if (p >= n) return;
    pos[p] = pt_xy((int) ann[3 * p], (int) ann[3 * p + 1]);
    d[p] = (float) ann[3 * p + 2];
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

namespace {

std::atomic<int> g_lean_kernels{1};

/* The specialised variants apply: the choose of a pass with only the table step, the pull of a
   schedule with one neighbour candidate (image mode; descriptor mode keeps the general kernels). */
bool lean_choose(const QPlan &q) {
    return g_lean_kernels.load(std::memory_order_relaxed) && !q.adesc && !q.do_kcoh && q.ntc == 0 && q.spatial == 0 &&
           !q.do_rs;
}
bool one_pull(const QPlan &q) { return g_lean_kernels.load(std::memory_order_relaxed) && !q.adesc && q.pull_max == 1; }

}  // namespace

extern "C" int pt_set_lean_kernels(int on) { return g_lean_kernels.exchange(on ? 1 : 0); }

static pt_status make_qplan(const QuerySetup &s, QPlan &q) {
    memset(&q, 0, sizeof(q));
    q.aw = s.aw; q.ah = s.ah; q.ew = s.aw - 7; q.eh = s.ah - 7;
    q.bw = s.bw; q.bh = s.bh; q.bew = s.bw - 7; q.beh = s.bh - 7;
    q.prop_scale = s.prop_scale;
    q.triangle = s.triangle_factor;
    q.kc = s.kcoherence;
    q.kc_try = (s.kc_try > 0 && s.kc_try < s.kcoherence) ? s.kc_try : s.kcoherence;
    q.ks = s.kcoherence_step;
    q.radius = s.radius;
    q.do_kcoh = s.kcoherence > 0;
    q.step = s.step < 1 ? 1 : s.step;
    q.pull_max = s.pull_max > 0 ? s.pull_max : 1 << 30;
    q.tile = s.tile > 0 ? s.tile : TWD;
    q.row0 = s.rows > 0 ? s.row0 : 0;
    q.rows = s.rows > 0 ? s.rows : q.eh;
    if (s.rows > 0 && (q.row0 < 0 || q.row0 + q.rows > q.eh))
        return pt_fail(PT_BAD_ARG, "query rows [%d, %d) outside 0..%d", q.row0, q.row0 + q.rows, q.eh);
    if (q.tile != 32 && q.tile != 64 && q.tile != 128 && q.tile != 256)
        return pt_fail(PT_BAD_ARG, "gpu_tile %d: query patches per CTA must be 32, 64, 128 or 256", s.tile);
    q.b1 = s.b1;
    q.allowed = s.allowed;
    q.allowed_index = s.allowed_index;
    q.adesc = reinterpret_cast<const float4 *>(s.adesc);
    q.bdesc = reinterpret_cast<const float4 *>(s.bdesc);
    q.ds4 = s.ds / 4;
    q.nd = s.nd;
    q.tcand_more = s.ntcand_more > 0 ? s.tcand_more : nullptr;
    q.ntc = q.tcand_more ? s.ntcand_more : 0;
    q.spatial = s.spatial > 0 ? s.spatial : 0;
    q.do_rs = s.do_rs;
    q.pass = s.pass;
    q.ann = s.ann;
    if (q.adesc) {
        if (!q.bdesc || (s.ds != 8 && s.ds != 16) || q.nd < 3 || q.nd > s.ds)
            return pt_fail(PT_BAD_ARG, "descriptor query: store of %d floats for %d dimensions", s.ds, q.nd);
    } else if (!q.b1) {
        return pt_fail(PT_BAD_ARG, "query without the shifted copy of the table image");
    }
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
    LearnedArgs none;
    memset(&none, 0, sizeof(none));
    if (q.adesc) {                       /* descriptor mode: one tile width, nothing staged */
        constexpr int T = TWD_DESC;
        dim3 grid((q.ew + T - 1) / T, q.rows);
        k_choose_tile<T, false, true><<<grid, T, 0, st>>>(q, a, b, cur_pos, cur_d, tcand, kcoh, do_table, ch_pos, ch_d,
                                                          kc_done, use_done, evals, none);
        PT_LAUNCHED();
        return PT_OK;
    }
#define PT_CHOOSE_T(T) { dim3 grid((q.ew + T - 1) / T, q.rows); \
        if (lean) k_choose_tile<T, false, false, true><<<grid, T, atile_bytes(T), st>>>( \
            q, a, b, cur_pos, cur_d, tcand, kcoh, do_table, ch_pos, ch_d, kc_done, use_done, evals, none); \
        else k_choose_tile<T, false, false><<<grid, T, atile_bytes(T), st>>>( \
            q, a, b, cur_pos, cur_d, tcand, kcoh, do_table, ch_pos, ch_d, kc_done, use_done, evals, none); }
    const bool lean = lean_choose(q);
    switch (q.tile) {
        case 32: PT_CHOOSE_T(32) break;
        case 64: PT_CHOOSE_T(64) break;
        case 128: PT_CHOOSE_T(128) break;
        default: PT_CHOOSE_T(256) break;
    }
#undef PT_CHOOSE_T
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
    if (q.adesc) return pt_fail(PT_UNSUPPORTED, "learned proposals in descriptor mode");
    LearnedArgs la;
    la.cand = lcand;
    la.conf = lconf;
    la.threshold = threshold;
    la.kcoh_confident = kcoh_confident;
    la.counters = lcounters;
#define PT_CHOOSE_L(T) { dim3 grid((q.ew + T - 1) / T, q.rows); \
        k_choose_tile<T, true, false><<<grid, T, atile_bytes(T), st>>>(q, a, b, cur_pos, cur_d, tcand, kcoh, \
                                                                                   do_table, ch_pos, ch_d, kc_done, use_done, \
                                                                                   evals, la); }
    switch (q.tile) {
        case 32: PT_CHOOSE_L(32) break;
        case 64: PT_CHOOSE_L(64) break;
        case 128: PT_CHOOSE_L(128) break;
        default: PT_CHOOSE_L(256) break;
    }
#undef PT_CHOOSE_L
    PT_LAUNCHED();
    return PT_OK;
}

pt_status pt_launch_pull(const QuerySetup &s, int n, const float4 *a, const float4 *b, const int *cur_pos, const float *cur_d,
                         const int *ch_pos, const float *ch_d, int *nxt_pos, float *nxt_d,
                         unsigned long long *evals, cudaStream_t st) {
    QPlan q;
    PT_TRY(make_qplan(s, q));
    (void) n;
    const bool r1 = q.radius <= 1;
    if (q.adesc) {
        constexpr int T = TWD_DESC;
        dim3 grid((q.ew + T - 1) / T, q.rows);
        if (r1) k_pull_tile<T, 1, true><<<grid, T, 0, st>>>(q, a, b, cur_pos, cur_d, ch_pos, ch_d, nxt_pos, nxt_d, evals);
        else k_pull_tile<T, 2, true><<<grid, T, 0, st>>>(q, a, b, cur_pos, cur_d, ch_pos, ch_d, nxt_pos, nxt_d, evals);
        PT_LAUNCHED();
        return PT_OK;
    }
#define PT_PULL_T(T, RR) { dim3 grid((q.ew + T - 1) / T, q.rows); \
        if (one) k_pull_tile<T, RR, false, true><<<grid, T, atile_bytes(T), st>>>( \
            q, a, b, cur_pos, cur_d, ch_pos, ch_d, nxt_pos, nxt_d, evals); \
        else k_pull_tile<T, RR, false><<<grid, T, atile_bytes(T), st>>>( \
            q, a, b, cur_pos, cur_d, ch_pos, ch_d, nxt_pos, nxt_d, evals); }
    const bool one = one_pull(q);
    switch (q.tile) {
        case 32: if (r1) PT_PULL_T(32, 1) else PT_PULL_T(32, 2) break;
        case 64: if (r1) PT_PULL_T(64, 1) else PT_PULL_T(64, 2) break;
        case 128: if (r1) PT_PULL_T(128, 1) else PT_PULL_T(128, 2) break;
        default: if (r1) PT_PULL_T(256, 1) else PT_PULL_T(256, 2) break;
    }
#undef PT_PULL_T
    PT_LAUNCHED();
    return PT_OK;
}

pt_status pt_launch_pack_nnf(long long n, const double *ann, int *pos, float *d, cudaStream_t st) {
    if (n <= 0) return PT_OK;
    k_pack_nnf<<<(unsigned) ((n + NT - 1) / NT), NT, 0, st>>>(n, ann, pos, d);
    PT_LAUNCHED();
    return PT_OK;
}

pt_status pt_launch_output(int n, const int *pos, const float *d, double *ann, cudaStream_t st) {
    k_output<<<(n + NT - 1) / NT, NT, 0, st>>>(n, pos, d, ann);
    PT_LAUNCHED();
    return PT_OK;
}

/* ---- batched launchers ---- */

namespace {

constexpr int BATCH_TW[PT_BATCH_NTW] = {32, 64, 128, 256};

template<class K>
int persistent_grid(K kernel, int threads, size_t smem, long long work) {
    static int nsm = 0;
    if (!nsm) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    }
    int per = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem) != cudaSuccess || per < 1) per = 1;
    const long long g = (long long) per * nsm;
    return (int) (work < g ? work : g);
}

}  // namespace

int pt_batch_tw(int twi) { return (twi >= 0 && twi < PT_BATCH_NTW) ? BATCH_TW[twi] : 0; }

pt_status pt_launch_choose_batch(const QuerySetup &s, const PtBatchImage *imgs, int n, long long nseg, int twi,
                                 const float4 *a, const float4 *b, const int *cur_pos, const float *cur_d,
                                 const int *tcand, const int2 *kcoh, int do_table, int *ch_pos, float *ch_d, int *kc_done,
                                 int use_done, unsigned long long *evals, unsigned long long *work, cudaStream_t st) {
    QPlan q;
    PT_TRY(make_qplan(s, q));
    if (nseg <= 0) return PT_OK;
    PT_CUDA(cudaMemsetAsync(work, 0, sizeof(unsigned long long), st));
#define PT_CHOOSE_B(T) { const size_t sm = atile_bytes(T); \
        if (lean) { const int g = persistent_grid(k_choose_batch<T, true>, T, sm, nseg); \
            k_choose_batch<T, true><<<g, T, sm, st>>>(q, imgs, n, nseg, twi, a, b, cur_pos, cur_d, tcand, kcoh, do_table, \
                                                      ch_pos, ch_d, kc_done, use_done, evals, work); } \
        else { const int g = persistent_grid(k_choose_batch<T>, T, sm, nseg); \
            k_choose_batch<T><<<g, T, sm, st>>>(q, imgs, n, nseg, twi, a, b, cur_pos, cur_d, tcand, kcoh, do_table, ch_pos, \
                                                ch_d, kc_done, use_done, evals, work); } }
    const bool lean = lean_choose(q);
    switch (BATCH_TW[twi]) {
        case 32: PT_CHOOSE_B(32) break;
        case 64: PT_CHOOSE_B(64) break;
        case 128: PT_CHOOSE_B(128) break;
        default: PT_CHOOSE_B(256) break;
    }
#undef PT_CHOOSE_B
    PT_LAUNCHED();
    return PT_OK;
}

pt_status pt_launch_pull_batch(const QuerySetup &s, const PtBatchImage *imgs, int n, long long nseg, int twi,
                               const float4 *a, const float4 *b, const int *cur_pos, const float *cur_d, const int *ch_pos,
                               const float *ch_d, int *nxt_pos, float *nxt_d, unsigned long long *evals,
                               unsigned long long *work, cudaStream_t st) {
    QPlan q;
    PT_TRY(make_qplan(s, q));
    if (nseg <= 0) return PT_OK;
    PT_CUDA(cudaMemsetAsync(work, 0, sizeof(unsigned long long), st));
#define PT_PULL_B(T, RR) { const size_t sm = atile_bytes(T); \
        if (one) { const int g = persistent_grid(k_pull_batch<T, RR, true>, T, sm, nseg); \
            k_pull_batch<T, RR, true><<<g, T, sm, st>>>(q, imgs, n, nseg, twi, a, b, cur_pos, cur_d, ch_pos, ch_d, nxt_pos, \
                                                        nxt_d, evals, work); } \
        else { const int g = persistent_grid(k_pull_batch<T, RR>, T, sm, nseg); \
            k_pull_batch<T, RR><<<g, T, sm, st>>>(q, imgs, n, nseg, twi, a, b, cur_pos, cur_d, ch_pos, ch_d, nxt_pos, nxt_d, \
                                                  evals, work); } }
    const bool one = one_pull(q);
    const bool r1 = q.radius <= 1;
    switch (BATCH_TW[twi]) {
        case 32: if (r1) PT_PULL_B(32, 1) else PT_PULL_B(32, 2) break;
        case 64: if (r1) PT_PULL_B(64, 1) else PT_PULL_B(64, 2) break;
        case 128: if (r1) PT_PULL_B(128, 1) else PT_PULL_B(128, 2) break;
        default: if (r1) PT_PULL_B(256, 1) else PT_PULL_B(256, 2) break;
    }
#undef PT_PULL_B
    PT_LAUNCHED();
    return PT_OK;
}

pt_status pt_launch_init_temporal(const QuerySetup &s, const double *prev, const float *scale_sv, int recalc, int sanitize,
                                  double temporal_scale, const float4 *a, const float4 *b, int *cur_pos, float *cur_d,
                                  double *orig, int *bad, cudaStream_t st) {
    QPlan q;
    PT_TRY(make_qplan(s, q));
    const int n = q.ew * q.eh;
    k_init_temporal<<<(n + NT - 1) / NT, NT, 0, st>>>(q, prev, scale_sv, recalc, sanitize, temporal_scale, a, b, cur_pos, cur_d,
                                                     orig, bad);
    PT_LAUNCHED();
    return PT_OK;
}

pt_status pt_launch_output_temporal(int n, const int *pos, const float *d, const int *pos0, const float *d0,
                                    const double *orig, double *ann, cudaStream_t st) {
    k_output_temporal<<<(n + NT - 1) / NT, NT, 0, st>>>(n, pos, d, pos0, d0, orig, ann);
    PT_LAUNCHED();
    return PT_OK;
}

pt_status pt_launch_init_random(const QuerySetup &s, const float4 *a, const float4 *b, int *cur_pos, float *cur_d,
                                cudaStream_t st) {
    QPlan q;
    PT_TRY(make_qplan(s, q));
    const int n = q.ew * q.eh;
    k_init_random<<<(n + NT - 1) / NT, NT, 0, st>>>(q, a, b, cur_pos, cur_d);
    PT_LAUNCHED();
    return PT_OK;
}
