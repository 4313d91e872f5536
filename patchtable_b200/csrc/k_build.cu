/* Table build kernels: per-dimension range, quantile samples, the query's cell lookup, and the
   distance transforms other than prop (populate and the prop DT are one cooperative launch,
   k_table_build.cu).

   References (patchtable/patchtable.h):
     set_min_max              :1758-1778
     PatchPartition1D         :1172-1286  (quantile centres; the to_bin table is built on the host)
     get_bin                  :1298-1325
     do_dt_brute              :2364-2413  (patch_dist_to_grid :1403-1425) */
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include "pt_bins.cuh"
#include "pt_internal.h"
#include "pt_kernels.h"

namespace {

constexpr int NT = 256;

struct BinPlan {
    int G;
    float min_val[PT_DESC_MAX];
    float range[PT_DESC_MAX];
    long long stride[PT_DESC_MAX];
};

/* PatchPartition1D::get_bin, patchtable.h:1298-1325 (pt_bins.cuh). */
__device__ __forceinline__ int get_bin(const BinPlan &c_bins, const int *__restrict__ to_bin, int d, float v) {
    return pt_get_bin(c_bins.min_val[d], c_bins.range[d], to_bin + d * PT_NMAP, v);
}

__device__ __forceinline__ bool allowed_at(const int *allowed, int allowed_index, long long p) {
    return allowed == nullptr || allowed[p] == allowed_index;
}

/* Per-block min/max of each grid dimension over allowed patches (set_min_max). */
__global__ void k_minmax(const float *__restrict__ desc, int ds, int G, long long P, const int *allowed,
                         int allowed_index, float *pmin, float *pmax) {
    __shared__ float smin[PT_DESC_MAX][NT / 32], smax[PT_DESC_MAX][NT / 32];
    float mn[PT_DESC_MAX], mx[PT_DESC_MAX];
    for (int d = 0; d < PT_DESC_MAX; d++) { mn[d] = 1e20f; mx[d] = -1e20f; }
    for (long long p = blockIdx.x * (long long) NT + threadIdx.x; p < P; p += (long long) gridDim.x * NT) {
        if (!allowed_at(allowed, allowed_index, p)) continue;
        const float *v = desc + p * ds;
        for (int d = 0; d < G; d++) { float x = v[d]; mn[d] = fminf(mn[d], x); mx[d] = fmaxf(mx[d], x); }
    }
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int d = 0; d < G; d++) {
        float a = mn[d], b = mx[d];
        for (int o = 16; o; o >>= 1) { a = fminf(a, __shfl_xor_sync(0xffffffffu, a, o)); b = fmaxf(b, __shfl_xor_sync(0xffffffffu, b, o)); }
        if (lane == 0) { smin[d][wid] = a; smax[d][wid] = b; }
    }
    __syncthreads();
    if (threadIdx.x < G) {
        int d = threadIdx.x;
        float a = smin[d][0], b = smax[d][0];
        for (int i = 1; i < NT / 32; i++) { a = fminf(a, smin[d][i]); b = fmaxf(b, smax[d][i]); }
        pmin[blockIdx.x * PT_DESC_MAX + d] = a;
        pmax[blockIdx.x * PT_DESC_MAX + d] = b;
    }
}

/* Values of dimension d of the patches used for the partition (every partition_step-th patch
   in x and y, allowed only; patchtable.h:1355-1380), compacted in any order. */
__global__ void k_gather_dim(const float *__restrict__ desc, int ds, int d, int eh, int ew, int step,
                             const int *allowed, int allowed_index, float *out, int *count) {
    long long p = blockIdx.x * (long long) NT + threadIdx.x;
    if (p >= (long long) eh * ew) return;
    int y = (int) (p / ew), x = (int) (p % ew);
    if (y % step || x % step || !allowed_at(allowed, allowed_index, p)) return;
    int slot = atomicAdd(count, 1);
    out[slot] = desc[p * ds + d];
}

__global__ void k_pick(const float *sorted, const int *idx, int n, float *out) {
    int i = blockIdx.x * NT + threadIdx.x;
    if (i < n) out[i] = sorted[idx[i]];
}

/* Table candidate of every query patch: the cell's stored patch (patchtable.h:3675-3686). */
__global__ void k_table_cand(const BinPlan c_bins, const float *__restrict__ desc, int ds, long long P,
                             const int *__restrict__ to_bin, const int *__restrict__ table, int *tcand) {
    long long p = blockIdx.x * (long long) NT + threadIdx.x;
    if (p >= P) return;
    const float *v = desc + p * ds;
    long long cell = 0;
    for (int d = 0; d < c_bins.G; d++) cell += (long long) get_bin(c_bins, to_bin, d, v[d]) * c_bins.stride[d];
    tcand[p] = __ldg(table + cell);
}

inline int blocks_for(long long n) { return (int) ((n + NT - 1) / NT); }

}  // namespace

pt_status pt_launch_minmax(PtPartScratch &s, const float *desc, int ds, int G, long long P, const int *allowed,
                           int allowed_index, float *hmin, float *hmax, cudaStream_t st) {
    const int NB = 296;
    PT_CUDA(s.pmin.reserve(NB * PT_DESC_MAX));
    PT_CUDA(s.pmax.reserve(NB * PT_DESC_MAX));
    k_minmax<<<NB, NT, 0, st>>>(desc, ds, G, P, allowed, allowed_index, s.pmin.p, s.pmax.p);
    PT_LAUNCHED();
    std::vector<float> a(NB * PT_DESC_MAX), b(NB * PT_DESC_MAX);
    PT_CUDA(cudaMemcpyAsync(a.data(), s.pmin.p, sizeof(float) * a.size(), cudaMemcpyDeviceToHost, st));
    PT_CUDA(cudaMemcpyAsync(b.data(), s.pmax.p, sizeof(float) * b.size(), cudaMemcpyDeviceToHost, st));
    PT_CUDA(cudaStreamSynchronize(st));
    for (int d = 0; d < G; d++) {
        float mn = 1e20f, mx = -1e20f;
        for (int i = 0; i < NB; i++) { mn = std::min(mn, a[i * PT_DESC_MAX + d]); mx = std::max(mx, b[i * PT_DESC_MAX + d]); }
        hmin[d] = mn; hmax[d] = mx;
    }
    return PT_OK;
}

pt_status pt_quantile_gather(PtPartScratch &s, const float *desc, int ds, int d, int eh, int ew, int step,
                             const int *allowed, int allowed_index, int *count_out, cudaStream_t st) {
    const long long P = (long long) eh * ew;
    PT_CUDA(s.keys.reserve(P));
    PT_CUDA(s.cnt.reserve(1));
    PT_CUDA(cudaMemsetAsync(s.cnt.p, 0, sizeof(int), st));
    k_gather_dim<<<blocks_for(P), NT, 0, st>>>(desc, ds, d, eh, ew, step, allowed, allowed_index, s.keys.p, s.cnt.p);
    PT_LAUNCHED();
    int n = 0;
    PT_CUDA(cudaMemcpyAsync(&n, s.cnt.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    PT_CUDA(cudaStreamSynchronize(st));
    *count_out = n;
    return PT_OK;
}

pt_status pt_quantile_pick(PtPartScratch &s, int n, const std::vector<int> &want, std::vector<float> &vals,
                           cudaStream_t st) {
    vals.clear();
    if (want.empty() || n < 1) return PT_OK;
    PT_CUDA(s.sorted.reserve(n));
    size_t tmp_bytes = 0;
    PT_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, s.keys.p, s.sorted.p, n, 0, 32, st));
    PT_CUDA(s.tmp.reserve(tmp_bytes));
    PT_CUDA(cub::DeviceRadixSort::SortKeys(s.tmp.p, tmp_bytes, s.keys.p, s.sorted.p, n, 0, 32, st));
    pt_count_launches(4);
    PT_CUDA(s.idx.reserve(want.size()));
    PT_CUDA(s.picked.reserve(want.size()));
    PT_CUDA(cudaMemcpyAsync(s.idx.p, want.data(), sizeof(int) * want.size(), cudaMemcpyHostToDevice, st));
    k_pick<<<blocks_for((long long) want.size()), NT, 0, st>>>(s.sorted.p, s.idx.p, (int) want.size(), s.picked.p);
    PT_LAUNCHED();
    vals.resize(want.size());
    PT_CUDA(cudaMemcpyAsync(vals.data(), s.picked.p, sizeof(float) * want.size(), cudaMemcpyDeviceToHost, st));
    PT_CUDA(cudaStreamSynchronize(st));
    return PT_OK;
}

static BinPlan bin_plan(const PtBins &bins) {
    BinPlan b;
    memset(&b, 0, sizeof(b));
    b.G = bins.G;
    for (int d = 0; d < bins.G; d++) { b.min_val[d] = bins.min_val[d]; b.range[d] = bins.range[d]; b.stride[d] = bins.stride[d]; }
    return b;
}

pt_status pt_launch_table_candidates(const PtBins &bins, const float *desc, int ds, long long P, const int *to_bin,
                                     const int *table, int *tcand, cudaStream_t st) {
    k_table_cand<<<blocks_for(P), NT, 0, st>>>(bin_plan(bins), desc, ds, P, to_bin, table, tcand);
    PT_LAUNCHED();
    return PT_OK;
}

/* The other distance transforms of the table build (patchtable.h:3271-3285):
     do_dt_prop1 + unmask_table  :2306-2336
     do_dt_downsample            :2339-2358 with dt_downsample / dt_upsample (dt_downsample.h)
     do_dt_euclidean             :4244-4340
   All three are pointwise per level or per line, so each runs as independent threads and the
   result is bit-identical to the sequential loops. */
namespace {

constexpr int HI_MASK = 1 << 30;        /* TABLE_HI_MASK, patchtable.h:109-112 */

/* A grid of G dimensions laid out row-major (dimension 0 slowest). */
struct GridShape {
    int G;
    long long n;
    long long stride[PT_DESC_MAX];
    int size[PT_DESC_MAX];
};

GridShape grid_shape(int G, const int *size) {
    GridShape s;
    s.G = G;
    s.n = 1;
    for (int d = G - 1; d >= 0; d--) { s.stride[d] = s.n; s.size[d] = size[d]; s.n *= size[d]; }
    return s;
}

/* do_dt_prop1: an unused cell takes, with the high bit set, the value of its lowest-indexed
   neighbour that was populated before the pass.  Neighbours this pass writes carry the high bit
   and populated cells are never written, so concurrent writes cannot change what a thread
   classifies as populated. */
__global__ void k_dt_prop1(int *table, const GridShape s) {
    long long j = blockIdx.x * (long long) NT + threadIdx.x;
    if (j >= s.n || table[j] != PT_UNUSED) return;
    long long best = -1;
    int val = 0;
    for (int d = 0; d < s.G; d++) {
        int c = (int) ((j / s.stride[d]) % s.size[d]);
        if (c > 0) {
            long long k = j - s.stride[d];
            int v = table[k];
            if (v != PT_UNUSED && !(v & HI_MASK) && (best < 0 || k < best)) { best = k; val = v; }
        }
        if (c + 1 < s.size[d]) {
            long long k = j + s.stride[d];
            int v = table[k];
            if (v != PT_UNUSED && !(v & HI_MASK) && (best < 0 || k < best)) { best = k; val = v; }
        }
    }
    if (best >= 0) table[j] = val | HI_MASK;
}

__global__ void k_dt_unmask(int *table, long long n) {
    long long j = blockIdx.x * (long long) NT + threadIdx.x;
    if (j < n) table[j] &= HI_MASK - 1;
}

/* dt_downsample: a coarse cell takes the first child, in lexicographic order with dimension 0
   slowest, holding a value without the high bit; otherwise it is unused.  Only dimensions where
   the cell has two children enter the enumeration, so its cost is 2^(such dimensions). */
__global__ void k_dt_down(const int *__restrict__ hi, const GridShape hs, int *lo, const GridShape ls) {
    long long j = blockIdx.x * (long long) NT + threadIdx.x;
    if (j >= ls.n) return;
    long long base = 0;
    long long twos[PT_DESC_MAX];
    int m = 0;
    for (int d = 0; d < ls.G; d++) {
        int c = (int) ((j / ls.stride[d]) % ls.size[d]);
        base += 2LL * c * hs.stride[d];
        if (2 * c + 1 < hs.size[d]) twos[m++] = hs.stride[d];
    }
    int out = PT_UNUSED;
    for (unsigned k = 0; k < (1u << m); k++) {
        long long h = base;
        for (int i = 0; i < m; i++)
            if ((k >> (m - 1 - i)) & 1) h += twos[i];
        int v = hi[h];
        if (!(v & HI_MASK) && v != PT_UNUSED) { out = v; break; }
    }
    lo[j] = out;
}

/* dt_upsample: every unused fine cell copies its parent. */
__global__ void k_dt_up(const int *__restrict__ lo, const GridShape ls, int *hi, const GridShape hs) {
    long long j = blockIdx.x * (long long) NT + threadIdx.x;
    if (j >= hs.n || hi[j] != PT_UNUSED) return;
    long long p = 0;
    for (int d = 0; d < hs.G; d++) p += (long long) (((j / hs.stride[d]) % hs.size[d]) / 2) * ls.stride[d];
    hi[j] = lo[p];
}

__global__ void k_edt_init(const int *__restrict__ table, float *dist, long long n) {
    long long j = blockIdx.x * (long long) NT + threadIdx.x;
    if (j < n) dist[j] = table[j] == PT_UNUSED ? 1e20f : 0.0f;
}

/* euclidean_dt along dimension dim, one thread per line: the lower envelope of the parabolas
   (q - v)^2 + f(v) with the reference's single-precision operation order, then the distances
   and, in place along the line, the value of each cell's envelope parabola (index_array,
   patchtable.h:4265).  The envelope lives in scratch laid out [k][line] so that neighbouring
   lines touch neighbouring words.  The intersection with the sentinel at -1E20 can never fall
   at or below it (distances are at most 1E20 and the denominator at least 2), so the k > 0
   guard never changes a result. */
__global__ void k_edt_line(int *table, const float *__restrict__ fin, float *fout, const GridShape s, int dim,
                           long long nlines, int *vs, float *zs) {
    long long l = blockIdx.x * (long long) NT + threadIdx.x;
    if (l >= nlines) return;
    long long base = 0, r = l;
    for (int d = s.G - 1; d >= 0; d--) {
        if (d == dim) continue;
        base += (r % s.size[d]) * s.stride[d];
        r /= s.size[d];
    }
    const int n = s.size[dim];
    const long long st = s.stride[dim];
#define V(k) vs[(long long) (k) * nlines + l]
#define Z(k) zs[(long long) (k) * nlines + l]
#define F(q) fin[base + (long long) (q) * st]
    /* Squares of ints wrap at 32 bits as in the reference's build (from 46341 cells on). */
    auto sq = [](int x) { return (float) (int) ((unsigned) x * (unsigned) x); };
    auto inter = [&](int q, float fq, int v) {
        float a = __fadd_rn(fq, sq(q));
        float b = __fadd_rn(F(v), sq(v));
        return __fdiv_rn(__fsub_rn(a, b), (float) (2 * q - 2 * v));
    };
    int k = 0;
    V(0) = 0;
    Z(0) = -1e20f;
    Z(1) = 1e20f;
    for (int q = 1; q < n; q++) {
        float fq = F(q);
        int v = V(k);
        float x = inter(q, fq, v);
        while (k > 0 && x <= Z(k)) {
            k--;
            v = V(k);
            x = inter(q, fq, v);
        }
        k++;
        V(k) = q;
        Z(k) = x;
        Z(k + 1) = 1e20f;
    }
    k = 0;
    for (int q = 0; q < n; q++) {
        while (Z(k + 1) < (float) q) k++;
        int v = V(k);
        fout[base + (long long) q * st] = __fadd_rn(sq(q - v), F(v));
        table[base + (long long) q * st] = table[base + (long long) v * st];
    }
#undef V
#undef Z
#undef F
}

/* do_dt_brute (patchtable.h:2364-2413): every cell takes the patch of b nearest its grid centre
   under patch_dist_to_grid<0> with TABLE_INFINITY_NORM (patchtable.h:1403-1425),
   max_d |wh_d - centre_d| / (rsize_d if wh_d - centre_d > 0 else lsize_d), over the whole valid
   patch region in raster order (the allowed mask is not consulted); patch 0 seeds the search and
   only a strictly smaller distance replaces it, so ties keep the earliest patch.  One thread per
   cell, descriptors streamed through shared memory in tiles that every thread of the CTA reads
   (broadcast loads).  The arithmetic is the reference's single-precision sequence: IEEE
   subtract and divide, maxima as (a > b ? a : b), so a NaN from a zero-width cell behaves as it
   does there.  Work is cells x patches x G: a validation algorithm, as in the reference. */
struct BrutePart {
    int ofs[PT_DESC_MAX];     /* per dimension: centres at ofs, lsizes at ofs + n, rsizes at ofs + 2n */
};

constexpr int BRUTE_TILE = 128;

template<int G>
__global__ void __launch_bounds__(NT) k_dt_brute(int *table, const GridShape s, const BrutePart bp,
                                                 const float *__restrict__ part, const float *__restrict__ desc,
                                                 int ds, long long P, int ew) {
    __shared__ float tile[BRUTE_TILE * G];
    const long long j = blockIdx.x * (long long) NT + threadIdx.x;
    const bool live = j < s.n;
    float c[G], lo[G], hi[G];
#pragma unroll
    for (int d = 0; d < G; d++) {
        const int n = s.size[d];
        const int g = live ? (int) ((j / s.stride[d]) % n) : 0;
        c[d] = part[bp.ofs[d] + g];
        lo[d] = part[bp.ofs[d] + n + g];
        hi[d] = part[bp.ofs[d] + 2 * n + g];
    }
    float best = 0.f;
    long long bestp = 0;
    for (long long base = 0; base < P; base += BRUTE_TILE) {
        const int m = (int) (P - base < BRUTE_TILE ? P - base : BRUTE_TILE);
        __syncthreads();
        for (int k = threadIdx.x; k < m * G; k += NT) tile[k] = desc[(base + k / G) * ds + k % G];
        __syncthreads();
        if (!live) continue;
        for (int q = 0; q < m; q++) {
            float ans = 0.f;
#pragma unroll
            for (int d = 0; d < G; d++) {
                const float delta = __fsub_rn(tile[q * G + d], c[d]);
                const float v = __fdiv_rn(fabsf(delta), delta > 0.f ? hi[d] : lo[d]);
                ans = ans > v ? ans : v;
            }
            if (base + q == 0) best = ans;
            else if (ans < best) { best = ans; bestp = base + q; }
        }
    }
    if (live) table[j] = pt_xy((int) (bestp % ew) + 7, (int) (bestp / ew) + 7);
}

}  // namespace

pt_status pt_dt_other(int *table, int G, const int *nslices, int dt_algo, cudaStream_t st) {
    if (G < 1 || G > PT_DESC_MAX) return pt_fail(PT_BAD_ARG, "grid dims %d outside 1..%d", G, PT_DESC_MAX);
    GridShape s = grid_shape(G, nslices);
    if (dt_algo == 5) {
        k_dt_prop1<<<blocks_for(s.n), NT, 0, st>>>(table, s);
        PT_LAUNCHED();
    }
    if (dt_algo == 4 || dt_algo == 5) {
        /* Pyramid down to all sizes 1, then back up (do_dt_downsample). */
        std::vector<GridShape> shapes{s};
        for (;;) {
            const GridShape &h = shapes.back();
            bool unit = true;
            int ls[PT_DESC_MAX];
            for (int d = 0; d < G; d++) { unit = unit && h.size[d] == 1; ls[d] = (h.size[d] + 1) / 2; }
            if (unit) break;
            shapes.push_back(grid_shape(G, ls));
        }
        std::vector<DevBuf<int>> lv(shapes.size());    /* lv[0] unused: level 0 is the table */
        for (size_t i = 1; i < shapes.size(); i++) PT_CUDA(lv[i].reserve(shapes[i].n));
        auto level = [&](size_t i) { return i == 0 ? table : lv[i].p; };
        for (size_t i = 1; i < shapes.size(); i++) {
            k_dt_down<<<blocks_for(shapes[i].n), NT, 0, st>>>(level(i - 1), shapes[i - 1], level(i), shapes[i]);
            PT_LAUNCHED();
        }
        for (size_t i = shapes.size() - 1; i >= 1; i--) {
            k_dt_up<<<blocks_for(shapes[i - 1].n), NT, 0, st>>>(level(i), shapes[i], level(i - 1), shapes[i - 1]);
            PT_LAUNCHED();
        }
        if (dt_algo == 5) {
            k_dt_unmask<<<blocks_for(s.n), NT, 0, st>>>(table, s.n);
            PT_LAUNCHED();
        }
        PT_CUDA(cudaStreamSynchronize(st));            /* the pyramid levels are freed on return */
        return PT_OK;
    }
    if (dt_algo == 6) {
        int maxn = 0;
        for (int d = 0; d < G; d++) maxn = std::max(maxn, nslices[d]);
        long long maxlines = 0;
        for (int d = 0; d < G; d++) maxlines = std::max(maxlines, s.n / nslices[d]);
        DevBuf<float> dist[2];
        DevBuf<int> vs;
        DevBuf<float> zs;
        PT_CUDA(dist[0].reserve(s.n));
        PT_CUDA(dist[1].reserve(s.n));
        PT_CUDA(vs.reserve(maxlines * maxn));
        PT_CUDA(zs.reserve(maxlines * (maxn + 1)));
        k_edt_init<<<blocks_for(s.n), NT, 0, st>>>(table, dist[0].p, s.n);
        PT_LAUNCHED();
        for (int d = 0; d < G; d++) {
            long long nl = s.n / nslices[d];
            k_edt_line<<<blocks_for(nl), NT, 0, st>>>(table, dist[d & 1].p, dist[(d + 1) & 1].p, s, d, nl, vs.p, zs.p);
            PT_LAUNCHED();
        }
        PT_CUDA(cudaStreamSynchronize(st));
        return PT_OK;
    }
    return pt_fail(PT_UNSUPPORTED, "dt_algo %d is not implemented on the GPU path", dt_algo);
}

pt_status pt_dt_brute(int *table, int G, const int *nslices, const float *part, const int *part_ofs, const float *desc,
                      int ds, long long P, int ew, cudaStream_t st) {
    if (G < 1 || G > PT_DESC_MAX) return pt_fail(PT_BAD_ARG, "grid dims %d outside 1..%d", G, PT_DESC_MAX);
    if (P < 1 || ew < 1) return pt_fail(PT_BAD_ARG, "brute distance transform over %lld patches", P);
    const GridShape s = grid_shape(G, nslices);
    BrutePart bp;
    for (int d = 0; d < PT_DESC_MAX; d++) bp.ofs[d] = d < G ? part_ofs[d] : 0;
    switch (G) {
#define PT_BRUTE_CASE(g) case g: k_dt_brute<g><<<blocks_for(s.n), NT, 0, st>>>(table, s, bp, part, desc, ds, P, ew); break;
        PT_BRUTE_CASE(1) PT_BRUTE_CASE(2) PT_BRUTE_CASE(3) PT_BRUTE_CASE(4) PT_BRUTE_CASE(5) PT_BRUTE_CASE(6)
        PT_BRUTE_CASE(7) PT_BRUTE_CASE(8) PT_BRUTE_CASE(9) PT_BRUTE_CASE(10) PT_BRUTE_CASE(11) PT_BRUTE_CASE(12)
        PT_BRUTE_CASE(13) PT_BRUTE_CASE(14) PT_BRUTE_CASE(15) PT_BRUTE_CASE(16)
#undef PT_BRUTE_CASE
    }
    PT_LAUNCHED();
    return PT_OK;
}
