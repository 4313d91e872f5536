/* The table's cells in one cooperative launch: fill, populate, resolve, seed, the propagation
   distance transform and fill_zeros.

   References (patchtable/patchtable.h):
     populate (fast, random order)  :3121-3159
     do_dt_prop                     :2081-2165  (edge labels PropEdge :1435-1447)
     fill_zeros                     :2063-2079

   Every CTA of the grid is resident at once (cudaLaunchCooperativeKernel), and the phases are
   separated by grid barriers whose waits are bounded: a CTA that polls longer than the process's
   spin limit (pt_set_spin_limit) records PT_TIMEOUT, and every CTA leaves at its next barrier, so
   the launch always ends and the host reports the status.

   Phases (one grid barrier after each):
     fill      every cell TABLE_UNUSED, every claim key empty;
     populate  each allowed patch's cell takes the smallest shuffle rank that reaches it (the first
               visitor of the reference's random_shuffle order wins);
     resolve   ranks become packed positions; each CTA counts the seeded cells of its contiguous
               range of cells;
     seed      the seeded cells, in increasing cell order, become the first frontier (label 0):
               each CTA writes its range at the prefix of the counts before it;
     levels    the reference's breadth-first fill, level-synchronously: every frontier element
               claims the unused neighbours its label allows with atomicMin on (element, edge) and
               keeps a bit mask of those edges; each CTA checks, for its contiguous range of
               elements, which of the masked claims they won (a second mask); winners fill their
               cells and append (cell, label) to the next frontier at the scanned offsets, i.e. in
               (element, edge) order, which is the order of the reference's next frontier list.
   The filled table is therefore bit-identical to the reference's.  Data written by other CTAs in
   an earlier phase is read with L2-only loads (ld.global.cg), never from a CTA's own L1. */
#include <cuda_runtime.h>
#include <cub/block/block_reduce.cuh>
#include <cub/block/block_scan.cuh>

#include <atomic>

#include "pt_bins.cuh"
#include "pt_internal.h"
#include "pt_kernels.h"

namespace {

constexpr int NT = 256;
constexpr long long KEY_ELEMENTS = 1ll << 27;   /* claim key = element << 5 | edge */

struct CellBuild {
    int G;
    float min_val[PT_DESC_MAX], range[PT_DESC_MAX];
    long long stride[PT_DESC_MAX];
    int nslices[PT_DESC_MAX];
    const float *desc;
    int ds;
    long long P;
    const int *rank;             /* shuffle rank of each patch, -1 when not allowed */
    const int *to_bin;
    const int *order_xy;         /* packed position of each rank */
    int *table;
    long long ncells;
    unsigned *claim;
    int *fidx[2];
    unsigned char *flab[2];
    unsigned *emask;             /* per frontier element: edges to unused neighbours, then the edges it won */
    long long *ctot;             /* per-CTA totals */
    unsigned *bar;               /* [0] arrivals, [1] generation */
    int *status;                 /* [0] pt_status of the launch, [1] levels, [2] phase that failed */
    long long *seeded;
    int run_dt, dt_iters, fill_zeros, vfill;
    long long spin_limit;
};

/* Grid barrier with a bounded wait.  Returns false once any CTA has recorded an error. */
__device__ __forceinline__ bool grid_barrier(const CellBuild &a, int phase) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *vgen = a.bar + 1;
        volatile int *vstatus = a.status;
        int ok = 1;
        const unsigned gen = *vgen;            /* read before arriving: it cannot move until we do */
        __threadfence();
        if (atomicAdd(a.bar, 1u) == gridDim.x - 1) {
            atomicExch(a.bar, 0u);
            __threadfence();
            atomicAdd(a.bar + 1, 1u);
        } else {
            long long polls = 0;
            while (*vgen == gen) {
                if (*vstatus != 0) { ok = 0; break; }
                if (++polls > a.spin_limit) {
                    if (atomicCAS(a.status, 0, (int) PT_TIMEOUT) == 0) a.status[2] = phase;
                    ok = 0;
                    break;
                }
                __nanosleep(128);
            }
        }
        __threadfence();
        if (*vstatus != 0) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

typedef cub::BlockReduce<long long, NT> Reduce;
typedef cub::BlockScan<int, NT> Scan;

union Shared {
    typename Reduce::TempStorage reduce;
    typename Scan::TempStorage scan;
};

/* Sum of a value over the CTA (every thread receives it). */
__device__ __forceinline__ long long cta_sum(Shared &sh, long long v) {
    __shared__ long long s_sum;
    __syncthreads();
    const long long t = Reduce(sh.reduce).Sum(v);
    if (threadIdx.x == 0) s_sum = t;
    __syncthreads();
    return s_sum;
}

/* Prefix of the per-CTA totals before this CTA, and their sum. */
__device__ __forceinline__ void cta_prefix(Shared &sh, const CellBuild &a, long long &before, long long &total) {
    long long b = 0, t = 0;
    for (int k = threadIdx.x; k < (int) gridDim.x; k += NT) {
        const long long v = __ldcg(a.ctot + k);
        t += v;
        if (k < (int) blockIdx.x) b += v;
    }
    before = cta_sum(sh, b);
    total = cta_sum(sh, t);
}

/* Edge e of label lab (patchtable.h:2101-2120): label 0 -> (i, -1), (i, +1) for every dimension i;
   label 2i + 1 + (dir + 1) / 2 -> (i, dir), then (j, -1), (j, +1) for every j > i.  The label the
   filled cell receives is that of the edge's own (dimension, direction). */
__device__ __forceinline__ int edge_count(int G, int lab) { return lab == 0 ? 2 * G : 1 + 2 * (G - 1 - (lab - 1) / 2); }

__device__ __forceinline__ void edge_of(int lab, int e, int &dim, int &dir) {
    if (lab == 0) { dim = e >> 1; dir = (e & 1) ? 1 : -1; return; }
    const int i = (lab - 1) >> 1;
    if (e == 0) { dim = i; dir = ((lab - 1) & 1) ? 1 : -1; return; }
    dim = i + 1 + ((e - 1) >> 1);
    dir = ((e - 1) & 1) ? 1 : -1;
}

/* Neighbour of cell g along (dim, dir) when it lies inside the grid and is still unused; -1 otherwise. */
__device__ __forceinline__ long long open_neighbour(const CellBuild &a, long long g, int dim, int dir) {
    const long long gp = g + dir * a.stride[dim];
    if (gp < 0 || gp >= a.ncells) return -1;
    const long long dp = (g / a.stride[dim]) % a.nslices[dim] + dir;
    if (dp < 0 || dp >= a.nslices[dim]) return -1;
    if (__ldcg(a.table + gp) != PT_UNUSED) return -1;
    return gp;
}

__global__ void __launch_bounds__(NT) k_table_build(const CellBuild a) {
    __shared__ Shared sh;
    const long long nthr = (long long) gridDim.x * NT;
    const long long tid = (long long) blockIdx.x * NT + threadIdx.x;

    /* fill */
    for (long long i = tid; i < a.ncells; i += nthr) {
        a.table[i] = PT_UNUSED;
        if (a.run_dt) a.claim[i] = 0xffffffffu;
    }
    if (!grid_barrier(a, 0)) return;

    /* populate: first visitor in shuffled order wins (patchtable.h:3142-3154) */
    for (long long p = tid; p < a.P; p += nthr) {
        const int r = __ldg(a.rank + p);
        if (r < 0) continue;
        const float *v = a.desc + p * a.ds;
        long long cell = 0;
        for (int d = 0; d < a.G; d++)
            cell += (long long) pt_get_bin(a.min_val[d], a.range[d], a.to_bin + d * PT_NMAP, __ldg(v + d)) * a.stride[d];
        atomicMin(a.table + cell, r);
    }
    if (!grid_barrier(a, 1)) return;

    /* resolve: ranks -> packed positions; seeded cells of this CTA's range */
    const long long chunk = (a.ncells + gridDim.x - 1) / gridDim.x;
    const long long c0 = min(a.ncells, (long long) blockIdx.x * chunk), c1 = min(a.ncells, c0 + chunk);
    {
        long long local = 0;
        for (long long j = c0 + threadIdx.x; j < c1; j += NT) {
            const int v = __ldcg(a.table + j);
            if (v != PT_UNUSED) { a.table[j] = __ldg(a.order_xy + v); local++; }
        }
        const long long s = cta_sum(sh, local);
        if (threadIdx.x == 0) a.ctot[blockIdx.x] = s;
    }
    if (!grid_barrier(a, 2)) return;

    long long before, n;
    cta_prefix(sh, a, before, n);
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.seeded = n;
    int levels = 0;
    if (a.run_dt) {
        /* seed: the first frontier in increasing cell order, label 0 (patchtable.h:2087-2093) */
        long long o = before;
        for (long long j0 = c0; j0 < c1; j0 += NT) {
            const long long j = j0 + threadIdx.x;
            const int f = (j < c1 && __ldcg(a.table + j) != PT_UNUSED) ? 1 : 0;
            int off, tot;
            __syncthreads();
            Scan(sh.scan).ExclusiveSum(f, off, tot);
            if (f) { a.fidx[0][o + off] = (int) j; a.flab[0][o + off] = 0; }
            o += tot;
        }
        if (!grid_barrier(a, 3)) return;
        int cur = 0;
        for (int iter = 0;; iter++) {
            if (a.dt_iters > 0 && iter > a.dt_iters) break;
            if (n == 0) break;
            if (n >= KEY_ELEMENTS) {
                if (blockIdx.x == 0 && threadIdx.x == 0 && atomicCAS(a.status, 0, (int) PT_UNSUPPORTED) == 0) a.status[2] = 4;
                return;
            }
            const int *fi = a.fidx[cur];
            const unsigned char *fl = a.flab[cur];
            /* claim: the smallest (element, edge) key wins each unused neighbour (:2131-2156); the
               element remembers which of its edges led to an unused neighbour */
            for (long long i = tid; i < n; i += nthr) {
                const long long g = __ldcg(fi + i);
                const int lab = __ldcg(fl + i), ne = edge_count(a.G, lab);
                unsigned open = 0;
                for (int e = 0; e < ne; e++) {
                    int dim, dir;
                    edge_of(lab, e, dim, dir);
                    const long long gp = open_neighbour(a, g, dim, dir);
                    if (gp >= 0) {
                        atomicMin(a.claim + gp, ((unsigned) i << 5) | (unsigned) e);
                        open |= 1u << e;
                    }
                }
                a.emask[i] = open;
            }
            if (!grid_barrier(a, 5)) return;
            /* count the claims each element of this CTA's range won (only its open edges) */
            const long long ech = (n + gridDim.x - 1) / gridDim.x;
            const long long e0 = min(n, (long long) blockIdx.x * ech), e1 = min(n, e0 + ech);
            {
                long long local = 0;
                for (long long i = e0 + threadIdx.x; i < e1; i += NT) {
                    unsigned open = __ldcg(a.emask + i), won = 0;
                    if (open) {
                        const long long g = __ldcg(fi + i);
                        const int lab = __ldcg(fl + i);
                        while (open) {
                            const int e = __ffs(open) - 1;
                            open &= open - 1;
                            int dim, dir;
                            edge_of(lab, e, dim, dir);
                            if (__ldcg(a.claim + g + dir * a.stride[dim]) == (((unsigned) i << 5) | (unsigned) e)) won |= 1u << e;
                        }
                    }
                    a.emask[i] = won;
                    local += __popc(won);
                }
                const long long s = cta_sum(sh, local);
                if (threadIdx.x == 0) a.ctot[blockIdx.x] = s;
            }
            if (!grid_barrier(a, 6)) return;
            long long base, next;
            cta_prefix(sh, a, base, next);
            /* emit: winners fill their cells and append to the next frontier in (element, edge) order */
            int *nfi = a.fidx[1 - cur];
            unsigned char *nfl = a.flab[1 - cur];
            long long o2 = base;
            for (long long t0 = e0; t0 < e1; t0 += NT) {
                const long long i = t0 + threadIdx.x;
                unsigned won = i < e1 ? __ldcg(a.emask + i) : 0u;
                int off, tot;
                __syncthreads();
                Scan(sh.scan).ExclusiveSum(__popc(won), off, tot);
                if (won) {
                    const long long g = __ldcg(fi + i);
                    const int lab = __ldcg(fl + i);
                    const int val = __ldcg(a.table + g);
                    long long w = o2 + off;
                    while (won) {
                        const int e = __ffs(won) - 1;
                        won &= won - 1;
                        int dim, dir;
                        edge_of(lab, e, dim, dir);
                        const long long gp = g + dir * a.stride[dim];
                        a.table[gp] = val;
                        nfi[w] = (int) gp;
                        nfl[w] = (unsigned char) (2 * dim + 1 + (dir + 1) / 2);
                        w++;
                    }
                }
                o2 += tot;
            }
            n = next;
            cur = 1 - cur;
            levels++;
            if (!grid_barrier(a, 7)) return;
        }
    }
    if (a.fill_zeros) {                      /* fill_zeros, patchtable.h:2063-2079 */
        for (long long i = tid; i < a.ncells; i += nthr)
            if (__ldcg(a.table + i) == PT_UNUSED) a.table[i] = a.vfill;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) a.status[1] = levels;
}

std::atomic<long long> g_spin_limit{1ll << 24};

}  // namespace

long long pt_spin_limit() { return g_spin_limit.load(); }

extern "C" int64_t pt_set_spin_limit(int64_t polls) {
    if (polls < 0) polls = 1ll << 24;
    return g_spin_limit.exchange(polls);
}

pt_status pt_build_cells(const PtBins &bins, const int *nslices, const float *desc, int ds, long long P, const int *rank,
                         const int *to_bin, const int *order_xy, int *table, long long ncells, int run_dt, int dt_iters,
                         int fill_zeros, int vfill, long long *seeded, int *levels, cudaStream_t st) {
    if (ncells >= (1ll << 31)) return pt_fail(PT_UNSUPPORTED, "tables above 2^31 cells are not supported");
    if (bins.G < 1 || bins.G > PT_DESC_MAX) return pt_fail(PT_UNSUPPORTED, "grid dims %d", bins.G);
    int dev = 0, coop = 0, nsm = 0, per = 0;
    PT_CUDA(cudaGetDevice(&dev));
    PT_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop) return pt_fail(PT_UNSUPPORTED, "the table build needs cooperative launches");
    PT_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    PT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_table_build, NT, 0));
    if (per < 1) return pt_fail(PT_CUDA_ERR, "the table build kernel cannot be resident");
    const int grid = nsm * per;

    CellBuild a;
    memset(&a, 0, sizeof(a));
    a.G = bins.G;
    for (int d = 0; d < bins.G; d++) {
        a.min_val[d] = bins.min_val[d];
        a.range[d] = bins.range[d];
        a.stride[d] = bins.stride[d];
        a.nslices[d] = nslices[d];
    }
    a.desc = desc; a.ds = ds; a.P = P; a.rank = rank; a.to_bin = to_bin; a.order_xy = order_xy;
    a.table = table; a.ncells = ncells;
    a.run_dt = run_dt; a.dt_iters = dt_iters; a.fill_zeros = fill_zeros; a.vfill = vfill;
    a.spin_limit = pt_spin_limit();
    /* Scratch: claim keys and two frontiers of at most one element per cell. */
    DevBuf<unsigned> claim;
    DevBuf<int> fidx0, fidx1, status;
    DevBuf<unsigned char> flab0, flab1;
    DevBuf<unsigned> emask;
    DevBuf<long long> ctot, seed_n;
    DevBuf<unsigned> bar;
    if (run_dt) {
        PT_CUDA(claim.reserve(ncells));
        PT_CUDA(fidx0.reserve(ncells)); PT_CUDA(fidx1.reserve(ncells));
        PT_CUDA(flab0.reserve(ncells)); PT_CUDA(flab1.reserve(ncells));
        PT_CUDA(emask.reserve(ncells));
    }
    PT_CUDA(ctot.reserve(grid));
    PT_CUDA(seed_n.reserve(1));
    PT_CUDA(bar.reserve(2));
    PT_CUDA(status.reserve(4));
    PT_CUDA(cudaMemsetAsync(bar.p, 0, 2 * sizeof(unsigned), st));
    PT_CUDA(cudaMemsetAsync(status.p, 0, 4 * sizeof(int), st));
    a.claim = claim.p;
    a.fidx[0] = fidx0.p; a.fidx[1] = fidx1.p;
    a.flab[0] = flab0.p; a.flab[1] = flab1.p;
    a.emask = emask.p;
    a.ctot = ctot.p;
    a.bar = bar.p;
    a.status = status.p;
    a.seeded = seed_n.p;
    void *args[] = {&a};
    PT_CUDA(cudaLaunchCooperativeKernel((const void *) k_table_build, grid, NT, args, 0, st));
    PT_LAUNCHED();
    int hs[4] = {0, 0, 0, 0};
    long long hn = 0;
    PT_CUDA(cudaMemcpyAsync(hs, status.p, sizeof(hs), cudaMemcpyDeviceToHost, st));
    PT_CUDA(cudaMemcpyAsync(&hn, seed_n.p, sizeof(hn), cudaMemcpyDeviceToHost, st));
    PT_CUDA(cudaStreamSynchronize(st));
    if (hs[0] == PT_TIMEOUT)
        return pt_fail(PT_TIMEOUT, "table build: a grid barrier wait gave up after %lld polls (phase %d)", a.spin_limit, hs[2]);
    if (hs[0] != 0) return pt_fail((pt_status) hs[0], "table build: a DT frontier reached 2^27 elements");
    if (seeded) *seeded = hn;
    if (levels) *levels = hs[1];
    return PT_OK;
}
