/* Host side of the PatchTable build and query (the C ABI of include/patchtable_b200.h).

   Build, PatchTableFixedN constructor (patchtable/patchtable.h:2584-3373), on the device:
     descriptor of b -> per-dimension range -> slice counts (host, scale_slices_to_limit)
     -> quantile centres (device sort, host arithmetic) and to_bin tables (host)
     -> k-coherence set -> populate in the reference's random_shuffle order -> DT.
   Query, lookup_templated (patchtable.h:3468-4217): descriptor of a -> cell of every patch
     -> choose / pull passes -> float64 NNF.

   The host keeps only parameters, partition arrays and shapes; images, descriptors, the table
   and the k-coherence set stay in device memory for the table's lifetime. */
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "patchtable_b200.h"
#include "pt_internal.h"
#include "pt_kernels.h"

namespace {

thread_local std::string g_last_error;
thread_local long long g_launches = 0;

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

/* scale_slices_to_limit, patchtable.cpp:611-642 (product/multiply: solver/util.cpp:186-205). */
std::vector<int> scale_slices_to_limit(std::vector<int> nslices, double limit) {
    auto product = [](const std::vector<int> &L) { double a = 1.0; for (int v : L) a *= v; return a; };
    if (limit > 0) {
        std::vector<int> nslices0(nslices);
        double factor = 1.0;
        for (auto &v : nslices) v = std::max(v, 1);
        while (product(nslices) > limit) {
            factor *= 0.995;
            for (size_t i = 0; i < nslices.size(); i++) nslices[i] = (int) (nslices0[i] * factor + 0.5);
            for (auto &v : nslices) v = std::max(v, 1);
        }
        for (;;) {
            nslices0 = nslices;
            bool success = false;
            for (size_t i = 0; i < nslices.size(); i++) {
                nslices[i]++;
                if (product(nslices) > limit) nslices = nslices0;
                else { success = true; nslices0 = nslices; }
            }
            if (!success) break;
        }
    }
    return nslices;
}

}  // namespace

pt_status pt_fail(pt_status s, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return s;
}

void pt_count_launches(int n) { g_launches += n; }

namespace {
std::atomic<long long> g_alloc_live{0};
std::atomic<long long> g_alloc_limit{-1};
}  // namespace

bool pt_alloc_admit(size_t bytes) {
    const long long lim = g_alloc_limit.load();
    const long long now = g_alloc_live.fetch_add((long long) bytes) + (long long) bytes;
    if (lim >= 0 && now > lim) {
        g_alloc_live.fetch_sub((long long) bytes);
        return false;
    }
    return true;
}

void pt_alloc_release(size_t bytes) { g_alloc_live.fetch_sub((long long) bytes); }

extern "C" int64_t pt_set_device_alloc_limit(int64_t bytes) { return g_alloc_limit.exchange(bytes < 0 ? -1 : bytes); }

extern "C" int64_t pt_device_bytes_in_use(void) { return g_alloc_live.load(); }

struct pt_table {
    pt_params p;
    int h = 0, w = 0, eh = 0, ew = 0;
    int nd = 0, G = 0, ds = 8;
    /* Descriptor mode (is_descriptor): b and the queries are descriptor images and h x w is the
       virtual image whose (h-7) x (w-7) patches are their pixels (get_padded_descriptor,
       patchtable.h:2498-2507); no RGB copy of b exists. */
    bool desc_mode = false;
    int in_padded = 0;
    /* -dim_algo pca: the basis fitted on b (patch_pca.h), used for b and every query */
    bool pca = false;
    DevBuf<float> pca_mean, pca_basis;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    cudaStream_t st2 = nullptr;       /* the build's second stream (range and partition) */
    DevBuf<float4> b_rgba;
    DevBuf<float4> b_rgba1;           /* b_rgba shifted by one pixel, b_rgba1[i] = b_rgba[i + 1] */
    DevBuf<float> b_desc;
    DevBuf<int> allowed;
    std::vector<int> nslices;
    std::vector<long long> stride;
    long long ncells = 0;
    std::vector<PtPartition> part;
    std::vector<float> min_val, max_val, range;
    PtBins bins;
    DevBuf<int> to_bin;
    DevBuf<float> part_dev;           /* per grid dimension: centres, lsizes, rsizes (proposal features) */
    int part_ofs[PT_DESC_MAX] = {};
    DevBuf<int> table;
    long long add_count = 0;
    int dt_levels = 0;
    /* wall-clock milliseconds of the build stages (pt_table_build_profile) */
    double build_ms[PT_BUILD_NSTAGES] = {};
    DevBuf<int2> kcoh;
    int kc_list = 0;
    /* ntables > 1: the further tables at limit / table_ratio^i (patchtable.h:3359-3371) and their
       entries for the current query, [table][patch] */
    std::vector<std::unique_ptr<pt_table>> subs;
    DevBuf<int> q_tcand_more;
    /* query scratch, reused across lookups (like lookup_buffer/lookup_wh, patchtable.h:1507-1509) */
    DevBuf<float> q_rgb;
    DevBuf<float4> q_rgba;
    DevBuf<float> q_desc;
    DevBuf<int> q_tcand;
    DevBuf<int> q_pos[2], q_chpos, q_kcdone;
    DevBuf<float> q_d[2], q_chd;
    DevBuf<double> q_ann;
    DevBuf<int> q_lcand;              /* learned proposals, P x PT_PROP_TOPK */
    DevBuf<double> q_prev, q_torig;   /* temporal lookups: previous NNF (host path), restored distances */
    DevBuf<float> q_sv, q_td0;
    DevBuf<int> q_tpos0, q_tbad;
    DevBuf<float> q_lconf;
    DevBuf<unsigned long long> q_counters;
    std::vector<cudaEvent_t> events;
    cudaStream_t st_in = nullptr, st_out = nullptr;    /* banded host lookups: upload / download */
    cudaStream_t st_choose = nullptr, st_pull = nullptr; /* banded host lookups: later phases */
    std::vector<cudaEvent_t> band_ev;
    PinnedBuf<int> h_pos;             /* banded host lookups: packed field downloaded per band */
    PinnedBuf<float> h_in;            /* banded host lookups: a pageable query image, staged per band */
    PinnedBuf<float> h_d;
    long long last_h2d = 0, last_d2h = 0;   /* bytes copied by the last host lookup */

    ~pt_table() {
        for (auto e : events) cudaEventDestroy(e);
        for (auto e : band_ev) cudaEventDestroy(e);
        if (st_in) cudaStreamDestroy(st_in);
        if (st_out) cudaStreamDestroy(st_out);
        if (st_choose) cudaStreamDestroy(st_choose);
        if (st_pull) cudaStreamDestroy(st_pull);
        if (own_stream && st) cudaStreamDestroy(st);
        if (st2) cudaStreamDestroy(st2);
    }
};

namespace {

pt_status check_params(const pt_params *p, int h, int w) {
    if (!p) return pt_fail(PT_BAD_ARG, "null params");
    if (p->patch_w != 8) return pt_fail(PT_UNSUPPORTED, "patch_w=%d: only 8x8 patches are supported (gck.h)", p->patch_w);
    if (h < 8 || w < 8) return pt_fail(PT_BAD_ARG, "image %dx%d is smaller than one 8x8 patch", w, h);
    if (w > 65535 || h > 16383) return pt_fail(PT_BAD_ARG, "image %dx%d exceeds the packed position range (XY_TO_INT)", w, h);
    if (p->dim_algo == 1 && (p->is_descriptor || p->pca_mean))
        return pt_fail(PT_UNSUPPORTED, "dim_algo pca with %s is not implemented on the GPU path",
                       p->is_descriptor ? "is_descriptor" : "pca_mean");
    if (p->dim_algo != 0 && p->dim_algo != 1) return pt_fail(PT_BAD_ARG, "dim_algo %d", p->dim_algo);
    if (p->convert_colorspace && p->colorspace != 0 && p->colorspace != 1)
        return pt_fail(PT_BAD_ARG, "colorspace %d", p->colorspace);
    if (p->lookup_algo != 0) return pt_fail(PT_UNSUPPORTED, "only lookup_algo table is implemented on the GPU path");
    if (p->kcoherence && p->kcoherence_algo != 0) return pt_fail(PT_UNSUPPORTED, "only kcoherence_algo flann (exact search) is implemented");
    if (p->incoherence) return pt_fail(PT_UNSUPPORTED, "incoherence is not implemented on the GPU path");
    /* randomize_dt and populate_nearest change nothing in the reference's build: with
       TABLE_POPULATE_FAST (patchtable.h:37) populate never calls add_patch (patchtable.h:3127-3159),
       so no adjacency is collected and do_after_dt (patchtable.h:1831-1866) keeps every cell. */
    if (p->ntables > 16) return pt_fail(PT_UNSUPPORTED, "ntables %d > 16", p->ntables);
    if (p->run_dt && p->dt_algo != 1 && p->dt_algo != 2 && p->dt_algo != 4 && p->dt_algo != 5 && p->dt_algo != 6)
        return pt_fail(PT_UNSUPPORTED, "dt_algo %d is not implemented on the GPU path", p->dt_algo);
    if (p->ndims < 1 || p->ndims > PT_DESC_MAX) return pt_fail(PT_UNSUPPORTED, "ndims %d outside 1..%d", p->ndims, PT_DESC_MAX);
    int G = p->grid_ndims < 0 ? p->ndims : p->grid_ndims;
    if (G < 1 || G > p->ndims) return pt_fail(PT_BAD_ARG, "grid_ndims %d outside 1..ndims", G);
    if (p->partition_step < 1 || p->kcoherence_step < 1 || p->flann_build_step < 1 || p->flann_reset_step < 1)
        return pt_fail(PT_BAD_ARG, "step parameters must be >= 1");
    return PT_OK;
}

pt_status upload_partition(pt_table *t, cudaStream_t st);

pt_status build_partition(pt_table *t, PtPartScratch &scratch, cudaStream_t st) {
    const int G = t->G;
    t->part.assign(G, PtPartition());
    for (int d = 0; d < G; d++) {
        PtPartition &P = t->part[d];
        int ns = t->nslices[d];
        P.nslices = ns;
        P.min_val = t->min_val[d];
        P.max_val = t->max_val[d];
        P.range = P.max_val - P.min_val;
        /* Count the partition sample first, then fetch the quantile values
           (PatchPartition1D, patchtable.h:1193-1201). */
        int N = 0;
        std::vector<float> vals;
        PT_TRY(pt_quantile_gather(scratch, t->b_desc.p, t->ds, d, t->eh, t->ew, t->p.partition_step, t->allowed.p,
                                  t->p.allowed_index, &N, st));
        if (N < 1) return pt_fail(PT_BAD_ARG, "no allowed patches to build a table from");
        std::vector<int> want;
        want.reserve(2 * ns);
        for (int i = 0; i < ns; i++) {
            want.push_back((int) ((long long) (N - 1) * i / ns));
            want.push_back((int) ((long long) (N - 1) * (i + 1) / ns));
        }
        PT_TRY(pt_quantile_pick(scratch, N, want, vals, st));
        P.centers.resize(ns);
        P.lsizes.resize(ns);
        P.rsizes.resize(ns);
        for (int i = 0; i < ns; i++) {
            float cell_min = vals[2 * i], cell_max = vals[2 * i + 1];
            P.centers[i] = (cell_min + cell_max) / 2;
        }
        for (int i = 0; i < ns; i++) {            /* patchtable.h:1203-1215 */
            float prev_center = (i - 1 >= 0) ? P.centers[i - 1] : P.min_val;
            float next_center = (i + 1 < ns) ? P.centers[i + 1] : P.max_val;
            P.lsizes[i] = P.centers[i] - prev_center;
            if (i - 1 >= 0) P.lsizes[i] /= 2;
            P.rsizes[i] = next_center - P.centers[i];
            if (i + 1 < ns) P.rsizes[i] /= 2;
        }
        P.to_bin.resize(PT_NMAP);                  /* patchtable.h:1219-1256 */
        int icenter = 0;
        for (int i = 0; i < PT_NMAP; i++) {
            double coord = P.min_val + (i + 0.5) * P.range / PT_NMAP;
            while (coord > P.centers[icenter]) {
                if (icenter + 1 < ns) icenter++;
                else break;
            }
            int prev_c = icenter - 1;
            if (prev_c < 0) prev_c = 0;
            int next_c = icenter;
            if (next_c == 0) next_c++;
            if (ns == 1) next_c = prev_c = 0;
            double mid = (P.centers[prev_c] + P.centers[next_c]) / 2.0;
            P.to_bin[i] = (coord < mid) ? prev_c : next_c;
        }
    }
    return upload_partition(t, st);
}

/* Device copies of the partition: the to_bin tables, the centres / sizes the proposal features
   read, and the per-dimension get_bin parameters. */
pt_status upload_partition(pt_table *t, cudaStream_t st) {
    const int G = t->G;
    std::vector<int> flat((size_t) G * PT_NMAP);
    for (int d = 0; d < G; d++) std::copy(t->part[d].to_bin.begin(), t->part[d].to_bin.end(), flat.begin() + (size_t) d * PT_NMAP);
    PT_CUDA(t->to_bin.reserve(flat.size()));
    PT_CUDA(cudaMemcpyAsync(t->to_bin.p, flat.data(), sizeof(int) * flat.size(), cudaMemcpyHostToDevice, st));
    {
        std::vector<float> pd;
        for (int d = 0; d < G; d++) {
            const PtPartition &P = t->part[d];
            t->part_ofs[d] = (int) pd.size();
            pd.insert(pd.end(), P.centers.begin(), P.centers.end());
            pd.insert(pd.end(), P.lsizes.begin(), P.lsizes.end());
            pd.insert(pd.end(), P.rsizes.begin(), P.rsizes.end());
        }
        PT_CUDA(t->part_dev.reserve(pd.size()));
        PT_CUDA(cudaMemcpyAsync(t->part_dev.p, pd.data(), sizeof(float) * pd.size(), cudaMemcpyHostToDevice, st));
        PT_CUDA(cudaStreamSynchronize(st));
    }
    memset(&t->bins, 0, sizeof(t->bins));
    t->bins.G = G;
    for (int d = 0; d < G; d++) {
        t->bins.min_val[d] = t->part[d].min_val;
        t->bins.range[d] = t->part[d].range;
        t->bins.stride[d] = t->stride[d];
    }
    return PT_OK;
}

/* Whether a host pointer is page-locked (cudaHostAlloc / cudaHostRegister / pinned tensors). */
bool host_pinned(const void *p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) == cudaSuccess) return at.type == cudaMemoryTypeHost;
    cudaGetLastError();
    return false;
}

bool host_allowed(const std::vector<int> &allowed, int idx, int py, int px, int ew) {
    return allowed.empty() || allowed[(size_t) py * ew + px] == idx;
}

pt_status build_kcoherence(pt_table *t, const std::vector<int> &allowed) {
    const pt_params &p = t->p;
    const int ew = t->ew, eh = t->eh;
    {
        /* The lists are generated on the device (no host loops or copies): regular grids without
           a mask, the same grids compacted to the allowed points with one. */
        const long long P = (long long) eh * ew;
        DevBuf<int> d_trows, d_tpos, d_qrows, d_qpos, d_qcell, d_seg;
        PT_CUDA(d_trows.reserve(P)); PT_CUDA(d_tpos.reserve(P));
        PT_CUDA(d_qrows.reserve(P)); PT_CUDA(d_qpos.reserve(P)); PT_CUDA(d_qcell.reserve(P)); PT_CUDA(d_seg.reserve(P + 1));
        int N = 0, Q = 0, nseg = 0;
        const pt_status lst =
            allowed.empty()
                ? pt_kc_lists(ew, eh, p.flann_build_step, p.kcoherence_step, p.flann_reset_step, d_trows.p, d_tpos.p,
                              d_qrows.p, d_qpos.p, d_qcell.p, d_seg.p, &N, &Q, &nseg, t->st)
                : pt_kc_lists_masked(ew, eh, p.flann_build_step, p.kcoherence_step, p.flann_reset_step, t->allowed.p,
                                     p.allowed_index, d_trows.p, d_tpos.p, d_qrows.p, d_qpos.p, d_qcell.p, d_seg.p, &N,
                                     &Q, &nseg, t->st);
        if (lst == PT_OK) {
            PT_CUDA(t->kcoh.reserve((size_t) P * p.kcoherence));
            PT_CUDA(cudaMemsetAsync(t->kcoh.p, 0, sizeof(int2) * (size_t) P * p.kcoherence, t->st));
            if (Q == 0) return PT_OK;
            DevBuf<float> train, qdesc;
            PT_CUDA(train.reserve((size_t) N * t->nd)); PT_CUDA(qdesc.reserve((size_t) Q * t->nd));
            PT_TRY(pt_gather_rows(t->b_desc.p, t->ds, t->nd, d_trows.p, N, train.p, t->st));
            PT_TRY(pt_gather_rows(t->b_desc.p, t->ds, t->nd, d_qrows.p, Q, qdesc.p, t->st));
            return pt_kcoherence(t->b_rgba.p, t->w, t->desc_mode ? t->b_desc.p : nullptr, t->ds, t->ew, train.p, N, t->nd,
                                 d_tpos.p, qdesc.p, d_qpos.p, d_qcell.p, Q, d_seg.p, nseg, p.kcoherence,
                                 p.kcoherence_min_dist, t->kcoh.p, &t->kc_list, t->st);
        }
    }
    /* Train set: build_flann_index_func (patchtable.h:822-861), allowed patches every
       flann_build_step pixels in raster order. */
    std::vector<int> trows, tpos;
    for (int y = 0; y < eh; y += p.flann_build_step)
        for (int x = 0; x < ew; x += p.flann_build_step)
            if (host_allowed(allowed, p.allowed_index, y, x, ew)) { trows.push_back(y * ew + x); tpos.push_back(pt_xy(x, y)); }
    /* Queries in the reference's loop order (patchtable.h:2705-2713) and the knn reset segments
       ((x / kcoherence_step) % flann_reset_step == 0 with x in padded coordinates, :2714). */
    std::vector<int> qrows, qpos, qcell, seg;
    int ks = p.kcoherence_step;
    for (int y = 7; y < t->h; y += ks)
        for (int x = 7; x < t->w; x += ks) {
            int py = y - 7, px = x - 7;
            if (!host_allowed(allowed, p.allowed_index, py, px, ew)) continue;
            int q = (int) qrows.size();
            if (q == 0 || (x / ks) % p.flann_reset_step == 0) seg.push_back(q);
            qrows.push_back(py * ew + px);
            qpos.push_back(pt_xy(px, py));
            qcell.push_back((py / ks) * ew + px / ks);
        }
    int N = (int) trows.size(), Q = (int) qrows.size(), nseg = (int) seg.size();
    PT_CUDA(t->kcoh.reserve((size_t) eh * ew * p.kcoherence));
    PT_CUDA(cudaMemsetAsync(t->kcoh.p, 0, sizeof(int2) * (size_t) eh * ew * p.kcoherence, t->st));
    if (Q == 0) return PT_OK;
    DevBuf<int> d_trows, d_tpos, d_qrows, d_qpos, d_qcell, d_seg;
    DevBuf<float> train, qdesc;
    PT_CUDA(d_trows.reserve(N)); PT_CUDA(d_tpos.reserve(N));
    PT_CUDA(d_qrows.reserve(Q)); PT_CUDA(d_qpos.reserve(Q)); PT_CUDA(d_qcell.reserve(Q)); PT_CUDA(d_seg.reserve(nseg));
    PT_CUDA(train.reserve((size_t) N * t->nd)); PT_CUDA(qdesc.reserve((size_t) Q * t->nd));
    PT_CUDA(cudaMemcpyAsync(d_trows.p, trows.data(), sizeof(int) * N, cudaMemcpyHostToDevice, t->st));
    PT_CUDA(cudaMemcpyAsync(d_tpos.p, tpos.data(), sizeof(int) * N, cudaMemcpyHostToDevice, t->st));
    PT_CUDA(cudaMemcpyAsync(d_qrows.p, qrows.data(), sizeof(int) * Q, cudaMemcpyHostToDevice, t->st));
    PT_CUDA(cudaMemcpyAsync(d_qpos.p, qpos.data(), sizeof(int) * Q, cudaMemcpyHostToDevice, t->st));
    PT_CUDA(cudaMemcpyAsync(d_qcell.p, qcell.data(), sizeof(int) * Q, cudaMemcpyHostToDevice, t->st));
    PT_CUDA(cudaMemcpyAsync(d_seg.p, seg.data(), sizeof(int) * nseg, cudaMemcpyHostToDevice, t->st));
    PT_TRY(pt_gather_rows(t->b_desc.p, t->ds, t->nd, d_trows.p, N, train.p, t->st));
    PT_TRY(pt_gather_rows(t->b_desc.p, t->ds, t->nd, d_qrows.p, Q, qdesc.p, t->st));
    PT_TRY(pt_kcoherence(t->b_rgba.p, t->w, t->desc_mode ? t->b_desc.p : nullptr, t->ds, t->ew, train.p, N, t->nd,
                         d_tpos.p, qdesc.p, d_qpos.p, d_qcell.p, Q, d_seg.p, nseg, p.kcoherence, p.kcoherence_min_dist,
                         t->kcoh.p, &t->kc_list, t->st));
    return PT_OK;
}

pt_status create_impl(const pt_params *pin, const float *b, int h, int w, int channels, const float *wh0,
                      const int32_t *allowed, pt_table **out) {
    if (!out) return pt_fail(PT_BAD_ARG, "null output pointer");
    *out = nullptr;
    if (!b) return pt_fail(PT_BAD_ARG, "null image");
    /* Descriptor mode takes ndims from the input and no chroma (patchtable.h:4398-4401); its
       patches are the input's pixels, so the build runs on the virtual image around them. */
    pt_params pd = *pin;
    int vh = h, vw = w;
    if (pin->is_descriptor) {
        if (wh0) return pt_fail(PT_UNSUPPORTED, "a precomputed padded descriptor in descriptor mode");
        if (channels < 3 || channels > PT_DESC_MAX)
            return pt_fail(PT_UNSUPPORTED, "descriptor mode with %d channels (3..%d are supported)", channels, PT_DESC_MAX);
        pd.ndims = channels;
        pd.nchroma = 0;
        vh = pin->descriptor_padded ? h - 7 : h + 7;
        vw = pin->descriptor_padded ? w - 7 : w + 7;
    } else if (channels != 3) {
        return pt_fail(PT_BAD_ARG, "expected a 3-channel RGB image, got %d channels", channels);
    }
    PT_TRY(check_params(&pd, vh, vw));
    std::unique_ptr<pt_table> t(new pt_table());
    t->p = pd;
    pt_params &p = t->p;
    if (p.grid_ndims < 0) p.grid_ndims = p.ndims;          /* patchtable.h:2603 */
    t->h = vh; t->w = vw; t->eh = vh - 7; t->ew = vw - 7;
    t->nd = p.ndims; t->G = p.grid_ndims;
    t->ds = p.ndims <= 8 ? 8 : 16;
    t->desc_mode = p.is_descriptor != 0;
    t->in_padded = p.descriptor_padded;
    if (!t->desc_mode && p.dim_algo == 0) PT_TRY(pt_descriptor_check(p.ndims, p.nchroma));
    PT_CUDA(cudaStreamCreateWithFlags(&t->st, cudaStreamNonBlocking));
    t->own_stream = true;
    const long long P = (long long) t->eh * t->ew;
    /* stage clock: every stage ends with the stream drained */
    const double t_start = now_s();
    double t_mark = t_start;
    auto stage_done = [&](int k) -> pt_status {
        PT_CUDA(cudaStreamSynchronize(t->st));
        const double t1 = now_s();
        t->build_ms[k] += 1000.0 * (t1 - t_mark);
        t_mark = t1;
        return PT_OK;
    };

    if (t->desc_mode) {
        DevBuf<float> in;
        const size_t nin = (size_t) h * w * channels;
        PT_CUDA(in.reserve(nin));
        PT_CUDA(cudaMemcpyAsync(in.p, b, sizeof(float) * nin, cudaMemcpyHostToDevice, t->st));
        PT_CUDA(t->b_desc.reserve((size_t) P * t->ds));
        PT_TRY(pt_launch_descriptor_input(in.p, h, w, channels, t->in_padded, t->b_desc.p, t->ds, t->st));
        PT_CUDA(cudaStreamSynchronize(t->st));
    } else {
    /* Descriptor of b (get_padded_descriptor, patchtable.h:2492-2546) and the RGBA copy kept as b0. */
        DevBuf<float> rgb;
        PT_CUDA(rgb.reserve((size_t) h * w * 3));
        PT_CUDA(cudaMemcpyAsync(rgb.p, b, sizeof(float) * (size_t) h * w * 3, cudaMemcpyHostToDevice, t->st));
        PT_CUDA(t->b_rgba.reserve((size_t) h * w));
        PT_CUDA(t->b_desc.reserve((size_t) P * t->ds));
        if (p.dim_algo == 1) {
            /* reduce_dim with TABLE_DIM_ALGO_PCA (patchtable.h:1709-1713): fit on b, then project */
            std::vector<float> mean, basis;
            PT_TRY(pt_pca_fit(b, h, w, pt_color_mode(p), p.pca_samples, p.pca_subtract_mean, p.ndims, mean, basis));
            t->pca = true;
            PT_CUDA(t->pca_mean.reserve(mean.size()));
            PT_CUDA(t->pca_basis.reserve(basis.size()));
            PT_CUDA(cudaMemcpyAsync(t->pca_mean.p, mean.data(), sizeof(float) * mean.size(), cudaMemcpyHostToDevice, t->st));
            PT_CUDA(cudaMemcpyAsync(t->pca_basis.p, basis.data(), sizeof(float) * basis.size(), cudaMemcpyHostToDevice, t->st));
            PT_TRY(pt_launch_pca(rgb.p, h, w, pt_color_mode(p), t->b_rgba.p, t->pca_mean.p, t->pca_basis.p, p.ndims,
                                 t->b_desc.p, t->ds, t->st));
            PT_CUDA(cudaStreamSynchronize(t->st));     /* the host vectors go out of scope */
        } else {
            PT_TRY(pt_launch_descriptor(p.ndims, p.nchroma, rgb.p, h, w, pt_color_mode(p), t->b_rgba.p, t->b_desc.p,
                                        t->ds, t->st));
        }
        if (wh0) {
            /* Caller-supplied padded descriptor (wh0_no_copy): interior patches only. */
            std::vector<float> packed((size_t) P * t->ds, 0.0f);
            for (int y = 0; y < t->eh; y++)
                for (int x = 0; x < t->ew; x++)
                    for (int d = 0; d < t->nd; d++)
                        packed[((size_t) y * t->ew + x) * t->ds + d] = wh0[((size_t) (y + 7) * (w + 7) + (x + 7)) * t->nd + d];
            PT_CUDA(cudaMemcpyAsync(t->b_desc.p, packed.data(), sizeof(float) * packed.size(), cudaMemcpyHostToDevice, t->st));
        }
        /* The query reads b patch rows with 32-byte loads: from b_rgba at even pixel indices and
           from this one-pixel-shifted copy at odd ones, so every load is 32-byte aligned. */
        const size_t npx = (size_t) h * w;
        PT_CUDA(t->b_rgba1.reserve(npx));
        PT_CUDA(cudaMemsetAsync(t->b_rgba1.p, 0, sizeof(float4) * npx, t->st));
        PT_CUDA(cudaMemcpyAsync(t->b_rgba1.p, t->b_rgba.p + 1, sizeof(float4) * (npx - 1), cudaMemcpyDeviceToDevice, t->st));
        PT_CUDA(cudaStreamSynchronize(t->st));
    }
    std::vector<int> allowed_h;
    if (allowed) {
        allowed_h.assign(allowed, allowed + P);
        PT_CUDA(t->allowed.reserve(P));
        PT_CUDA(cudaMemcpyAsync(t->allowed.p, allowed, sizeof(int) * P, cudaMemcpyHostToDevice, t->st));
    }
    PT_TRY(stage_done(PT_BUILD_DESCRIPTOR));

    /* Three independent steps run at once, each on its own host thread: the k-coherence set on the
       table's stream (computed before the table in the reference, patchtable.h:2653), the range and
       partition on a second stream, and the populate order on the host.  Only the populate order
       draws from rand(), as the reference's does at this point; nothing else draws meanwhile. */
    auto timed = [](double &ms, auto &&fn) -> pt_status {
        const double t0 = now_s();
        const pt_status r = fn();
        ms = 1000.0 * (now_s() - t0);
        return r;
    };
    /* Populate in std::random_shuffle order (patchtable.h:3142-3154): the permutation is drawn
       from the C library rand(), consuming it exactly as the reference does. */
    std::vector<int> order_xy, rank(P, -1);
    double shuffle_ms = 0.0;
    std::thread shuffler([&] {
        const double t0 = now_s();
        order_xy.reserve(P);
        for (int y = 0; y < t->eh; y++)
            for (int x = 0; x < t->ew; x++)
                if (host_allowed(allowed_h, p.allowed_index, y, x, t->ew)) order_xy.push_back(pt_xy(x + 7, y + 7));
        if (p.populate_random)
            for (size_t i = 1; i < order_xy.size(); i++) {
                size_t j = (size_t) (rand() % (int) (i + 1));
                if (i != j) std::swap(order_xy[i], order_xy[j]);
            }
        for (size_t i = 0; i < order_xy.size(); i++) {
            int v = order_xy[i];
            rank[(size_t) (pt_y(v) - 7) * t->ew + (pt_x(v) - 7)] = (int) i;
        }
        shuffle_ms = 1000.0 * (now_s() - t0);
    });
    /* set_min_max + set_nslices (patchtable.h:1758-1810, 2567-2582), then the partition */
    if (!t->st2) {
        /* highest priority: the partition's short kernels take SMs as the k-NN search's CTAs
           retire instead of queueing behind the whole search */
        int least = 0, greatest = 0;
        cudaDeviceGetStreamPriorityRange(&least, &greatest);
        cudaError_t e = cudaStreamCreateWithPriority(&t->st2, cudaStreamNonBlocking, greatest);
        if (e != cudaSuccess) { shuffler.join(); return pt_fail(PT_CUDA_ERR, "stream: %s", cudaGetErrorString(e)); }
    }
    double part_ms = 0.0;
    PtPartScratch part_scratch;       /* freed when the build returns, after the search has ended */
    std::string part_err;
    pt_status part_st = PT_OK;
    std::thread partitioner([&] {
        part_st = timed(part_ms, [&]() -> pt_status {
            cudaStream_t s2 = t->st2;
            t->min_val.assign(t->G, 0.f);
            t->max_val.assign(t->G, 0.f);
            PT_TRY(pt_launch_minmax(part_scratch, t->b_desc.p, t->ds, t->G, P, t->allowed.p, p.allowed_index, t->min_val.data(),
                                    t->max_val.data(), s2));
            t->range.resize(t->G);
            for (int d = 0; d < t->G; d++) t->range[d] = t->max_val[d] - t->min_val[d];
            std::vector<int> ns(t->G);
            if (p.n_nslices == 0) {
                float max_range = t->range[0];
                for (int d = 1; d < t->G; d++) if (t->range[d] > max_range) max_range = t->range[d];
                double scale = 200.0 / max_range;
                for (int d = 0; d < t->G; d++) ns[d] = (int) (t->range[d] * scale);
            } else {
                if (p.n_nslices != t->G) return pt_fail(PT_BAD_ARG, "-nslices has %d entries, grid has %d dims", p.n_nslices, t->G);
                for (int d = 0; d < t->G; d++) ns[d] = p.nslices[d];
            }
            t->nslices = scale_slices_to_limit(ns, p.limit);
            t->stride.assign(t->G, 1);
            t->ncells = 1;
            for (int d = t->G - 1; d >= 0; d--) { t->stride[d] = t->ncells; t->ncells *= t->nslices[d]; }
            if (t->ncells >= (1ll << 31)) return pt_fail(PT_UNSUPPORTED, "table of %lld cells exceeds 2^31", t->ncells);
            PT_TRY(build_partition(t.get(), part_scratch, s2));
            PT_CUDA(cudaStreamSynchronize(s2));
            return PT_OK;
        });
        if (part_st != PT_OK) part_err = pt_last_error();
    });
    pt_status kc_st = PT_OK;
    if (p.kcoherence > 0) kc_st = build_kcoherence(t.get(), allowed_h);
    if (kc_st == PT_OK) kc_st = stage_done(PT_BUILD_KCOHERENCE);
    partitioner.join();
    shuffler.join();
    t_mark = now_s();
    if (kc_st != PT_OK) return kc_st;
    if (part_st != PT_OK) return pt_fail(part_st, "%s", part_err.c_str());
    t->build_ms[PT_BUILD_PARTITION] = part_ms;
    t->build_ms[PT_BUILD_SHUFFLE] = shuffle_ms;
    if (order_xy.empty()) return pt_fail(PT_BAD_ARG, "no allowed patches");
    {
        DevBuf<int> d_rank, d_order;
        PT_CUDA(d_rank.reserve(P));
        PT_CUDA(d_order.reserve(order_xy.size()));
        PT_CUDA(cudaMemcpyAsync(d_rank.p, rank.data(), sizeof(int) * P, cudaMemcpyHostToDevice, t->st));
        PT_CUDA(cudaMemcpyAsync(d_order.p, order_xy.data(), sizeof(int) * order_xy.size(), cudaMemcpyHostToDevice, t->st));
        PT_CUDA(t->table.reserve(t->ncells));
        /* Distance transform (patchtable.h:3254-3298): prop is the level-synchronous fill inside
           the cooperative build launch; the others run on its resolved table. */
        const bool prop = p.run_dt && p.dt_algo == 1;
        /* fill_zeros (patchtable.h:2063-2079) after no DT or a prop DT cut short by dt_iters */
        const bool fill_zeros = !p.run_dt || (prop && p.dt_iters > 0);
        int vfill = pt_xy(7, 7);
        if (!allowed_h.empty())
            for (long long i = 0; i < P; i++)
                if (allowed_h[i] == p.allowed_index) { vfill = pt_xy((int) (i % t->ew) + 7, (int) (i / t->ew) + 7); break; }
        PT_TRY(pt_build_cells(t->bins, t->nslices.data(), t->b_desc.p, t->ds, P, d_rank.p, t->to_bin.p, d_order.p,
                              t->table.p, t->ncells, prop, p.dt_iters, fill_zeros, vfill, &t->add_count, &t->dt_levels,
                              t->st));
        if (p.run_dt && p.dt_algo == 2)
            PT_TRY(pt_dt_brute(t->table.p, t->G, t->nslices.data(), t->part_dev.p, t->part_ofs, t->b_desc.p, t->ds, P, t->ew,
                               t->st));
        else if (p.run_dt && !prop)
            PT_TRY(pt_dt_other(t->table.p, t->G, t->nslices.data(), p.dt_algo, t->st));
        PT_CUDA(cudaStreamSynchronize(t->st));
    }
    PT_TRY(stage_done(PT_BUILD_POPULATE_DT));
    t->build_ms[PT_BUILD_TOTAL] = 1000.0 * (now_s() - t_start);
    *out = t.release();
    return PT_OK;
}

/* Input dimensions of a query on the virtual image h x w (descriptor mode) and the floats it holds. */
void query_input_dims(const pt_table *t, int h, int w, int &ih, int &iw, size_t &floats) {
    if (t->desc_mode) {
        ih = t->in_padded ? h + 7 : h - 7;
        iw = t->in_padded ? w + 7 : w - 7;
        floats = (size_t) ih * iw * t->nd;
    } else {
        ih = h; iw = w;
        floats = (size_t) h * w * 3;
    }
}

/* The virtual image of a query input of h x w (pixels or descriptors). */
pt_status query_dims(const pt_table *t, int h, int w, int &vh, int &vw) {
    if (t->desc_mode) {
        vh = t->in_padded ? h - 7 : h + 7;
        vw = t->in_padded ? w - 7 : w + 7;
    } else {
        vh = h; vw = w;
    }
    if (vh < 8 || vw < 8) return pt_fail(PT_BAD_ARG, "query %dx%d holds no patch", w, h);
    return PT_OK;
}

pt_status ensure_query_buffers(pt_table *t, int h, int w) {
    long long P = (long long) (h - 7) * (w - 7);
    int ih, iw;
    size_t in_floats;
    query_input_dims(t, h, w, ih, iw, in_floats);
    PT_CUDA(t->q_rgb.reserve(std::max((size_t) h * w * 3, in_floats)));
    PT_CUDA(t->q_rgba.reserve((size_t) h * w));
    PT_CUDA(t->q_desc.reserve((size_t) P * t->ds));
    PT_CUDA(t->q_tcand.reserve(P));
    for (int k = 0; k < 2; k++) { PT_CUDA(t->q_pos[k].reserve(P)); PT_CUDA(t->q_d[k].reserve(P)); }
    PT_CUDA(t->q_chpos.reserve(P));
    PT_CUDA(t->q_kcdone.reserve(P));
    PT_CUDA(t->q_chd.reserve(P));
    PT_CUDA(t->q_counters.reserve(6));
    return PT_OK;
}

/* Stage timing of one lookup (pt_table_lookup_profile). */
struct LookupProfile {
    enum { DESC, CELLS, INIT, CHOOSE, PULL, OUTPUT, PROPOSAL, NSTAGES };
    std::vector<std::pair<int, int>> marks;   /* (stage, event index) */
    int next = 0;
};

pt_status mark(pt_table *t, LookupProfile *prof, int stage, cudaStream_t st) {
    if (!prof) return PT_OK;
    if (prof->next >= (int) t->events.size()) {
        cudaEvent_t e;
        PT_CUDA(cudaEventCreate(&e));
        t->events.push_back(e);
    }
    PT_CUDA(cudaEventRecord(t->events[prof->next], st));
    prof->marks.push_back({stage, prof->next});
    prof->next++;
    return PT_OK;
}

/* Proposals handed in by the caller instead of the network's (pt_table_lookup_proposed_profile). */
struct ExtProposals {
    const int *cand;          /* P x PT_PROP_TOPK table entries, -1 = none */
    const float *conf;        /* P confidences */
    float threshold;
    int kcoh_confident;
};

/* The device part of a lookup: a_rgb (device, h x w x 3) -> d_ann (device doubles).  With prof,
   an event is recorded after every stage and SSD work is counted. */
pt_status lookup_device(pt_table *t, const float *a_rgb, int h, int w, double *d_ann, cudaStream_t st,
                        LookupProfile *prof = nullptr, pt_proposal *net = nullptr, const double *d_prev = nullptr,
                        const float *d_sv = nullptr, const ExtProposals *ext = nullptr) {
    const bool learned = net || ext;
    const pt_params &p = t->p;
    long long P = (long long) (h - 7) * (w - 7);
    if (P >= (1ll << 31)) return pt_fail(PT_BAD_ARG, "query image too large");
    int n = (int) P;
    PT_TRY(ensure_query_buffers(t, h, w));
    unsigned long long *ctr = prof ? t->q_counters.p : nullptr;
    if (ctr) PT_CUDA(cudaMemsetAsync(ctr, 0, sizeof(unsigned long long) * 6, st));
    PT_TRY(mark(t, prof, -1, st));
    if (t->desc_mode) {
        if (learned) return pt_fail(PT_UNSUPPORTED, "learned proposals in descriptor mode");
        int ih, iw;
        size_t nin;
        query_input_dims(t, h, w, ih, iw, nin);
        PT_TRY(pt_launch_descriptor_input(a_rgb, ih, iw, t->nd, t->in_padded, t->q_desc.p, t->ds, st));
    } else if (t->pca) {
        PT_TRY(pt_launch_pca(a_rgb, h, w, pt_color_mode(p), t->q_rgba.p, t->pca_mean.p, t->pca_basis.p, t->nd,
                             t->q_desc.p, t->ds, st));
    } else if (learned || !t->subs.empty()) {
        PT_TRY(pt_launch_descriptor(p.ndims, p.nchroma, a_rgb, h, w, pt_color_mode(p), t->q_rgba.p, t->q_desc.p,
                                    t->ds, st));
    }
    /* The plain single-table query needs its descriptors only for the table step: one fused pass. */
    const bool fused = !t->desc_mode && !t->pca && !learned && t->subs.empty();
    if (fused)
        PT_TRY(pt_launch_descriptor_cells(p.ndims, p.nchroma, a_rgb, h, w, pt_color_mode(p), t->q_rgba.p, t->bins,
                                          t->to_bin.p, t->table.p, t->q_tcand.p, 0, (h - 7 + 7) / 8, st));
    PT_TRY(mark(t, prof, LookupProfile::DESC, st));
    if (!fused)
        PT_TRY(pt_launch_table_candidates(t->bins, t->q_desc.p, t->ds, P, t->to_bin.p, t->table.p, t->q_tcand.p, st));
    if (!t->subs.empty()) {
        PT_CUDA(t->q_tcand_more.reserve((size_t) P * t->subs.size()));
        for (size_t i = 0; i < t->subs.size(); i++) {
            const pt_table *u = t->subs[i].get();
            PT_TRY(pt_launch_table_candidates(u->bins, t->q_desc.p, t->ds, P, u->to_bin.p, u->table.p,
                                              t->q_tcand_more.p + i * (size_t) P, st));
        }
    }
    PT_TRY(mark(t, prof, LookupProfile::CELLS, st));
    if (net && !ext) {
        PtTableView v;
        PT_TRY(pt_table_view(t, &v));
        PT_CUDA(t->q_lcand.reserve((size_t) P * PT_PROP_TOPK));
        PT_CUDA(t->q_lconf.reserve(P));
        PT_TRY(pt_launch_prop_infer(v, net, t->q_desc.p, n, t->q_lcand.p, t->q_lconf.p, nullptr, st));
        PT_TRY(mark(t, prof, LookupProfile::PROPOSAL, st));
    }
    QuerySetup qs;
    qs.aw = w; qs.ah = h; qs.bw = t->w; qs.bh = t->h;
    qs.prop_scale = 1.0 / (1 + p.coherence_spatial);
    qs.triangle_factor = p.triangle_factor;
    qs.kcoherence = p.kcoherence;
    qs.kc_try = p.gpu_kc_max;
    qs.kcoherence_step = p.kcoherence_step;
    qs.spatial = p.spatial;
    qs.do_rs = p.do_rs;
    qs.radius = p.query_step + p.prop_dist;
    qs.b1 = t->b_rgba1.p;
    qs.pull_max = p.gpu_pull_max;
    qs.tile = p.gpu_tile;
    qs.allowed = t->allowed.p;
    qs.allowed_index = p.allowed_index;
    qs.stream = st;
    if (t->desc_mode) {
        qs.adesc = t->q_desc.p;
        qs.bdesc = t->b_desc.p;
        qs.ds = t->ds;
        qs.nd = t->nd;
    }
    if (!t->subs.empty()) {
        qs.tcand_more = t->q_tcand_more.p;
        qs.ntcand_more = (int) t->subs.size();
    }
    if (qs.radius > 2) qs.radius = 2;
    const double temporal_scale = 1.0 / (1 + p.coherence_temporal);          /* patchtable.h:3488 */
    if (d_prev) {                             /* no bad previous matches so far (read by the host lookup) */
        PT_CUDA(t->q_tbad.reserve(1));
        PT_CUDA(cudaMemsetAsync(t->q_tbad.p, 0, sizeof(int), st));
    }
    if (p.init_random) {                      /* takes precedence over ann_prev, patchtable.h:3522-3537 */
        PT_TRY(pt_launch_init_random(qs, t->q_rgba.p, t->b_rgba.p, t->q_pos[0].p, t->q_d[0].p, st));
    } else if (d_prev) {
        PT_CUDA(t->q_tpos0.reserve(P));
        PT_CUDA(t->q_td0.reserve(P));
        PT_CUDA(t->q_torig.reserve(P));
        PT_TRY(pt_launch_init_temporal(qs, d_prev, d_sv, p.recalc_dist_temporal, p.sanitize_input, temporal_scale,
                                       t->q_rgba.p, t->b_rgba.p, t->q_pos[0].p, t->q_d[0].p, t->q_torig.p, t->q_tbad.p, st));
        PT_CUDA(cudaMemcpyAsync(t->q_tpos0.p, t->q_pos[0].p, sizeof(int) * n, cudaMemcpyDeviceToDevice, st));
        PT_CUDA(cudaMemcpyAsync(t->q_td0.p, t->q_d[0].p, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
    } else if (learned || pt_default_passes(p) == 0) {
        /* Initial field (patchtable.h:3538-3547): x = b0_ew + 1, dist = DIST_INFINITY. */
        PT_TRY(pt_launch_init(n, pt_xy(t->ew + 1, 0), (float) PT_DIST_INF, t->q_pos[0].p, t->q_d[0].p, st));
    }
    /* Otherwise the first pass reads no state arrays: its kernels start from the initial field. */
    const bool fresh = !p.init_random && !d_prev && !learned && pt_default_passes(p) > 0;
    /* the last pull writes the NNF itself unless the temporal output has to restore distances */
    const bool direct_out = p.do_prop && pt_default_passes(p) > 0 && !(d_prev && !p.init_random && p.coherence_temporal != 0.0);
    PT_TRY(mark(t, prof, LookupProfile::INIT, st));
    int passes = pt_default_passes(p);
    int jump = pt_default_jump(p, passes);
    int cur = 0;
    for (int i = 0; i < passes; i++) {
        /* Pass 0 plays the reference's first iteration (table lookup, :3641); k-coherence runs
           on the passes of the sweeps that kcoherence_iter selects.  A pass skips a repeated
           k-coherence search only when the previous pass ran one (and so wrote kc_done). */
        bool do_table = i == 0 && p.do_table_lookup;
        QuerySetup qi = qs;
        qi.pass = i;
        if (!pt_pass_kcoh(p, i, passes)) qi.kcoherence = 0;
        const int use_done = i > 0 && pt_pass_kcoh(p, i - 1, passes);
        if (learned)
            PT_TRY(pt_launch_choose_learned(qi, t->q_rgba.p, t->b_rgba.p, t->q_pos[cur].p, t->q_d[cur].p, t->q_tcand.p,
                                            t->kcoh.p, do_table, t->q_chpos.p, t->q_chd.p, t->q_kcdone.p, use_done,
                                            i == 0 ? (ext ? ext->cand : t->q_lcand.p) : nullptr,
                                            ext ? ext->conf : t->q_lconf.p, ext ? ext->threshold : pt_prop_threshold(net),
                                            ext ? ext->kcoh_confident : pt_prop_kcoh_confident(net), ctr,
                                            ctr ? ctr + 4 : nullptr, st));
        else
            PT_TRY(pt_launch_choose(qi, n, t->q_rgba.p, t->b_rgba.p, fresh && i == 0 ? nullptr : t->q_pos[cur].p,
                                    fresh && i == 0 ? nullptr : t->q_d[cur].p, t->q_tcand.p, t->kcoh.p, do_table,
                                    t->q_chpos.p, t->q_chd.p, t->q_kcdone.p, use_done, ctr, st));
        PT_TRY(mark(t, prof, LookupProfile::CHOOSE, st));
        if (p.do_prop) {
            QuerySetup qp = qs;
            qp.step = pt_pass_step(i, passes, jump);
            if (i == passes - 1 && direct_out) qp.ann = d_ann;
            PT_TRY(pt_launch_pull(qp, n, t->q_rgba.p, t->b_rgba.p, fresh && i == 0 ? nullptr : t->q_pos[cur].p,
                                  fresh && i == 0 ? nullptr : t->q_d[cur].p, t->q_chpos.p, t->q_chd.p,
                                  t->q_pos[1 - cur].p, t->q_d[1 - cur].p, ctr ? ctr + 2 : nullptr, st));
            PT_TRY(mark(t, prof, LookupProfile::PULL, st));
            cur = 1 - cur;
        } else {
            PT_CUDA(cudaMemcpyAsync(t->q_pos[cur].p, t->q_chpos.p, sizeof(int) * n, cudaMemcpyDeviceToDevice, st));
            PT_CUDA(cudaMemcpyAsync(t->q_d[cur].p, t->q_chd.p, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
        }
    }
    if (d_prev && !p.init_random && p.coherence_temporal != 0.0)
        PT_TRY(pt_launch_output_temporal(n, t->q_pos[cur].p, t->q_d[cur].p, t->q_tpos0.p, t->q_td0.p, t->q_torig.p, d_ann, st));
    else if (!direct_out)
        PT_TRY(pt_launch_output(n, t->q_pos[cur].p, t->q_d[cur].p, d_ann, st));
    PT_TRY(mark(t, prof, LookupProfile::OUTPUT, st));
    return PT_OK;
}

/* The host lookup of a one-pass schedule, pipelined over bands of patch rows.  A band needs only
   its own pixel rows plus 7; its choose also reads the next band's RGBA rows (written by that
   band's descriptor launch) and its pull the next band's choices.  Four streams carry the phases:
   upload of band b -> descriptor and table entries of band b (one fused pass) -> choose of band
   b-1 -> pull of band b-2 -> download of band b-2, each waiting on the events its inputs come
   from; choose and pull start from the initial field without reading state arrays.  Consecutive
   bands' kernels overlap (filling each other's last waves) and the copies overlap the kernels.
   Concurrent kernels always touch disjoint rows (bands are at least 32 rows; a pull reads at most
   16 rows beyond its band).  Every kernel computes exactly what the whole-image launch computes
   for its rows, so the result is identical.  The download carries the packed field (int32
   position, float32 distance: 8 bytes per patch instead of the float64 record's 24) into pinned
   staging; once a band has arrived, the host threads widen it into the caller's float64 buffer
   while later bands are still computed and copied.  The launches are enqueued directly: replaying
   the same sequence as a recorded CUDA graph measured slower (1.45 against 1.29 ms at 1080p).
   Device-resident lookups keep the whole-image launches: the same bands on three streams without
   copies measured 1.10 against 0.98 ms. */
int band_rows(const pt_table *t, int h, int w) {
    const pt_params &p = t->p;
    const int eh = h - 7, ew = w - 7;
    int B = 0;
    if (p.gpu_bands <= 0) {
        /* Default: the band's choose launch fills whole waves.  A choose CTA of tw patches is
           resident about 10 * 64 / tw times per SM, so one wave covers sms * 640 / (tw * segments)
           patch rows; B is the largest multiple of 8 rows within k waves, for the smallest k giving at
           least 32 rows and at most 24 bands (measured e2e: 720p 9 bands 0.71 ms, 1080p 20 bands
           of 56 rows = 0.95 wave 1.35 ms against 1.41 at 16 bands of 1.22 waves, 1440p 17 bands).
           Fewer than 8 bands would lose the overlap: then about 16 bands. */
        static int sms = 0;
        if (!sms) {
            int dev = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (sms < 1) sms = 148;
        }
        const int tw = (p.gpu_tile == 64 || p.gpu_tile == 128 || p.gpu_tile == 256) ? p.gpu_tile : 32;
        const double rows_wave = (double) sms * (10 * 64 / tw) / ((ew + tw - 1) / tw);
        for (int k = 1; k <= 64; k++) {
            B = (int) (k * rows_wave / 8) * 8;
            if (B >= 32 && (eh + B - 1) / B <= 24) break;
        }
        if (B < 32 || (eh + B - 1) / B < 8 || (eh + B - 1) / B > 24) B = 0;
    }
    if (B == 0) {
        const int want = p.gpu_bands > 0 ? p.gpu_bands : 16;
        B = ((eh + want - 1) / want + 7) / 8 * 8;       /* about `want` bands, each a multiple of 8 rows */
        if (B < 32) B = 32;
    }
    return B;
}

/* Enqueues the band pipeline on the table's streams, starting after the work queued on t->st and
   joining every stream back into t->st at the end.  ev_d[b] marks band b's download. */
/* A band pipeline's host image (uploaded band by band into the table's buffer) and its output:
   the packed field downloaded for host widening (widen) or the float64 records downloaded to
   ann_out. */
struct BandIO {
    const float *a = nullptr;
    double *ann_out = nullptr;
    bool widen = false;
    cudaStream_t origin = nullptr;    /* the pipeline starts after and joins into this stream */
    std::atomic<int> *recorded = nullptr;   /* bands whose download event this call has recorded */
    float *stage = nullptr;           /* page-locked copy of a pageable query image, or NULL */
};

/* Row boundaries of the bands: B rows each (a multiple of 8: the descriptor pass works on 8-row
   tiles), the last band ending at eh.  Shortening the last two bands to B/2 and B/4, so that less
   work lands after the last upload, measured no faster (1.23-1.38 against 1.16-1.33 ms at 1080p). */
std::vector<int> band_edges(int eh, int B) {
    std::vector<int> e{0};
    while (e.back() < eh) e.push_back(std::min(eh, e.back() + B));
    return e;
}

pt_status enqueue_bands(pt_table *t, const BandIO &io, int h, int w, const std::vector<int> &edge, int nb) {
    const pt_params &p = t->p;
    const int eh = h - 7, ew = w - 7;
    const long long P = (long long) eh * ew;
    const float *a = io.a;
    double *ann_out = io.ann_out;
    const bool widen = io.widen;
    const float *rgb = t->q_rgb.p;
    cudaEvent_t *ev_in = t->band_ev.data(), *ev_a = ev_in + nb, *ev_b = ev_a + nb, *ev_c = ev_b + nb, *ev_d = ev_c + nb;
    cudaEvent_t ev_start = t->band_ev[5 * nb], *ev_join = &t->band_ev[5 * nb + 1];
    cudaStream_t sa = t->st, sb = t->st_choose, sc = t->st_pull;
    PT_CUDA(cudaEventRecord(ev_start, io.origin));
    for (cudaStream_t s2 : {sa, t->st_in, sb, sc, t->st_out})
        if (s2 != io.origin) PT_CUDA(cudaStreamWaitEvent(s2, ev_start, 0));
    QuerySetup qs;
    qs.aw = w; qs.ah = h; qs.bw = t->w; qs.bh = t->h;
    qs.prop_scale = 1.0 / (1 + p.coherence_spatial);
    qs.triangle_factor = p.triangle_factor;
    qs.kcoherence = pt_pass_kcoh(p, 0, 1) ? p.kcoherence : 0;
    qs.kc_try = p.gpu_kc_max;
    qs.kcoherence_step = p.kcoherence_step;
    qs.spatial = p.spatial;
    qs.do_rs = p.do_rs;
    qs.radius = std::min(2, p.query_step + p.prop_dist);
    qs.b1 = t->b_rgba1.p;
    qs.pull_max = p.gpu_pull_max;
    qs.tile = p.gpu_tile;
    qs.allowed = t->allowed.p;
    qs.allowed_index = p.allowed_index;
    QuerySetup qp = qs;
    qp.step = pt_pass_step(0, 1, pt_default_jump(p, 1));
    /* Every band's upload is enqueued first, so the image streams in without gaps and each band's
       kernels start as soon as its rows have arrived. */
    for (int b = 0; b < nb; b++) {
        const int r0 = edge[b], r1 = edge[b + 1];
        const int p0 = b == 0 ? 0 : r0 + 7, p1 = b == nb - 1 ? h : r1 + 7;
        const size_t px0 = (size_t) p0 * w * 3, npx = (size_t) (p1 - p0) * w * 3;
        const float *src = a + px0;
        if (io.stage) {
            /* a pageable image: host threads copy the band into page-locked memory, and its upload
               runs while the next band is copied */
            pt_host_copy(io.stage + px0, a + px0, npx);
            src = io.stage + px0;
        }
        PT_CUDA(cudaMemcpyAsync(t->q_rgb.p + px0, src, sizeof(float) * npx, cudaMemcpyHostToDevice, t->st_in));
        PT_CUDA(cudaEventRecord(ev_in[b], t->st_in));
    }
    for (int b = 0; b <= nb + 1; b++) {
        if (b < nb) {
            const int r0 = edge[b], r1 = edge[b + 1];
            PT_CUDA(cudaStreamWaitEvent(sa, ev_in[b], 0));
            PT_TRY(pt_launch_descriptor_cells(p.ndims, p.nchroma, rgb, h, w, pt_color_mode(p), t->q_rgba.p,
                                              t->bins, t->to_bin.p, t->table.p, t->q_tcand.p, r0 / 8, (r1 - r0 + 7) / 8, sa));
            PT_CUDA(cudaEventRecord(ev_a[b], sa));
        }
        if (b >= 1 && b - 1 < nb) {
            const int r0 = edge[b - 1], r1 = edge[b];
            PT_CUDA(cudaStreamWaitEvent(sb, ev_a[b < nb ? b : nb - 1], 0));
            QuerySetup qc = qs;
            qc.row0 = r0;
            qc.rows = r1 - r0;
            qc.stream = sb;
            PT_TRY(pt_launch_choose(qc, (int) P, t->q_rgba.p, t->b_rgba.p, nullptr, nullptr, t->q_tcand.p, t->kcoh.p,
                                    p.do_table_lookup, t->q_chpos.p, t->q_chd.p, t->q_kcdone.p, 0, nullptr, sb));
            PT_CUDA(cudaEventRecord(ev_b[b - 1], sb));
        }
        if (b >= 2) {
            const int r0 = edge[b - 2], r1 = edge[b - 1];
            PT_CUDA(cudaStreamWaitEvent(sc, ev_b[b - 1 < nb ? b - 1 : nb - 1], 0));
            QuerySetup qb = qp;
            qb.row0 = r0;
            qb.rows = r1 - r0;
            qb.stream = sc;
            /* the pull writes the band's final field: packed position and float distance, or
               (without host widening) the float64 records */
            if (!widen) qb.ann = t->q_ann.p;
            PT_TRY(pt_launch_pull(qb, (int) P, t->q_rgba.p, t->b_rgba.p, nullptr, nullptr, t->q_chpos.p, t->q_chd.p,
                                  t->q_pos[1].p, t->q_d[1].p, nullptr, sc));
            const size_t o = (size_t) r0 * ew;
            const size_t n = (size_t) (r1 - r0) * ew;
            PT_CUDA(cudaEventRecord(ev_c[b - 2], sc));
            PT_CUDA(cudaStreamWaitEvent(t->st_out, ev_c[b - 2], 0));
            if (widen) {
                PT_CUDA(cudaMemcpyAsync(t->h_pos.p + o, t->q_pos[1].p + o, sizeof(int) * n, cudaMemcpyDeviceToHost, t->st_out));
                PT_CUDA(cudaMemcpyAsync(t->h_d.p + o, t->q_d[1].p + o, sizeof(float) * n, cudaMemcpyDeviceToHost, t->st_out));
            } else {
                PT_CUDA(cudaMemcpyAsync(ann_out + 3 * o, t->q_ann.p + 3 * o, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost,
                                        t->st_out));
            }
            PT_CUDA(cudaEventRecord(ev_d[b - 2], t->st_out));
            if (io.recorded) io.recorded->store(b - 1, std::memory_order_release);
        }
    }
    int k = 0;
    for (cudaStream_t s2 : {sa, t->st_in, sb, sc, t->st_out}) {
        if (s2 == io.origin) continue;
        PT_CUDA(cudaEventRecord(ev_join[k], s2));
        PT_CUDA(cudaStreamWaitEvent(io.origin, ev_join[k], 0));
        k++;
    }
    return PT_OK;
}

/* Lookups that run as a band pipeline: the plain single-table query of one pass with
   propagation, from the default field, on images of at least 64 patch rows. */
bool banded_schedule(const pt_table *t, int h) {
    /* a band's pull reads the choices of rows up to step * radius below it, which must lie in the
       next band (every band but the last has at least 8 rows) */
    const int reach = pt_pass_step(0, 1, pt_default_jump(t->p, 1)) * std::min(2, t->p.query_step + t->p.prop_dist);
    return !t->desc_mode && !t->pca && t->subs.empty() && !t->p.init_random && pt_default_passes(t->p) == 1 &&
           t->p.do_prop && h - 7 >= 64 && reach <= 8;
}

pt_status lookup_banded(pt_table *t, const float *a, int h, int w, double *ann_out) {
    const int eh = h - 7, ew = w - 7;
    const long long P = (long long) eh * ew;
    PT_TRY(ensure_query_buffers(t, h, w));
    for (cudaStream_t *sp : {&t->st_in, &t->st_out, &t->st_choose, &t->st_pull})
        if (!*sp) PT_CUDA(cudaStreamCreateWithFlags(sp, cudaStreamNonBlocking));
    const std::vector<int> edge = band_edges(eh, band_rows(t, h, w));
    const int nb = (int) edge.size() - 1;
    while ((int) t->band_ev.size() < 5 * nb + 6) {
        cudaEvent_t e;
        PT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        t->band_ev.push_back(e);
    }
    const bool widen = pt_host_widen();
    if (widen) {
        PT_CUDA(t->h_pos.reserve(P));
        PT_CUDA(t->h_d.reserve(P));
    } else {
        PT_CUDA(t->q_ann.reserve((size_t) P * 3));
    }
    BandIO io;
    io.a = a;
    io.ann_out = ann_out;
    if (!host_pinned(a)) {
        PT_CUDA(t->h_in.reserve((size_t) h * w * 3));
        io.stage = t->h_in.p;
    }
    io.widen = widen;
    io.origin = t->st;
    /* Each band is widened as soon as it has arrived, by a second host thread (with the widening
       pool), while this thread is still enqueueing the later bands: enqueueing a band takes about
       as long as the GPU takes to run it, so widening only after the last enqueue would leave the
       first bands' records waiting. */
    std::atomic<int> recorded(0);
    std::atomic<bool> stop(false);
    cudaError_t widen_err = cudaSuccess;
    cudaEvent_t *ev_d = t->band_ev.data() + 4 * nb;
    std::thread widener;
    if (widen) {
        io.recorded = &recorded;
        widener = std::thread([&] {
            for (int b = 0; b < nb; b++) {
                while (recorded.load(std::memory_order_acquire) <= b) {
                    if (stop.load(std::memory_order_acquire)) return;
                    std::this_thread::yield();
                }
                const cudaError_t e = cudaEventSynchronize(ev_d[b]);
                if (e != cudaSuccess) { widen_err = e; return; }
                const int r0 = edge[b], r1 = edge[b + 1];
                const size_t o = (size_t) r0 * ew;
                pt_expand_nnf(t->h_pos.p + o, t->h_d.p + o, (long long) (r1 - r0) * ew, ann_out + 3 * o);
            }
        });
    }
    const pt_status est = enqueue_bands(t, io, h, w, edge, nb);
    if (est != PT_OK) stop.store(true, std::memory_order_release);
    if (widener.joinable()) widener.join();
    if (est != PT_OK) {
        for (cudaStream_t s2 : {t->st, t->st_in, t->st_choose, t->st_pull, t->st_out})
            cudaStreamSynchronize(s2);       /* nothing of this call stays in flight */
        return est;
    }
    t->last_h2d = (long long) sizeof(float) * h * w * 3;
    t->last_d2h = (long long) (widen ? sizeof(int) + sizeof(float) : 3 * sizeof(double)) * P;
    if (widen_err != cudaSuccess) return pt_fail(PT_CUDA_ERR, "band download: %s", cudaGetErrorString(widen_err));
    PT_CUDA(cudaStreamSynchronize(t->st));
    return PT_OK;
}

/* lookup_device with stage events; stage_ms[nst] receives summed stage times, counters[nctr] the
   SSD work counters. */
pt_status profile_impl(pt_table *t, pt_proposal *net, const float *d_a, int ih, int iw, double *d_ann, cudaStream_t st,
                       double *stage_ms, int nst, uint64_t *counters, int nctr, const ExtProposals *ext = nullptr) {
    if (!t || !d_a || !d_ann) return pt_fail(PT_BAD_ARG, "null argument");
    int h, w;
    PT_TRY(query_dims(t, ih, iw, h, w));
    LookupProfile prof;
    PT_TRY(lookup_device(t, d_a, h, w, d_ann, st, &prof, net, nullptr, nullptr, ext));
    PT_CUDA(cudaStreamSynchronize(st));
    if (net) PT_TRY(pt_prop_check_error(net, st));
    double ms_all[LookupProfile::NSTAGES] = {0};
    for (size_t k = 1; k < prof.marks.size(); k++) {
        float ms = 0;
        PT_CUDA(cudaEventElapsedTime(&ms, t->events[prof.marks[k - 1].second], t->events[prof.marks[k].second]));
        ms_all[prof.marks[k].first] += ms;
    }
    if (stage_ms) for (int i = 0; i < nst; i++) stage_ms[i] = ms_all[i];
    if (counters) {
        unsigned long long c[6];
        PT_CUDA(cudaMemcpy(c, t->q_counters.p, sizeof(c), cudaMemcpyDeviceToHost));
        for (int i = 0; i < nctr; i++) counters[i] = c[i];
    }
    return PT_OK;
}

}  // namespace

namespace {

/* ---- table files in the reference's format ----
   PatchTableFixedN::save / load (patchtable.h:1574-1593) over the serialisation primitives of
   patchtable.cpp:499-573: a string is its int32 length and its bytes, a vector its int32 length
   and its elements, an Array its sizes (a vector<int>) and its elements, all little-endian.  A
   file holds "PatchTable", the table (sizes = nslices), b0 (h, w, 3), wh0 (h+7, w+7, ndims),
   nslices, the partition ("PatchPartition", count, then per dimension "PatchPartition1D", to_bin,
   centers, lsizes, rsizes, min_val, max_val, range, nslices, "EndPatchPartition1D"),
   "EndPatchPartition" and "EndPatchTable". */
struct FileOut {
    FILE *f;
    bool ok = true;
    void raw(const void *p, size_t n) { if (ok && n && fwrite(p, 1, n, f) != n) ok = false; }
    void i32(int v) { raw(&v, 4); }
    void f32(float v) { raw(&v, 4); }
    void str(const char *s) { int n = (int) strlen(s); i32(n); raw(s, n); }
    template<class T> void vec(const std::vector<T> &v) { i32((int) v.size()); raw(v.data(), sizeof(T) * v.size()); }
};

struct FileIn {
    FILE *f;
    bool ok = true;
    void raw(void *p, size_t n) { if (ok && n && fread(p, 1, n, f) != n) ok = false; }
    int i32() { int v = 0; raw(&v, 4); return v; }
    float f32() { float v = 0; raw(&v, 4); return v; }
    bool id(const char *s) {
        int n = i32();
        if (!ok || n != (int) strlen(s)) { ok = false; return false; }
        std::string got(n, 0);
        raw(&got[0], n);
        ok = ok && got == s;
        return ok;
    }
    /* a vector of at most `cap` elements */
    template<class T> bool vec(std::vector<T> &v, long long cap) {
        int n = i32();
        if (!ok || n < 0 || n > cap) { ok = false; return false; }
        v.resize(n);
        raw(v.data(), sizeof(T) * (size_t) n);
        return ok;
    }
};

pt_status save_impl(const pt_table *t, const char *filename) {
    if (t->desc_mode || t->pca) return pt_fail(PT_UNSUPPORTED, "saving a descriptor mode or PCA table");
    const int h = t->h, w = t->w, nd = t->nd;
    std::vector<int> cells((size_t) t->ncells);
    std::vector<float4> rgba((size_t) h * w);
    std::vector<float> desc((size_t) t->eh * t->ew * t->ds);
    PT_CUDA(cudaMemcpyAsync(cells.data(), t->table.p, sizeof(int) * cells.size(), cudaMemcpyDeviceToHost, t->st));
    PT_CUDA(cudaMemcpyAsync(rgba.data(), t->b_rgba.p, sizeof(float4) * rgba.size(), cudaMemcpyDeviceToHost, t->st));
    PT_CUDA(cudaMemcpyAsync(desc.data(), t->b_desc.p, sizeof(float) * desc.size(), cudaMemcpyDeviceToHost, t->st));
    PT_CUDA(cudaStreamSynchronize(t->st));
    std::vector<float> b0((size_t) h * w * 3);
    for (size_t i = 0; i < rgba.size(); i++) { b0[3 * i] = rgba[i].x; b0[3 * i + 1] = rgba[i].y; b0[3 * i + 2] = rgba[i].z; }
    /* wh0 holds the descriptor of the patch with top-left (x, y) at (y + 7, x + 7); the partial
       windows of the reference's "full" padding are not kept by this library and are written as 0 */
    std::vector<float> wh0((size_t) (h + 7) * (w + 7) * nd, 0.f);
    for (int y = 0; y < t->eh; y++)
        for (int x = 0; x < t->ew; x++)
            for (int d = 0; d < nd; d++)
                wh0[((size_t) (y + 7) * (w + 7) + (x + 7)) * nd + d] = desc[((size_t) y * t->ew + x) * t->ds + d];
    FILE *f = fopen(filename, "wb");
    if (!f) return pt_fail(PT_IO, "cannot open %s for writing", filename);
    FileOut o{f};
    o.str("PatchTable");
    o.vec(t->nslices);
    o.raw(cells.data(), sizeof(int) * cells.size());
    o.vec(std::vector<int>{h, w, 3});
    o.raw(b0.data(), sizeof(float) * b0.size());
    o.vec(std::vector<int>{h + 7, w + 7, nd});
    o.raw(wh0.data(), sizeof(float) * wh0.size());
    o.vec(t->nslices);
    o.str("PatchPartition");
    o.i32(t->G);
    for (int d = 0; d < t->G; d++) {
        const PtPartition &P = t->part[d];
        o.str("PatchPartition1D");
        o.vec(P.to_bin);
        o.vec(P.centers);
        o.vec(P.lsizes);
        o.vec(P.rsizes);
        o.f32(P.min_val);
        o.f32(P.max_val);
        o.f32(P.range);
        o.i32(P.nslices);
        o.str("EndPatchPartition1D");
    }
    o.str("EndPatchPartition");
    o.str("EndPatchTable");
    const bool ok = o.ok;
    if (fclose(f) != 0 || !ok) return pt_fail(PT_IO, "writing %s failed", filename);
    return PT_OK;
}

pt_status load_impl(const pt_params *pin, const char *filename, pt_table **out) {
    *out = nullptr;
    if (pin->is_descriptor || pin->dim_algo != 0) return pt_fail(PT_UNSUPPORTED, "loading a descriptor mode or PCA table");
    FILE *f = fopen(filename, "rb");
    if (!f) return pt_fail(PT_IO, "cannot open %s", filename);
    struct Closer { FILE *f; ~Closer() { fclose(f); } } closer{f};
    FileIn in{f};
    std::vector<int> tsizes, bsizes, wsizes, nslices;
    std::vector<int> cells;
    if (!in.id("PatchTable") || !in.vec(tsizes, PT_DESC_MAX)) return pt_fail(PT_IO, "%s: not a PatchTable file", filename);
    long long ncells = 1;
    for (int v : tsizes) {
        if (v < 1) return pt_fail(PT_IO, "%s: bad table size", filename);
        ncells *= v;
        if (ncells >= (1ll << 31)) return pt_fail(PT_IO, "%s: table exceeds 2^31 cells", filename);
    }
    cells.resize((size_t) ncells);
    in.raw(cells.data(), sizeof(int) * cells.size());
    if (!in.vec(bsizes, 3) || bsizes.size() != 3 || bsizes[2] != 3) return pt_fail(PT_IO, "%s: bad b0 array", filename);
    const int h = bsizes[0], w = bsizes[1];
    PT_TRY(check_params(pin, h, w));
    std::vector<float> b0((size_t) h * w * 3);
    in.raw(b0.data(), sizeof(float) * b0.size());
    if (!in.vec(wsizes, 3) || wsizes.size() != 3 || wsizes[0] != h + 7 || wsizes[1] != w + 7)
        return pt_fail(PT_IO, "%s: bad wh0 array", filename);
    const int nd = wsizes[2];
    if (nd != pin->ndims) return pt_fail(PT_BAD_ARG, "%s holds %d descriptor dimensions; the parameters ask for %d", filename, nd, pin->ndims);
    std::vector<float> wh0((size_t) (h + 7) * (w + 7) * nd);
    in.raw(wh0.data(), sizeof(float) * wh0.size());
    if (!in.vec(nslices, PT_DESC_MAX) || nslices != tsizes) return pt_fail(PT_IO, "%s: nslices do not match the table", filename);
    const int G = (int) nslices.size();
    if (G < 1 || G > nd) return pt_fail(PT_IO, "%s: %d grid dimensions for %d descriptor dimensions", filename, G, nd);
    if (!in.id("PatchPartition") || in.i32() != G) return pt_fail(PT_IO, "%s: bad partition", filename);
    std::unique_ptr<pt_table> t(new pt_table());
    t->part.assign(G, PtPartition());
    for (int d = 0; d < G; d++) {
        PtPartition &P = t->part[d];
        if (!in.id("PatchPartition1D") || !in.vec(P.to_bin, PT_NMAP) || (int) P.to_bin.size() != PT_NMAP ||
            !in.vec(P.centers, nslices[d]) || !in.vec(P.lsizes, nslices[d]) || !in.vec(P.rsizes, nslices[d]))
            return pt_fail(PT_IO, "%s: bad partition of dimension %d", filename, d);
        P.min_val = in.f32();
        P.max_val = in.f32();
        P.range = in.f32();
        P.nslices = in.i32();
        if (!in.id("EndPatchPartition1D") || P.nslices != nslices[d] || (int) P.centers.size() != nslices[d] ||
            (int) P.lsizes.size() != nslices[d] || (int) P.rsizes.size() != nslices[d])
            return pt_fail(PT_IO, "%s: bad partition of dimension %d", filename, d);
        for (int v : P.to_bin)
            if (v < 0 || v >= nslices[d]) return pt_fail(PT_IO, "%s: to_bin entry out of range", filename);
    }
    if (!in.id("EndPatchPartition") || !in.id("EndPatchTable")) return pt_fail(PT_IO, "%s: truncated file", filename);
    for (int v : cells)
        if (pt_x(v) < 7 || pt_y(v) < 7 || pt_x(v) >= w || pt_y(v) >= h)
            return pt_fail(PT_IO, "%s: table entry outside the image", filename);

    t->p = *pin;
    pt_params &p = t->p;
    p.grid_ndims = G;
    t->h = h; t->w = w; t->eh = h - 7; t->ew = w - 7;
    t->nd = nd; t->G = G;
    t->ds = nd <= 8 ? 8 : 16;
    PT_TRY(pt_descriptor_check(p.ndims, p.nchroma));
    PT_CUDA(cudaStreamCreateWithFlags(&t->st, cudaStreamNonBlocking));
    t->own_stream = true;
    const long long P = (long long) t->eh * t->ew;
    {
        DevBuf<float> rgb;
        PT_CUDA(rgb.reserve(b0.size()));
        PT_CUDA(cudaMemcpyAsync(rgb.p, b0.data(), sizeof(float) * b0.size(), cudaMemcpyHostToDevice, t->st));
        PT_CUDA(t->b_rgba.reserve((size_t) h * w));
        PT_TRY(pt_launch_descriptor(p.ndims, p.nchroma, rgb.p, h, w, pt_color_mode(p), t->b_rgba.p, nullptr, t->ds, t->st));
        std::vector<float> packed((size_t) P * t->ds, 0.0f);
        for (int y = 0; y < t->eh; y++)
            for (int x = 0; x < t->ew; x++)
                for (int d = 0; d < nd; d++)
                    packed[((size_t) y * t->ew + x) * t->ds + d] = wh0[((size_t) (y + 7) * (w + 7) + (x + 7)) * nd + d];
        PT_CUDA(t->b_desc.reserve(packed.size()));
        PT_CUDA(cudaMemcpyAsync(t->b_desc.p, packed.data(), sizeof(float) * packed.size(), cudaMemcpyHostToDevice, t->st));
        const size_t npx = (size_t) h * w;
        PT_CUDA(t->b_rgba1.reserve(npx));
        PT_CUDA(cudaMemsetAsync(t->b_rgba1.p, 0, sizeof(float4) * npx, t->st));
        PT_CUDA(cudaMemcpyAsync(t->b_rgba1.p, t->b_rgba.p + 1, sizeof(float4) * (npx - 1), cudaMemcpyDeviceToDevice, t->st));
        PT_CUDA(cudaStreamSynchronize(t->st));
    }
    /* the file has no k-coherence set (the reference's load leaves it empty); it is rebuilt from
       the stored descriptors */
    if (p.kcoherence > 0) PT_TRY(build_kcoherence(t.get(), std::vector<int>()));
    t->nslices = nslices;
    t->stride.assign(G, 1);
    t->ncells = 1;
    for (int d = G - 1; d >= 0; d--) { t->stride[d] = t->ncells; t->ncells *= nslices[d]; }
    t->min_val.resize(G); t->max_val.resize(G); t->range.resize(G);
    for (int d = 0; d < G; d++) {
        t->min_val[d] = t->part[d].min_val;
        t->max_val[d] = t->part[d].max_val;
        t->range[d] = t->part[d].range;
    }
    PT_TRY(upload_partition(t.get(), t->st));
    PT_CUDA(t->table.reserve(t->ncells));
    PT_CUDA(cudaMemcpyAsync(t->table.p, cells.data(), sizeof(int) * cells.size(), cudaMemcpyHostToDevice, t->st));
    PT_CUDA(cudaStreamSynchronize(t->st));
    t->add_count = 0;
    t->dt_levels = 0;
    *out = t.release();
    return PT_OK;
}

}  // namespace

extern "C" {

/* The further tables of ntables > 1 (patchtable.h:3359-3371): each is a full table of b at
   limit int(limit / table_ratio^i), without k-coherence, built after the first (and after its
   save, which each further table then repeats with the same file name, as in the reference).
   A caller-supplied descriptor of b (wh0) serves them too: it is the descriptor they would
   compute from b. */
pt_status build_subtables(pt_table *t, const float *b, int h, int w, int channels, const int32_t *allowed,
                          const float *wh0) {
    for (int i = 1; i < t->p.ntables; i++) {
        pt_params pc = t->p;
        pc.limit = (double) (int) (pc.limit * (1.0 / pow(pc.table_ratio, i)));
        pc.kcoherence = 0;
        pc.ntables = 1;
        pt_table *u = nullptr;
        if (wh0) PT_TRY(create_impl(&pc, b, h, w, channels, wh0, allowed, &u));
        else PT_TRY(pt_table_create(&pc, b, h, w, channels, allowed, &u));
        t->subs.emplace_back(u);
    }
    return PT_OK;
}

pt_status pt_table_create(const pt_params *p, const float *b, int h, int w, int channels, const int32_t *allowed,
                          pt_table **out) {
    if (p && p->load_filename[0]) return load_impl(p, p->load_filename, out);      /* patchtable.h:2591-2594 */
    PT_TRY(create_impl(p, b, h, w, channels, nullptr, allowed, out));
    if (p->save_filename[0]) {                                                   /* patchtable.h:3326-3328 */
        pt_status s = save_impl(*out, p->save_filename);
        if (s != PT_OK) { pt_table_free(*out); *out = nullptr; return s; }
    }
    pt_status s = build_subtables(*out, b, h, w, channels, allowed, nullptr);
    if (s != PT_OK) { pt_table_free(*out); *out = nullptr; }
    return s;
}

pt_status pt_table_create_with_descriptor(const pt_params *p, const float *b, int h, int w, const float *wh0,
                                          const int32_t *allowed, pt_table **out) {
    if (!wh0) return pt_fail(PT_BAD_ARG, "null descriptor");
    PT_TRY(create_impl(p, b, h, w, 3, wh0, allowed, out));
    pt_status s = build_subtables(*out, b, h, w, 3, allowed, wh0);
    if (s != PT_OK) { pt_table_free(*out); *out = nullptr; }
    return s;
}

pt_status pt_table_subtable(pt_table *t, int i, pt_table **out) {
    if (!t || !out) return pt_fail(PT_BAD_ARG, "null argument");
    if (i < 0 || i >= (int) t->subs.size()) return pt_fail(PT_BAD_ARG, "table %d of %d further tables", i, (int) t->subs.size());
    *out = t->subs[i].get();
    return PT_OK;
}

void pt_table_free(pt_table *t) { delete t; }

pt_status pt_table_lookup(pt_table *t, const float *a, int ih, int iw, double *ann_out, const double *ann_prev,
                          const float *coh_sv, double *seconds) {
    double T0 = now_s();
    if (!t || !a || !ann_out) return pt_fail(PT_BAD_ARG, "null argument");
    int h, w;
    PT_TRY(query_dims(t, ih, iw, h, w));
    if (coh_sv && !ann_prev) return pt_fail(PT_BAD_ARG, "coherence_temporal_sv without ann_prev");
    long long P = (long long) (h - 7) * (w - 7);
    const size_t in_floats = (size_t) ih * iw * (t->desc_mode ? t->nd : 3);
    if (ann_prev) {
        PT_TRY(ensure_query_buffers(t, h, w));
        PT_CUDA(t->q_ann.reserve((size_t) P * 3));
        PT_CUDA(t->q_prev.reserve((size_t) P * 3));
        PT_CUDA(cudaMemcpyAsync(t->q_prev.p, ann_prev, sizeof(double) * (size_t) P * 3, cudaMemcpyHostToDevice, t->st));
        if (coh_sv) {
            PT_CUDA(t->q_sv.reserve(P));
            PT_CUDA(cudaMemcpyAsync(t->q_sv.p, coh_sv, sizeof(float) * P, cudaMemcpyHostToDevice, t->st));
        }
        PT_CUDA(cudaMemcpyAsync(t->q_rgb.p, a, sizeof(float) * in_floats, cudaMemcpyHostToDevice, t->st));
        PT_TRY(lookup_device(t, t->q_rgb.p, h, w, t->q_ann.p, t->st, nullptr, nullptr, t->q_prev.p,
                             coh_sv ? t->q_sv.p : nullptr));
        PT_CUDA(cudaMemcpyAsync(ann_out, t->q_ann.p, sizeof(double) * (size_t) P * 3, cudaMemcpyDeviceToHost, t->st));
        t->last_h2d = (long long) (sizeof(double) * 3 * P + sizeof(float) * in_floats + (coh_sv ? sizeof(float) * P : 0));
        t->last_d2h = (long long) sizeof(double) * 3 * P;
        int bad = 0;
        PT_CUDA(cudaMemcpyAsync(&bad, t->q_tbad.p, sizeof(int), cudaMemcpyDeviceToHost, t->st));
        PT_CUDA(cudaStreamSynchronize(t->st));
        if (bad) return pt_fail(PT_BAD_ARG, "ann_prev holds matches outside the table image and sanitize_input is 0");
        if (seconds) *seconds = now_s() - T0;
        return PT_OK;
    }
    if (banded_schedule(t, h)) {
        PT_TRY(lookup_banded(t, a, h, w, ann_out));
        if (seconds) *seconds = now_s() - T0;
        return PT_OK;
    }
    PT_TRY(ensure_query_buffers(t, h, w));
    PT_CUDA(t->q_ann.reserve((size_t) P * 3));
    /* a pageable image is copied into page-locked memory by the host threads first */
    const float *src = a;
    if (!host_pinned(a)) {
        PT_CUDA(t->h_in.reserve(in_floats));
        pt_host_copy(t->h_in.p, a, in_floats);
        src = t->h_in.p;
    }
    PT_CUDA(cudaMemcpyAsync(t->q_rgb.p, src, sizeof(float) * in_floats, cudaMemcpyHostToDevice, t->st));
    PT_TRY(lookup_device(t, t->q_rgb.p, h, w, t->q_ann.p, t->st));
    t->last_h2d = (long long) (sizeof(float) * in_floats);
    if (pt_host_widen()) {
        /* 8 bytes per patch over PCIe, widened to the float64 records by the host threads */
        PT_CUDA(t->h_pos.reserve(P));
        PT_CUDA(t->h_d.reserve(P));
        PT_TRY(pt_launch_pack_nnf(P, t->q_ann.p, t->q_pos[1].p, t->q_d[1].p, t->st));
        PT_CUDA(cudaMemcpyAsync(t->h_pos.p, t->q_pos[1].p, sizeof(int) * P, cudaMemcpyDeviceToHost, t->st));
        PT_CUDA(cudaMemcpyAsync(t->h_d.p, t->q_d[1].p, sizeof(float) * P, cudaMemcpyDeviceToHost, t->st));
        PT_CUDA(cudaStreamSynchronize(t->st));
        pt_expand_nnf(t->h_pos.p, t->h_d.p, P, ann_out);
        t->last_d2h = (long long) (sizeof(int) + sizeof(float)) * P;
    } else {
        PT_CUDA(cudaMemcpyAsync(ann_out, t->q_ann.p, sizeof(double) * (size_t) P * 3, cudaMemcpyDeviceToHost, t->st));
        PT_CUDA(cudaStreamSynchronize(t->st));
        t->last_d2h = (long long) sizeof(double) * 3 * P;
    }
    if (seconds) *seconds = now_s() - T0;
    return PT_OK;
}

pt_status pt_table_last_transfer(const pt_table *t, int64_t *h2d_bytes, int64_t *d2h_bytes) {
    if (!t || !h2d_bytes || !d2h_bytes) return pt_fail(PT_BAD_ARG, "null argument");
    *h2d_bytes = t->last_h2d;
    *d2h_bytes = t->last_d2h;
    return PT_OK;
}

pt_status pt_table_lookup_device_temporal(pt_table *t, const float *d_a, int ih, int iw, const double *d_ann_prev,
                                         const float *d_coh_sv, double *d_ann, void *stream) {
    if (!t || !d_a || !d_ann || !d_ann_prev) return pt_fail(PT_BAD_ARG, "null argument");
    int h, w;
    PT_TRY(query_dims(t, ih, iw, h, w));
    return lookup_device(t, d_a, h, w, d_ann, (cudaStream_t) stream, nullptr, nullptr, d_ann_prev, d_coh_sv);
}

pt_status pt_table_lookup_device(pt_table *t, const float *d_a, int ih, int iw, double *d_ann, void *stream) {
    if (!t || !d_a || !d_ann) return pt_fail(PT_BAD_ARG, "null argument");
    int h, w;
    PT_TRY(query_dims(t, ih, iw, h, w));
    return lookup_device(t, d_a, h, w, d_ann, (cudaStream_t) stream);
}

/* Diagnostics (no reference counterpart): pt_table_lookup_device with a CUDA event after every
   stage.  stage_ms[6] receives the summed device time of {descriptor, cells, init, choose, pull,
   output}; counters[4] = {choose candidates, choose SSD rows, pull candidates, pull SSD rows}
   (one SSD row = 24 subtractions, multiplications and additions).  Synchronizes the stream. */
pt_status pt_table_lookup_profile(pt_table *t, const float *d_a, int h, int w, double *d_ann, void *stream,
                                  double *stage_ms, uint64_t *counters) {
    return profile_impl(t, nullptr, d_a, h, w, d_ann, (cudaStream_t) stream, stage_ms, LookupProfile::PROPOSAL,
                        counters, 4);
}

pt_status pt_table_lookup_learned_profile(pt_table *t, pt_proposal *net, const float *d_a, int h, int w, double *d_ann,
                                          void *stream, double *stage_ms, uint64_t *counters) {
    if (!net) return pt_fail(PT_BAD_ARG, "null proposal network");
    return profile_impl(t, net, d_a, h, w, d_ann, (cudaStream_t) stream, stage_ms, LookupProfile::NSTAGES, counters, 6);
}

pt_status pt_table_lookup_proposed_profile(pt_table *t, const float *d_a, int h, int w, const int32_t *d_cand,
                                           const float *d_conf, float threshold, int kcoh_confident, double *d_ann,
                                           void *stream, double *stage_ms, uint64_t *counters) {
    if (!d_cand || !d_conf) return pt_fail(PT_BAD_ARG, "null proposals");
    ExtProposals ext{d_cand, d_conf, threshold, kcoh_confident};
    return profile_impl(t, nullptr, d_a, h, w, d_ann, (cudaStream_t) stream, stage_ms, LookupProfile::NSTAGES, counters, 6,
                        &ext);
}

pt_status pt_table_lookup_learned(pt_table *t, pt_proposal *net, const float *a, int h, int w, double *ann_out,
                                  double *seconds) {
    double T0 = now_s();
    if (!t || !net || !a || !ann_out) return pt_fail(PT_BAD_ARG, "null argument");
    if (h < 8 || w < 8) return pt_fail(PT_BAD_ARG, "image %dx%d is smaller than one 8x8 patch", w, h);
    long long P = (long long) (h - 7) * (w - 7);
    PT_TRY(ensure_query_buffers(t, h, w));
    PT_CUDA(t->q_ann.reserve((size_t) P * 3));
    PT_CUDA(cudaMemcpyAsync(t->q_rgb.p, a, sizeof(float) * (size_t) h * w * 3, cudaMemcpyHostToDevice, t->st));
    PT_TRY(lookup_device(t, t->q_rgb.p, h, w, t->q_ann.p, t->st, nullptr, net));
    PT_CUDA(cudaMemcpyAsync(ann_out, t->q_ann.p, sizeof(double) * (size_t) P * 3, cudaMemcpyDeviceToHost, t->st));
    PT_TRY(pt_prop_check_error(net, t->st));
    if (seconds) *seconds = now_s() - T0;
    return PT_OK;
}

pt_status pt_table_lookup_learned_device(pt_table *t, pt_proposal *net, const float *d_a, int h, int w, double *d_ann,
                                         void *stream) {
    if (!t || !net || !d_a || !d_ann) return pt_fail(PT_BAD_ARG, "null argument");
    if (h < 8 || w < 8) return pt_fail(PT_BAD_ARG, "image %dx%d is smaller than one 8x8 patch", w, h);
    return lookup_device(t, d_a, h, w, d_ann, (cudaStream_t) stream, nullptr, net);
}

pt_status pt_table_proposal_samples(pt_table *t, const float *d_a, int h, int w, const double *d_ann, void *X,
                                    uint8_t *labels, void *stream) {
    if (!t || !d_a || !d_ann || !X || !labels) return pt_fail(PT_BAD_ARG, "null argument");
    if (h < 8 || w < 8) return pt_fail(PT_BAD_ARG, "image %dx%d is smaller than one 8x8 patch", w, h);
    cudaStream_t st = (cudaStream_t) stream;
    long long P = (long long) (h - 7) * (w - 7);
    PT_TRY(ensure_query_buffers(t, h, w));
    PtTableView v;
    PT_TRY(pt_table_view(t, &v));
    PT_TRY(pt_prop_check_table(v));
    PT_TRY(pt_launch_descriptor(t->p.ndims, t->p.nchroma, d_a, h, w, pt_color_mode(t->p), nullptr, t->q_desc.p, t->ds,
                                st));
    return pt_launch_prop_samples(v, t->q_desc.p, (int) P, d_ann, X, labels, st);
}

pt_status pt_table_proposal_infer(pt_table *t, pt_proposal *net, const float *d_a, int h, int w, int32_t *cand,
                                  float *conf, float *logits, void *stream) {
    if (!t || !net || !d_a || !cand || !conf) return pt_fail(PT_BAD_ARG, "null argument");
    if (h < 8 || w < 8) return pt_fail(PT_BAD_ARG, "image %dx%d is smaller than one 8x8 patch", w, h);
    cudaStream_t st = (cudaStream_t) stream;
    long long P = (long long) (h - 7) * (w - 7);
    PT_TRY(ensure_query_buffers(t, h, w));
    PtTableView v;
    PT_TRY(pt_table_view(t, &v));
    PT_TRY(pt_launch_descriptor(t->p.ndims, t->p.nchroma, d_a, h, w, pt_color_mode(t->p), nullptr, t->q_desc.p, t->ds,
                                st));
    PT_TRY(pt_launch_prop_infer(v, net, t->q_desc.p, (int) P, cand, conf, logits, st));
    return pt_prop_check_error(net, st);
}


int pt_table_shape(const pt_table *t, int *nslices, int64_t *ncells) {
    if (!t) return -1;
    if (nslices) for (int i = 0; i < PT_MAX_DIMS; i++) nslices[i] = i < t->G ? t->nslices[i] : 0;
    if (ncells) *ncells = t->ncells;
    return t->G;
}

pt_status pt_table_build_profile(const pt_table *t, double *ms, int n) {
    if (!t || !ms || n < 0) return pt_fail(PT_BAD_ARG, "null argument");
    for (int i = 0; i < n; i++) ms[i] = i < PT_BUILD_NSTAGES ? t->build_ms[i] : 0.0;
    return PT_OK;
}

pt_status pt_table_get_cells(const pt_table *t, int32_t *out) {
    if (!t || !out) return pt_fail(PT_BAD_ARG, "null argument");
    PT_CUDA(cudaMemcpyAsync(out, t->table.p, sizeof(int) * (size_t) t->ncells, cudaMemcpyDeviceToHost, t->st));
    PT_CUDA(cudaStreamSynchronize(t->st));
    return PT_OK;
}

pt_status pt_table_get_descriptor(const pt_table *t, float *out) {
    if (!t || !out) return pt_fail(PT_BAD_ARG, "null argument");
    long long P = (long long) t->eh * t->ew;
    std::vector<float> tmp((size_t) P * t->ds);
    PT_CUDA(cudaMemcpyAsync(tmp.data(), t->b_desc.p, sizeof(float) * tmp.size(), cudaMemcpyDeviceToHost, t->st));
    PT_CUDA(cudaStreamSynchronize(t->st));
    for (long long i = 0; i < P; i++)
        for (int d = 0; d < t->nd; d++) out[i * t->nd + d] = tmp[i * t->ds + d];
    return PT_OK;
}

pt_status pt_table_get_partition(const pt_table *t, int dim, float *centers, float *lsizes, float *rsizes,
                                 int32_t *to_bin, float *mmr) {
    if (!t || dim < 0 || dim >= t->G) return pt_fail(PT_BAD_ARG, "bad dimension");
    const PtPartition &P = t->part[dim];
    for (int i = 0; i < P.nslices; i++) {
        if (centers) centers[i] = P.centers[i];
        if (lsizes) lsizes[i] = P.lsizes[i];
        if (rsizes) rsizes[i] = P.rsizes[i];
    }
    if (to_bin) for (int i = 0; i < PT_NMAP; i++) to_bin[i] = P.to_bin[i];
    if (mmr) { mmr[0] = P.min_val; mmr[1] = P.max_val; mmr[2] = P.range; }
    return PT_OK;
}

pt_status pt_table_get_kcoherence(const pt_table *t, int32_t *pos, float *dist) {
    if (!t) return pt_fail(PT_BAD_ARG, "null table");
    if (t->p.kcoherence <= 0) return PT_OK;
    size_t n = (size_t) t->eh * t->ew * t->p.kcoherence;
    std::vector<int2> tmp(n);
    PT_CUDA(cudaMemcpyAsync(tmp.data(), t->kcoh.p, sizeof(int2) * n, cudaMemcpyDeviceToHost, t->st));
    PT_CUDA(cudaStreamSynchronize(t->st));
    for (size_t i = 0; i < n; i++) {
        if (pos) pos[i] = tmp[i].x;
        if (dist) memcpy(&dist[i], &tmp[i].y, sizeof(float));
    }
    return PT_OK;
}

int64_t pt_table_add_count(const pt_table *t) { return t ? t->add_count : -1; }

pt_status pt_table_set_params(pt_table *t, const pt_params *p) {
    if (!t || !p) return pt_fail(PT_BAD_ARG, "null argument");
    pt_params &q = t->p;
    q.prop_iters = p->prop_iters;
    q.query_step = p->query_step;
    q.prop_dist = p->prop_dist;
    q.do_prop = p->do_prop;
    q.do_table_lookup = p->do_table_lookup;
    q.coherence_spatial = p->coherence_spatial;
    q.coherence_temporal = p->coherence_temporal;
    q.recalc_dist_temporal = p->recalc_dist_temporal;
    q.sanitize_input = p->sanitize_input;
    q.triangle_factor = p->triangle_factor;
    q.kcoherence_iter = p->kcoherence_iter;
    q.gpu_prop_passes = p->gpu_prop_passes;
    q.gpu_jump = p->gpu_jump;
    q.gpu_pull_max = p->gpu_pull_max;
    q.gpu_tile = p->gpu_tile;
    q.gpu_bands = p->gpu_bands;
    q.gpu_kc_max = p->gpu_kc_max;
    q.do_rs = p->do_rs;
    q.spatial = p->spatial;
    q.init_random = p->init_random;
    return PT_OK;
}

pt_status pt_descriptor(const pt_params *p, const float *rgb, int h, int w, float *out) {
    PT_TRY(check_params(p, h, w));
    long long P = (long long) (h - 7) * (w - 7);
    int ds = p->ndims <= 8 ? 8 : 16;
    DevBuf<float> d_rgb, d_desc;
    PT_CUDA(d_rgb.reserve((size_t) h * w * 3));
    PT_CUDA(d_desc.reserve((size_t) P * ds));
    PT_CUDA(cudaMemcpy(d_rgb.p, rgb, sizeof(float) * (size_t) h * w * 3, cudaMemcpyHostToDevice));
    PT_TRY(pt_launch_descriptor(p->ndims, p->nchroma, d_rgb.p, h, w, pt_color_mode(*p), nullptr, d_desc.p, ds, 0));
    std::vector<float> tmp((size_t) P * ds);
    PT_CUDA(cudaMemcpy(tmp.data(), d_desc.p, sizeof(float) * tmp.size(), cudaMemcpyDeviceToHost));
    for (long long i = 0; i < P; i++)
        for (int d = 0; d < p->ndims; d++) out[i * p->ndims + d] = tmp[i * ds + d];
    return PT_OK;
}

pt_status pt_table_save(const pt_table *t, const char *filename) {
    if (!t || !filename) return pt_fail(PT_BAD_ARG, "null argument");
    return save_impl(t, filename);
}

pt_status pt_table_load(const pt_params *p, const char *filename, pt_table **out) {
    if (!p || !filename || !out) return pt_fail(PT_BAD_ARG, "null argument");
    return load_impl(p, filename, out);
}

pt_status pt_table_image_shape(const pt_table *t, int *h, int *w) {
    if (!t) return pt_fail(PT_BAD_ARG, "null table");
    if (h) *h = t->h;
    if (w) *w = t->w;
    return PT_OK;
}

int64_t pt_kernel_launch_count(void) { return g_launches; }

}  // extern "C"

pt_status pt_table_view(const pt_table *t, PtTableView *v) {
    if (!t || !v) return pt_fail(PT_BAD_ARG, "null argument");
    if (t->desc_mode || t->pca || !t->subs.empty() || t->p.init_random)
        return pt_fail(PT_UNSUPPORTED, "descriptor mode, PCA, multi-table tables and init_random serve pt_table_lookup, "
                                       "pt_table_lookup_device(_temporal) and the profile only");
    v->p = t->p;
    v->h = t->h; v->w = t->w; v->ds = t->ds;
    v->b_rgba = t->b_rgba.p;
    v->b_rgba1 = t->b_rgba1.p;
    v->table = t->table.p;
    v->to_bin = t->to_bin.p;
    v->kcoh = t->kcoh.p;
    v->bins = t->bins;
    v->b_desc = t->b_desc.p;
    v->allowed = t->allowed.p;
    v->part = t->part_dev.p;
    for (int d = 0; d < PT_DESC_MAX; d++) {
        v->part_ofs[d] = d < t->G ? t->part_ofs[d] : 0;
        v->nslices[d] = d < t->G ? t->nslices[d] : 0;
    }
    return PT_OK;
}

extern "C" {

void pt_kernel_launch_count_reset(void) { g_launches = 0; }

const char *pt_last_error(void) { return g_last_error.c_str(); }
const char *pt_version(void) { return "patchtable_b200 0.1 (sm_100a)"; }

/* Diagnostics (no reference counterpart): DT levels and SSD evaluations of the last lookup. */
int pt_table_dt_levels(const pt_table *t) { return t ? t->dt_levels : -1; }

}  // extern "C"
