/* Batched queries: many query images of any sizes against one table, in one pass of launches.

   The reference matches one image per lookup() call (patchtable/patchtable.h:4448).  A batch
   concatenates its images -- RGB pixels, RGBA copies, table entries, query state and the float64
   NNF -- and runs every phase of the query once for all of them: one descriptor launch over the
   flattened list of 64 x 8 descriptor tiles that also looks each patch's cell up in the table,
   and per propagation pass one choose and one pull launch over the flattened list of row segments
   (the first pass starts from the initial field, the last pull writes the NNF).  The choose /
   pull / descriptor launches are persistent (as many CTAs as fit on the GPU); a work counter per
   launch hands the segments out one at a time to whichever CTA is free, and each CTA finds the
   image that owns its segment by binary search over per-image prefix counts.  Every patch is computed exactly as the
   single-image query computes it, so each image's NNF equals its own pt_table_lookup_device
   result.

   The number of query patches a CTA covers (32, 64, 128 or 256) is picked by pt_batch_autotune,
   and the whole launch sequence can be captured once into a CUDA graph (pt_batch_capture) and
   replayed (pt_batch_replay) with no host work per launch. */
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "pt_internal.h"
#include "pt_kernels.h"

struct pt_batch {
    pt_table *t = nullptr;
    int n = 0;
    std::vector<PtBatchImage> imgs;
    DevBuf<PtBatchImage> d_imgs;
    long long npix = 0, P = 0, ntiles = 0, nseg[PT_BATCH_NTW] = {0, 0, 0, 0};
    int twi = PT_BATCH_NTW - 1;           /* 256 query patches per CTA until tuned */
    DevBuf<float4> rgba;
    DevBuf<int> tcand, pos[2], chpos, kcdone;
    DevBuf<float> dd[2], chd;
    DevBuf<unsigned long long> work;      /* work counters of the persistent launches */
    cudaStream_t cap_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~pt_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (cap_stream) cudaStreamDestroy(cap_stream);
    }
};

namespace {

constexpr int DESC_TW = 64, DESC_TH = 8;   /* descriptor tile (k_descriptor.cu) */

pt_status run(pt_batch *B, const float *d_rgb, double *d_ann, cudaStream_t st) {
    PtTableView v;
    PT_TRY(pt_table_view(B->t, &v));
    const pt_params &p = v.p;
    const int ds = v.ds;
    (void) ds;
    /* descriptors are needed only for the table step: one fused pass writes the table entries */
    PT_TRY(pt_launch_descriptor_cells_batch(p.ndims, p.nchroma, B->d_imgs.p, B->n, B->ntiles, d_rgb, pt_color_mode(p),
                                            B->rgba.p, v.bins, v.to_bin, v.table, B->tcand.p, B->work.p, st));
    QuerySetup qs;
    qs.aw = 0; qs.ah = 0; qs.bw = v.w; qs.bh = v.h;
    qs.prop_scale = 1.0 / (1 + p.coherence_spatial);
    qs.triangle_factor = p.triangle_factor;
    qs.kcoherence = p.kcoherence;
    qs.kc_try = p.gpu_kc_max;
    qs.kcoherence_step = p.kcoherence_step;
    qs.spatial = p.spatial;
    qs.do_rs = p.do_rs;
    qs.radius = std::min(2, p.query_step + p.prop_dist);
    qs.b1 = v.b_rgba1;
    qs.pull_max = p.gpu_pull_max;
    qs.allowed = v.allowed;
    qs.allowed_index = p.allowed_index;
    qs.stream = st;
    const int n = (int) B->P;
    /* the first pass starts from the initial field without state arrays; the last pull writes
       the NNF */
    const int passes = pt_default_passes(p);
    const bool direct_out = p.do_prop && passes > 0;
    const int jump = pt_default_jump(p, passes);
    int cur = 0;
    for (int i = 0; i < passes; i++) {
        const bool do_table = i == 0 && p.do_table_lookup;
        QuerySetup qi = qs;
        qi.pass = i;
        if (!pt_pass_kcoh(p, i, passes)) qi.kcoherence = 0;
        const int use_done = i > 0 && pt_pass_kcoh(p, i - 1, passes);
        PT_TRY(pt_launch_choose_batch(qi, B->d_imgs.p, B->n, B->nseg[B->twi], B->twi, B->rgba.p, v.b_rgba,
                                      i == 0 ? nullptr : B->pos[cur].p, i == 0 ? nullptr : B->dd[cur].p, B->tcand.p, v.kcoh,
                                      do_table, B->chpos.p, B->chd.p, B->kcdone.p, use_done, nullptr, B->work.p + 1, st));
        if (p.do_prop) {
            QuerySetup qp = qs;
            qp.step = pt_pass_step(i, passes, jump);
            if (i == passes - 1 && direct_out) qp.ann = d_ann;
            PT_TRY(pt_launch_pull_batch(qp, B->d_imgs.p, B->n, B->nseg[B->twi], B->twi, B->rgba.p, v.b_rgba,
                                        i == 0 ? nullptr : B->pos[cur].p, i == 0 ? nullptr : B->dd[cur].p, B->chpos.p, B->chd.p,
                                        B->pos[1 - cur].p, B->dd[1 - cur].p, nullptr, B->work.p + 2, st));
            cur = 1 - cur;
        } else {
            PT_CUDA(cudaMemcpyAsync(B->pos[cur].p, B->chpos.p, sizeof(int) * n, cudaMemcpyDeviceToDevice, st));
            PT_CUDA(cudaMemcpyAsync(B->dd[cur].p, B->chd.p, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
        }
    }
    if (direct_out) return PT_OK;
    if (passes == 0) PT_TRY(pt_launch_init(n, pt_xy(v.w - 7 + 1, 0), (float) PT_DIST_INF, B->pos[0].p, B->dd[0].p, st));
    return pt_launch_output(n, B->pos[cur].p, B->dd[cur].p, d_ann, st);
}

}  // namespace

extern "C" {

pt_status pt_batch_create(pt_table *t, int n, const int *h, const int *w, pt_batch **out) {
    if (!t || !out || n < 1 || !h || !w) return pt_fail(PT_BAD_ARG, "pt_batch_create: null argument or empty batch");
    *out = nullptr;
    PtTableView v;
    PT_TRY(pt_table_view(t, &v));
    PT_TRY(pt_descriptor_check(v.p.ndims, v.p.nchroma));
    pt_batch *B = new pt_batch();
    B->t = t;
    B->n = n;
    B->imgs.resize(n);
    long long pix = 0, pat = 0, tiles = 0, seg[PT_BATCH_NTW] = {0, 0, 0, 0};
    for (int i = 0; i < n; i++) {
        if (h[i] < 8 || w[i] < 8 || w[i] > 65535 || h[i] > 16383) {
            delete B;
            return pt_fail(PT_BAD_ARG, "batch image %d is %dx%d: each side must be 8..16383 (width 8..65535)", i, w[i], h[i]);
        }
        PtBatchImage &g = B->imgs[i];
        g.h = h[i]; g.w = w[i]; g.eh = h[i] - 7; g.ew = w[i] - 7;
        g.pix_off = pix;
        g.patch_off = pat;
        g.tile_off = tiles;
        for (int k = 0; k < PT_BATCH_NTW; k++) {
            g.seg_off[k] = seg[k];
            const int tw = pt_batch_tw(k);
            seg[k] += (long long) g.eh * ((g.ew + tw - 1) / tw);
        }
        pix += (long long) h[i] * w[i];
        pat += (long long) g.eh * g.ew;
        tiles += (long long) ((g.ew + DESC_TW - 1) / DESC_TW) * ((g.eh + DESC_TH - 1) / DESC_TH);
    }
    if (pat >= (1ll << 31)) {
        delete B;
        return pt_fail(PT_BAD_ARG, "batch of %lld patches exceeds 2^31", pat);
    }
    B->npix = pix;
    B->P = pat;
    B->ntiles = tiles;
    for (int k = 0; k < PT_BATCH_NTW; k++) B->nseg[k] = seg[k];
    auto fail = [&](pt_status s) { delete B; return s; };
    if (B->d_imgs.reserve(n) || B->rgba.reserve(pix) || B->tcand.reserve(pat) ||
        B->pos[0].reserve(pat) || B->pos[1].reserve(pat) || B->dd[0].reserve(pat) || B->dd[1].reserve(pat) ||
        B->chpos.reserve(pat) || B->chd.reserve(pat) || B->kcdone.reserve(pat) || B->work.reserve(3))
        return fail(pt_fail(PT_OOM, "batch buffers for %lld pixels / %lld patches", pix, pat));
    if (cudaMemcpy(B->d_imgs.p, B->imgs.data(), sizeof(PtBatchImage) * n, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(pt_fail(PT_CUDA_ERR, "batch geometry upload"));
    *out = B;
    return PT_OK;
}

void pt_batch_free(pt_batch *b) { delete b; }

pt_status pt_batch_layout(const pt_batch *b, int64_t *pixel_offset, int64_t *patch_offset, int64_t *totals) {
    if (!b) return pt_fail(PT_BAD_ARG, "null batch");
    for (int i = 0; i < b->n; i++) {
        if (pixel_offset) pixel_offset[i] = b->imgs[i].pix_off;
        if (patch_offset) patch_offset[i] = b->imgs[i].patch_off;
    }
    if (totals) { totals[0] = b->npix; totals[1] = b->P; }
    return PT_OK;
}

pt_status pt_batch_set_tile(pt_batch *b, int patches_per_cta) {
    if (!b) return pt_fail(PT_BAD_ARG, "null batch");
    for (int k = 0; k < PT_BATCH_NTW; k++)
        if (pt_batch_tw(k) == patches_per_cta) {
            b->twi = k;
            return PT_OK;
        }
    return pt_fail(PT_BAD_ARG, "patches per CTA must be 32, 64, 128 or 256 (got %d)", patches_per_cta);
}

int pt_batch_tile(const pt_batch *b) { return b ? pt_batch_tw(b->twi) : 0; }

pt_status pt_batch_lookup(pt_batch *b, const float *d_rgb, double *d_ann, void *stream) {
    if (!b || !d_rgb || !d_ann) return pt_fail(PT_BAD_ARG, "null argument");
    return run(b, d_rgb, d_ann, (cudaStream_t) stream);
}

pt_status pt_batch_autotune(pt_batch *b, const float *d_rgb, double *d_ann, void *stream, int *best, float *ms_out) {
    if (!b || !d_rgb || !d_ann) return pt_fail(PT_BAD_ARG, "null argument");
    cudaStream_t st = (cudaStream_t) stream;
    cudaEvent_t e0, e1;
    PT_CUDA(cudaEventCreate(&e0));
    PT_CUDA(cudaEventCreate(&e1));
    const int keep = b->twi;
    float best_ms = 0.f;
    int best_k = keep;
    pt_status s = PT_OK;
    for (int k = 0; k < PT_BATCH_NTW && s == PT_OK; k++) {
        b->twi = k;
        s = run(b, d_rgb, d_ann, st);                       /* warm-up */
        float tot = 0.f;
        for (int r = 0; r < 3 && s == PT_OK; r++) {
            if (cudaEventRecord(e0, st) != cudaSuccess) { s = pt_fail(PT_CUDA_ERR, "event"); break; }
            s = run(b, d_rgb, d_ann, st);
            if (s != PT_OK) break;
            float ms = 0.f;
            if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) { s = pt_fail(PT_CUDA_ERR, "autotune timing"); break; }
            tot = r == 0 ? ms : std::min(tot, ms);
        }
        if (s != PT_OK) break;
        if (ms_out) ms_out[k] = tot;
        if (k == 0 || tot < best_ms) { best_ms = tot; best_k = k; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->twi = s == PT_OK ? best_k : keep;
    if (best) *best = pt_batch_tw(b->twi);
    return s;
}

pt_status pt_batch_capture(pt_batch *b, const float *d_rgb, double *d_ann, void *stream) {
    (void) stream;                         /* the graph is recorded on the batch's own stream */
    if (!b || !d_rgb || !d_ann) return pt_fail(PT_BAD_ARG, "null argument");
    if (!b->cap_stream) PT_CUDA(cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking));
    /* one eager run first: every launch attribute and occupancy query is settled outside capture */
    PT_TRY(run(b, d_rgb, d_ann, b->cap_stream));
    PT_CUDA(cudaStreamSynchronize(b->cap_stream));
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    PT_CUDA(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
    pt_status s = run(b, d_rgb, d_ann, b->cap_stream);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->cap_stream, &g);
    if (s != PT_OK) { if (g) cudaGraphDestroy(g); return s; }
    if (e != cudaSuccess) return pt_fail(PT_CUDA_ERR, "graph capture: %s", cudaGetErrorString(e));
    b->graph = g;
    PT_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
    return PT_OK;
}

pt_status pt_batch_replay(pt_batch *b, void *stream) {
    if (!b) return pt_fail(PT_BAD_ARG, "null batch");
    if (!b->exec) return pt_fail(PT_BAD_ARG, "pt_batch_replay before pt_batch_capture");
    PT_CUDA(cudaGraphLaunch(b->exec, (cudaStream_t) stream));
    return PT_OK;
}

pt_status pt_table_lookup_batch(pt_table *t, int n, const float *const *a, const int *h, const int *w,
                                double *const *ann_out) {
    if (!t || n < 0 || (n > 0 && (!a || !h || !w || !ann_out))) return pt_fail(PT_BAD_ARG, "null argument");
    if (n == 0) return PT_OK;
    for (int i = 0; i < n; i++)
        if (!a[i] || !ann_out[i]) return pt_fail(PT_BAD_ARG, "null image or output %d", i);
    pt_batch *B = nullptr;
    PT_TRY(pt_batch_create(t, n, h, w, &B));
    struct Guard { pt_batch *b; ~Guard() { pt_batch_free(b); } } guard{B};
    PtTableView v;
    PT_TRY(pt_table_view(t, &v));
    DevBuf<float> rgb;
    DevBuf<double> ann;
    PT_CUDA(rgb.reserve((size_t) B->npix * 3));
    PT_CUDA(ann.reserve((size_t) B->P * 3));
    cudaStream_t st = nullptr;
    PT_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct SGuard { cudaStream_t s; ~SGuard() { cudaStreamDestroy(s); } } sguard{st};
    for (int i = 0; i < n; i++)
        PT_CUDA(cudaMemcpyAsync(rgb.p + 3 * B->imgs[i].pix_off, a[i], sizeof(float) * 3 * (size_t) h[i] * w[i],
                                cudaMemcpyHostToDevice, st));
    PT_TRY(run(B, rgb.p, ann.p, st));
    for (int i = 0; i < n; i++)
        PT_CUDA(cudaMemcpyAsync(ann_out[i], ann.p + 3 * B->imgs[i].patch_off,
                                sizeof(double) * 3 * (size_t) B->imgs[i].eh * B->imgs[i].ew, cudaMemcpyDeviceToHost, st));
    PT_CUDA(cudaStreamSynchronize(st));
    return PT_OK;
}

}  // extern "C"
