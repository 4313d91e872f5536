/* Host-side launchers of the CUDA kernels (one translation unit per stage). */
#pragma once

#include <cuda_runtime.h>
#include <vector>

#include "pt_internal.h"

/* Colour conversion before the descriptor (get_padded_descriptor, patchtable.h:2510-2522):
   none, ARRAY_RGB2YUV, or Array::rgb2lab with its PowTable lookups. */
#define PT_COLOR_NONE 0
#define PT_COLOR_YUV 1
#define PT_COLOR_LAB 2
#define PT_LAB_N 1024
inline int pt_color_mode(const pt_params &p) { return p.convert_colorspace ? (p.colorspace == 1 ? PT_COLOR_LAB : PT_COLOR_YUV) : PT_COLOR_NONE; }
/* PowTable<float, 1024> contents for p = 2.4 and 1/3 (pt_pca.cpp) and their upload to the
   current device, once (k_descriptor.cu). */
void pt_lab_pow_tables(float (*tab)[PT_LAB_N]);
pt_status pt_lab_tables_ready();

/* k_descriptor.cu */
pt_status pt_descriptor_check(int ndims, int nchroma);
/* desc may be NULL (only the RGBA copy is written); rgba may be NULL. */
pt_status pt_launch_descriptor(int ndims, int nchroma, const float *rgb, int h, int w, int convert, float4 *rgba,
                               float *desc, int ds, cudaStream_t st);
/* Rows [trow0, trow0 + trows) of 8-patch descriptor tiles only (for banded lookups). */
pt_status pt_launch_descriptor_rows(int ndims, int nchroma, const float *rgb, int h, int w, int convert, float4 *rgba,
                                    float *desc, int ds, int trow0, int trows, cudaStream_t st);
/* -dim_algo pca: the basis fit on the host (pt_pca.cpp: mean[PT_PCA_DIM], basis[ncomp][PT_PCA_DIM],
   consuming 2 x samples rand() values like the reference) and the projection of every patch of an
   RGB image (k_descriptor.cu), which also writes the RGBA copy when rgba is set. */
#define PT_PCA_DIM 192
pt_status pt_pca_fit(const float *rgb, int h, int w, int convert, int samples, int subtract_mean, int ncomp,
                     std::vector<float> &mean, std::vector<float> &basis);
pt_status pt_launch_pca(const float *rgb, int h, int w, int convert, float4 *rgba, const float *mean, const float *basis,
                        int ncomp, float *desc, int ds, cudaStream_t st);
/* Descriptor mode: the store entries (ds floats per patch) of an H x W x nd descriptor image,
   padded (descriptor_padded: patches (H-14) x (W-14)) or not (patches H x W). */
pt_status pt_launch_descriptor_input(const float *in, int H, int W, int nd, int padded, float *desc, int ds,
                                     cudaStream_t st);

/* k_build.cu */
/* Device scratch of the range and partition stages.  The build runs them beside the k-coherence
   search, so the scratch is owned by the caller and freed after both have finished: a cudaFree
   inside the stages would wait for the whole device, the search included. */
#ifdef __CUDACC__
struct PtPartScratch {
    DevBuf<float> pmin, pmax, keys, sorted, picked;
    DevBuf<int> cnt, idx;
    DevBuf<unsigned char> tmp;
};
#else
struct PtPartScratch;
#endif
pt_status pt_launch_minmax(PtPartScratch &s, const float *desc, int ds, int G, long long P, const int *allowed,
                           int allowed_index, float *hmin, float *hmax, cudaStream_t st);
/* The partition sample of dimension d (every step-th allowed patch, patchtable.h:1193-1201) into
   s.keys; *count_out = its size. */
pt_status pt_quantile_gather(PtPartScratch &s, const float *desc, int ds, int d, int eh, int ew, int step,
                             const int *allowed, int allowed_index, int *count_out, cudaStream_t st);
/* vals[i] = the want[i]-th smallest of the n gathered values. */
pt_status pt_quantile_pick(PtPartScratch &s, int n, const std::vector<int> &want, std::vector<float> &vals,
                           cudaStream_t st);
/* Per-dimension get_bin parameters of a built table. */
struct PtBins {
    int G;
    float min_val[PT_DESC_MAX], range[PT_DESC_MAX];
    long long stride[PT_DESC_MAX];
};
/* Table entry of every query patch's cell (patchtable.h:3675-3686): tcand[p] = table[cell(p)]. */
pt_status pt_launch_table_candidates(const PtBins &bins, const float *desc, int ds, long long P, const int *to_bin,
                                     const int *table, int *tcand, cudaStream_t st);
/* The descriptor pass of query tile rows [trow0, trow0 + trows) fused with the table step: writes
   the RGBA copy and tcand[p] = table[cell(p)] for every patch of those rows, no descriptors. */
pt_status pt_launch_descriptor_cells(int ndims, int nchroma, const float *rgb, int h, int w, int convert, float4 *rgba,
                                     const PtBins &bins, const int *to_bin, const int *table, int *tcand, int trow0,
                                     int trows, cudaStream_t st);
/* k_table_build.cu: the table's cells in one cooperative launch -- fill with TABLE_UNUSED, populate in
   shuffle-rank order (rank[p] < 0: patch not allowed; order_xy[rank] = packed position), the
   propagation DT when run_dt (at most dt_iters levels when > 0), and fill_zeros with vfill when
   asked.  *seeded receives table_add_count, *levels the DT levels run.  Grid-barrier waits give up
   after pt_spin_limit() polls and the call returns PT_TIMEOUT. */
pt_status pt_build_cells(const PtBins &bins, const int *nslices, const float *desc, int ds, long long P, const int *rank,
                         const int *to_bin, const int *order_xy, int *table, long long ncells, int run_dt, int dt_iters,
                         int fill_zeros, int vfill, long long *seeded, int *levels, cudaStream_t st);
/* dt_algo 4 downsample, 5 hybrid (prop1 + downsample + unmask), 6 euclidean on a table whose
   populated cells hold packed positions. */
pt_status pt_dt_other(int *table, int G, const int *nslices, int dt_algo, cudaStream_t st);
/* dt_algo 2 brute: every cell takes the nearest of the P patches of the descriptor store (ds floats
   per patch, ew patches per row) under the partition's infinity norm; part / part_ofs hold each
   grid dimension's centres, lsizes and rsizes. */
pt_status pt_dt_brute(int *table, int G, const int *nslices, const float *part, const int *part_ofs, const float *desc,
                      int ds, long long P, int ew, cudaStream_t st);

/* k_kcoh.cu */
#define PT_KNN_WIDE_MAX 1024                 /* largest neighbour list of the k-coherence search */
pt_status pt_launch_knn(const float *train, int N, int nd, const float *qdesc, int Q, int K, int *out, cudaStream_t st);
pt_status pt_gather_rows(const float *desc, int ds, int nd, const int *rows, int n, float *out, cudaStream_t st);
/* The k-coherence index lists of a build without an allowed mask, generated on the device (train
   rows / positions, query rows / positions / cells, segment starts; buffers sized for every patch,
   seg for every query + 1); PT_UNSUPPORTED when the general host path must be used. */
pt_status pt_kc_lists(int ew, int eh, int fbs, int ks, int reset, int *trows, int *tpos, int *qrows, int *qpos,
                      int *qcell, int *seg, int *n_out, int *q_out, int *nseg_out, cudaStream_t st);
/* The same lists for a build with an allowed mask (allowed: ew x eh patches on the device):
   only points whose entry equals allowed_index, in the same order. */
pt_status pt_kc_lists_masked(int ew, int eh, int fbs, int ks, int reset, const int *allowed, int allowed_index,
                             int *trows, int *tpos, int *qrows, int *qpos, int *qcell, int *seg, int *n_out, int *q_out,
                             int *nseg_out, cudaStream_t st);
/* Exact distances from b_rgba (image mode) or, when bdesc is set, from the descriptor store
   (descriptor mode: ds floats per patch, ew patches per row). */
pt_status pt_kcoherence(const float4 *b_rgba, int bw, const float *bdesc, int ds, int ew, const float *train, int N, int nd, const int *tpos,
                        const float *qdesc, const int *qpos, const int *qcell, int Q, const int *seg_start, int nseg,
                        int kc, int min_dist, int2 *kcoh, int *max_knn_out, cudaStream_t st);

/* k_query.cu */
struct QuerySetup {
    int aw, ah, bw, bh;
    double prop_scale, triangle_factor;
    int kcoherence, kcoherence_step, radius;
    int kc_try = 0;          /* k-coherence neighbours tried per patch (0 = all kcoherence) */
    int step = 1;            /* neighbour spacing of a pull pass */
    int pull_max = 0;        /* most neighbour candidates a pull scores per patch (0 = all) */
    int tile = 0;            /* query patches per CTA in choose / pull: 32, 64, 128, 256 (0 = 32) */
    int row0 = 0, rows = 0;  /* patch rows [row0, row0 + rows) of a single-image launch (rows 0 = all) */
    const float4 *b1 = nullptr;   /* the table image shifted by one pixel, b1[i] = b[i + 1] */
    const int *allowed = nullptr; /* b patches a match may use (allowed[p] == allowed_index), or NULL */
    int allowed_index = 0;
    /* Descriptor mode (is_descriptor): distances are patch_dist_approx between the query's and the
       table's descriptor store entries (pt_descdist.cuh) instead of RGB patch SSDs. */
    const float *adesc = nullptr; /* query descriptors, (ah-7) x (aw-7) entries of ds floats, or NULL */
    const float *bdesc = nullptr; /* table descriptors, (bh-7) x (bw-7) entries of ds floats */
    int ds = 8, nd = 0;
    /* Further tables (ntables > 1, patchtable.h:3711-3738): their entries for every query patch,
       [table][patch], tried after the first table's in the table step. */
    const int *tcand_more = nullptr;
    int ntcand_more = 0;
    /* Random / spatial search after k-coherence (do_rs, spatial; patchtable.h:3854-3905) and the
       index of the pass, which seeds the random search. */
    int spatial = 0, do_rs = 0, pass = 0;
    /* Last pull of a query: the NNF is written here directly (x, y, dist as float64 per patch,
       the output step fused) instead of the next state arrays; NULL otherwise. */
    double *ann = nullptr;
    cudaStream_t stream;
};
/* Query schedule.  By default two choose + pull passes stand in for each of the reference's
   sequential sweeps (prop_iters, patchtable.h:3608), and the first pull reaches neighbours
   min(8, 2^(passes-1)) patches away, halving on each pass (jump flooding). */
inline int pt_default_passes(const pt_params &p) {
    if (p.gpu_prop_passes > 0) return p.gpu_prop_passes;
    return p.prop_iters <= 0 ? 0 : 2 * p.prop_iters;
}
inline int pt_default_jump(const pt_params &p, int passes) {
    if (p.gpu_jump > 0) return p.gpu_jump;
    int j = 1;
    for (int i = 1; i < passes && j < 8; i++) j *= 2;
    return j;
}
/* Whether choose pass i of `passes` runs k-coherence.  The reference runs it on every sweep, or
   only on sweep kcoherence_iter when that is >= 0 (patchtable.h:3612); GPU pass i stands in for
   sweep floor(i * prop_iters / passes), i.e. passes 2n and 2n+1 for sweep n by default. */
inline bool pt_pass_kcoh(const pt_params &p, int i, int passes) {
    if (p.kcoherence <= 0 || p.gpu_kc_max < 0) return false;
    if (p.kcoherence_iter < 0) return true;
    const int iters = p.prop_iters > 0 ? p.prop_iters : 1;
    const int sweep = passes > 0 ? (int) ((long long) i * iters / passes) : 0;
    return sweep == p.kcoherence_iter;
}
/* Neighbour spacing of pull pass i: halving from `jump` down to 1, then 1. */
inline int pt_pass_step(int i, int n, int jump) {
    (void) n;
    int s = jump > 1 ? jump : 1;
    for (int k = 0; k < i && s > 1; k++) s /= 2;
    return s;
}
pt_status pt_launch_init(int n, int pos, float d, int *cur_pos, float *cur_d, cudaStream_t st);
pt_status pt_launch_choose(const QuerySetup &s, int n, const float4 *a, const float4 *b, const int *cur_pos, const float *cur_d,
                           const int *tcand, const int2 *kcoh, int do_table, int *ch_pos,
                           float *ch_d, int *kc_done, int use_done, unsigned long long *evals, cudaStream_t st);
/* choose with the learned network's proposals (k_proposal.cu) for patches with lconf >= threshold;
   lcand (n x PT_PROP_TOPK table entries) may be NULL on passes without proposals; lcounters
   (may be NULL) accumulates {confident patches, proposals scored}. */
pt_status pt_launch_choose_learned(const QuerySetup &s, const float4 *a, const float4 *b, const int *cur_pos,
                                   const float *cur_d, const int *tcand, const int2 *kcoh, int do_table, int *ch_pos,
                                   float *ch_d, int *kc_done, int use_done, const int *lcand, const float *lconf,
                                   float threshold, int kcoh_confident, unsigned long long *evals,
                                   unsigned long long *lcounters, cudaStream_t st);
pt_status pt_launch_pull(const QuerySetup &s, int n, const float4 *a, const float4 *b, const int *cur_pos, const float *cur_d,
                         const int *ch_pos, const float *ch_d, int *nxt_pos, float *nxt_d,
                         unsigned long long *evals, cudaStream_t st);
/* Packed positions and float distances of a float64 NNF whose distances are float values. */
pt_status pt_launch_pack_nnf(long long n, const double *ann, int *pos, float *d, cudaStream_t st);
pt_status pt_launch_output(int n, const int *pos, const float *d, double *ann, cudaStream_t st);
/* Temporal lookups (ann_prev): initial field from the previous NNF and the final restore of the
   unscaled distance (patchtable.h:3548-3585, 4178-4193); *bad becomes 1 when a previous match lies
   outside the table image and sanitize is off. */
/* init_random: a hashed random match and its distance per patch. */
pt_status pt_launch_init_random(const QuerySetup &s, const float4 *a, const float4 *b, int *cur_pos, float *cur_d,
                                cudaStream_t st);
pt_status pt_launch_init_temporal(const QuerySetup &s, const double *prev, const float *scale_sv, int recalc, int sanitize,
                                  double temporal_scale, const float4 *a, const float4 *b, int *cur_pos, float *cur_d,
                                  double *orig, int *bad, cudaStream_t st);
pt_status pt_launch_output_temporal(int n, const int *pos, const float *d, const int *pos0, const float *d0,
                                    const double *orig, double *ann, cudaStream_t st);

/* Batched queries (pt_batch.cu): the images of a batch are concatenated -- pixels, patches and
   query state -- and every phase is one persistent launch over the flattened list of row
   segments, handed out one at a time through a work counter (`work`, zeroed by the launcher).  seg_off[t] is the image's first segment when a CTA covers PT_BATCH_TW(t) patches. */
#define PT_BATCH_NTW 4
struct PtBatchImage {
    int h, w, eh, ew;
    long long pix_off, patch_off;
    long long seg_off[PT_BATCH_NTW];
    long long tile_off;                  /* first 64 x 8 descriptor tile */
};
int pt_batch_tw(int twi);
pt_status pt_launch_choose_batch(const QuerySetup &s, const PtBatchImage *imgs, int n, long long nseg, int twi,
                                 const float4 *a, const float4 *b, const int *cur_pos, const float *cur_d,
                                 const int *tcand, const int2 *kcoh, int do_table, int *ch_pos, float *ch_d, int *kc_done,
                                 int use_done, unsigned long long *evals, unsigned long long *work, cudaStream_t st);
pt_status pt_launch_pull_batch(const QuerySetup &s, const PtBatchImage *imgs, int n, long long nseg, int twi,
                               const float4 *a, const float4 *b, const int *cur_pos, const float *cur_d, const int *ch_pos,
                               const float *ch_d, int *nxt_pos, float *nxt_d, unsigned long long *evals,
                               unsigned long long *work, cudaStream_t st);
/* The batch's descriptor pass fused with the table step: tcand[p] = table[cell(p)] for every
   patch of every image, no descriptors stored. */
pt_status pt_launch_descriptor_cells_batch(int ndims, int nchroma, const PtBatchImage *imgs, int n, long long ntiles,
                                           const float *rgb, int convert, float4 *rgba, const PtBins &bins, const int *to_bin,
                                           const int *table, int *tcand, unsigned long long *work, cudaStream_t st);

/* Read-only view of a built table, for entry points outside pt_table.cu. */
struct PtTableView {
    pt_params p;
    int h, w, ds;
    const float4 *b_rgba;
    const float4 *b_rgba1;               /* b_rgba shifted by one pixel (32-byte aligned row loads) */
    const int *table;
    const int *to_bin;
    const int2 *kcoh;
    PtBins bins;
    const float *b_desc;                 /* (h-7) x (w-7) x ds */
    const int *allowed;                  /* (h-7) x (w-7) allowed mask of the build, or NULL */
    const float *part;                   /* per grid dimension: centres, left sizes, right sizes */
    int part_ofs[PT_DESC_MAX];           /* offset of dimension d's centres in part */
    int nslices[PT_DESC_MAX];
};
pt_status pt_table_view(const pt_table *t, PtTableView *v);

/* k_proposal.cu */
pt_status pt_prop_check_table(const PtTableView &v);
pt_status pt_launch_prop_samples(const PtTableView &v, const float *qdesc, int n, const double *ann, void *X,
                                 unsigned char *labels, cudaStream_t st);
pt_status pt_launch_prop_infer(const PtTableView &v, pt_proposal *q, const float *qdesc, int n, int *cand, float *conf,
                               float *logits, cudaStream_t st);
float pt_prop_threshold(const pt_proposal *q);
int pt_prop_kcoh_confident(const pt_proposal *q);
pt_status pt_prop_check_error(pt_proposal *q, cudaStream_t st);
