/* patchtable_b200 -- C ABI of the B200 PatchTable build + query path.

   Plain pointers and sizes only; no CUDA or torch types cross this boundary (streams are passed
   as void *).  Every entry point returns a pt_status; pt_last_error() gives the message of the
   last failure on the calling thread.  Host buffers are never retained: the library copies
   what it needs to device memory.

   Each declaration names the reference interface it replaces (paths relative to the
   reference project root, uva-graphics/patchtable). */
#ifndef PATCHTABLE_B200_H
#define PATCHTABLE_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PT_OK = 0,
    PT_BAD_ARG = 1,       /* invalid size, pointer or parameter */
    PT_OOM = 2,           /* device or host allocation failed */
    PT_CUDA_ERR = 3,      /* a CUDA call failed; see pt_last_error() */
    PT_TIMEOUT = 4,       /* a bounded device wait gave up */
    PT_UNSUPPORTED = 5,   /* parameter combination not implemented on the GPU path */
    PT_IO = 6             /* table file could not be read or written */
} pt_status;

#define PT_MAX_DIMS 16
#define PT_PATH_MAX 256

/* Numeric fields of PatchTableParams (patchtable/patchtable_params.h:23-161) read by the
   build/query path, with the reference's names and meanings. */
typedef struct pt_params {
    double limit;                 /* max table cells (switch value x 1e6), patchtable.cpp:171 */
    int ndims, nchroma, grid_ndims;
    int nslices[PT_MAX_DIMS];     /* explicit -nslices (n_nslices > 0) */
    int n_nslices;
    int partition_step;
    int populate_random, populate_nearest;
    int run_dt, dt_algo, dt_iters;        /* dt_algo: 0 raster 1 prop 2 brute 3 kdtree 4 downsample 5 hybrid 6 euclidean */
    int kcoherence, kcoherence_min_dist, kcoherence_step, kcoherence_iter;
    int flann_reset_step, flann_build_step;
    double triangle_factor;
    int prop_iters, query_step, do_prop, prop_dist;
    double coherence_spatial, coherence_temporal;
    int do_table_lookup, do_rs, spatial;
    int allowed_index;
    int recalc_dist_temporal, sanitize_input, init_random;
    int convert_colorspace, colorspace;   /* colorspace: 0 yuv, 1 lab */
    int is_descriptor, descriptor_padded;
    int patch_w;
    int threads, verbose, query_iters, ntables;
    double table_ratio;
    int lookup_algo, kcoherence_algo, dim_algo;
    int incoherence, randomize_dt, parallel_dt, populate_exptime, dt_mode;
    char load_filename[PT_PATH_MAX];
    char save_filename[PT_PATH_MAX];
    /* GPU query schedule (no reference counterpart): number of parallel propagation passes
       that replace the reference's sequential scanline sweeps (0 picks the default), and the
       neighbour spacing of the first pass, halved on each later pass down to 1 (jump
       flooding; 0 or 1 = plain neighbours), and the most neighbour offsets a pull pass scores per
       patch, best-first by the neighbour's own distance (0 = all of them), and the query patches one
       CTA covers in the choose and pull kernels (32, 64, 128 or 256; 0 picks the default, 32; the
       result does not depend on it). */
    int gpu_prop_passes;
    int gpu_jump;
    int gpu_pull_max;
    int gpu_tile;
    /* -dim_algo pca (patch_pca.h): random patches fitted, mean subtracted from them, first channel
       from the patch mean (patchtable.cpp:86-89, 226-228). */
    int pca_samples, pca_subtract_mean, pca_mean;
    /* Row bands of the pipelined host lookup (no reference counterpart; 0 sizes them so that a
       band's launches fill whole waves of the GPU): uploads, kernels and downloads of consecutive
       bands overlap.  The result does not depend on it. */
    int gpu_bands;
    /* k-coherence neighbours the query tries per patch (no reference counterpart; a GPU schedule
       knob like gpu_pull_max): 0 = every one the set lists (the reference's behaviour), n > 0 =
       at most the first n, negative = none (the table step and the pulls alone; the table's
       k-coherence set is still built).  Trades NNF quality for speed; distances stay exact. */
    int gpu_kc_max;
} pt_params;

typedef struct pt_table pt_table;

/* PatchTableParams::PatchTableParams() = set_defaults() + set_speed(3),
   patchtable.cpp:26-136, 380-382. */
void pt_params_default(pt_params *p);

/* PatchTableParams::set_speed(i), patchtable.cpp:138-150.  PT_BAD_ARG unless 0 <= i <= 9.
   As in the reference, the preset string's first switch (-ndims) is not applied. */
pt_status pt_params_set_speed(pt_params *p, int speed);

/* PatchTableParams::set_from_switches(string), patchtable.cpp:152-373: "-name value" pairs with
   the reference's switch names, "-speed" applied first, "-limit" in millions.  Exactly like the
   reference, the first token of the string is ignored (it fills argv[0]); pass a command line
   such as "patchtable -speed 3 -coherence_spatial 4" to have every switch applied. */
pt_status pt_params_from_switches(pt_params *p, const char *switches);

/* PatchTable<float,float,int32_t>(PatchTableParams *p, const Array<float> &b,
   Array<int32_t> *allowed_patches = NULL), patchtable.h:4397-4424 -> PatchTableFixedN ctor
   patchtable.h:2584-3373.  b is h x w x 3 float RGB (row-major, channels interleaved);
   allowed is (h-7) x (w-7) int32 or NULL.  In descriptor mode (p->is_descriptor, 3 <= channels
   <= 16) b is h x w x channels descriptors, the table takes ndims = channels and nchroma = 0
   (patchtable.h:4398-4401), every pixel is a patch (every pixel but a 7-wide border with
   p->descriptor_padded, patchtable.h:2498-2507), allowed holds one entry per such patch, and
   distances are patch_dist_approx of the descriptors (patchtable.h:376-437).  Descriptor mode
   tables serve pt_table_lookup, pt_table_lookup_device(_temporal) and pt_table_lookup_profile;
   batches, learned proposals and table files return PT_UNSUPPORTED. */
pt_status pt_table_create(const pt_params *p, const float *b, int h, int w, int channels,
                          const int32_t *allowed, pt_table **out);

/* PatchTableFixedN(p, b, allowed, b0_no_copy, wh0_no_copy), patchtable.h:2584: build from a
   precomputed padded descriptor wh0 of (h+7) x (w+7) x ndims floats instead of computing it. */
pt_status pt_table_create_with_descriptor(const pt_params *p, const float *b, int h, int w,
                                          const float *wh0, const int32_t *allowed, pt_table **out);

/* PatchTableFixedN(PatchTableParams *, string filename) / load(), patchtable.h:1574-1622: reads
   the reference's table file (PT_IO if it is not one, PT_BAD_ARG if its descriptor dimensions
   differ from p->ndims).  The file holds no k-coherence set; it is rebuilt from the stored
   descriptors when p->kcoherence > 0.  pt_table_create also loads when p->load_filename is set
   and saves after building when p->save_filename is set, as the reference's constructor does. */
pt_status pt_table_load(const pt_params *p, const char *filename, pt_table **out);

/* PatchTable<>::save(string), patchtable.h:4470-4490 / PatchTableFixedN::save, :1574-1605, in
   the reference's format (the reference loads it).  The padding rows and columns of wh0, which
   this library does not keep, are written as 0. */
pt_status pt_table_save(const pt_table *t, const char *filename);

/* Image size (b0) of a table, e.g. one loaded from a file. */
pt_status pt_table_image_shape(const pt_table *t, int *h, int *w);

void pt_table_free(pt_table *t);

/* With ntables > 1 the table keeps ntables-1 further tables of b, built like the reference's
   (patchtable.h:3359-3371: limit int(limit / table_ratio^i), no k-coherence) and tried in order in
   the query's table step (patchtable.h:3711-3735).  *out receives further table i (0-based) as a
   handle owned by t (do not free it), for inspection with the accessors below. */
pt_status pt_table_subtable(pt_table *t, int i, pt_table **out);

/* The reference's table keeps a pointer to the caller's PatchTableParams (patchtable.h:1546) and
   lookup() reads the query fields from it on every call (prop_iters, query_step, prop_dist,
   do_prop, do_table_lookup, coherence_spatial/temporal, recalc_dist_temporal, sanitize_input,
   triangle_factor, kcoherence_iter, do_rs, spatial).  This copies those fields (and the GPU
   schedule fields) into the table; fields that shaped the build are left unchanged.  The random
   search (do_rs) draws its neighbour from a hash of the patch and pass instead of rand(), so it
   is deterministic and consumes no rand() values. */
pt_status pt_table_set_params(pt_table *t, const pt_params *p);

/* double PatchTable<>::lookup(const Array<float> &a, Array<double> &ann,
   Array<double> *ann_prev = NULL, Array<float> *coherence_temporal_sv = NULL),
   patchtable.h:4448-4468 -> lookup_templated, :3468-4217.
   a: h x w x 3 host floats.  ann_out: (h-7) x (w-7) x 3 host doubles [NNF_X, NNF_Y, NNF_DIST]
   (patchtable.h:175-177).  ann_prev: same layout or NULL.  coh_sv: (h-7) x (w-7) floats or NULL.
   *seconds (may be NULL) receives the wall time of the call including a's descriptor, like the
   reference's return value (patchtable.h:3477, 4211).  In descriptor mode a is h x w x ndims
   descriptors and the NNF has h x w records ((h-14) x (w-14) with descriptor_padded). */
pt_status pt_table_lookup(pt_table *t, const float *a, int h, int w, double *ann_out,
                          const double *ann_prev, const float *coh_sv, double *seconds);

/* Device-resident form of pt_table_lookup (no reference counterpart; the reference has no
   device memory): d_a and d_ann are device pointers with the host layouts above; the call is
   asynchronous on `stream` (a cudaStream_t, NULL = legacy default stream). */
pt_status pt_table_lookup_device(pt_table *t, const float *d_a, int h, int w, double *d_ann,
                                 void *stream);

/* Device form of pt_table_lookup with the previous frame's NNF (patchtable.h:3548-3585,
   4178-4193): d_ann_prev ((h-7) x (w-7) x 3 doubles) seeds the field; d_coh_sv ((h-7) x (w-7)
   floats, may be NULL) replaces the temporal scale 1/(1+coherence_temporal) per patch when the
   distance is recomputed (recalc_dist_temporal).  Previous matches outside the table image are
   clamped (the host form reports them with PT_BAD_ARG when sanitize_input is 0). */
pt_status pt_table_lookup_device_temporal(pt_table *t, const float *d_a, int h, int w, const double *d_ann_prev,
                                         const float *d_coh_sv, double *d_ann, void *stream);

/* Zero-allocation form of pt_table_lookup_device (no counterpart in the reference).  For
   callers that may not allocate device memory during queries -- a frame loop with a fixed
   latency budget (cudaMalloc/cudaFree synchronise the device), or an application whose own
   allocator owns the GPU's memory -- every intermediate buffer comes from one 20 MiB file-scope
   device array instead of cudaMalloc.  Limits: at most PT_NOALLOC_MAX_PIXELS query pixels and
   ndims <= 8 (PT_BAD_ARG / PT_UNSUPPORTED otherwise).  All calls share that array, so calls
   that overlap on the GPU race and must be serialised.  The first call on a device resolves the
   array's address (cudaGetSymbolAddress) and should come before any stream capture. */
#define PT_NOALLOC_MAX_PIXELS (1 << 18)
pt_status pt_table_lookup_device_noalloc(pt_table *t, const float *d_a, int h, int w, double *d_ann,
                                         void *stream);

/* Batched query (no reference counterpart; the reference matches one image per lookup() call,
   patchtable.h:4448): n query images of individual sizes against one table.  The images are
   concatenated on the device and every phase of the query is one launch for all of them
   (persistent kernels over the flattened list of row segments).  a[i] / ann_out[i] are host
   buffers with the pt_table_lookup layouts; each ann_out[i] equals what pt_table_lookup returns
   for a[i] alone. */
pt_status pt_table_lookup_batch(pt_table *t, int n, const float *const *a, const int *h,
                                const int *w, double *const *ann_out);

/* Reusable device-side batch (no reference counterpart).  pt_batch_create fixes the image sizes
   and allocates the concatenated buffers; pt_batch_layout gives each image's first pixel (RGB
   triples) in the concatenated input and first patch (NNF record) in the concatenated output,
   and totals[2] = {pixels, patches}.  pt_batch_lookup enqueues the whole query on `stream`
   (d_rgb: concatenated h x w x 3 floats; d_ann: concatenated (h-7) x (w-7) x 3 doubles) with the
   table's current parameters.  pt_batch_set_tile / pt_batch_autotune choose how many query
   patches one CTA covers (32, 64, 128, 256; the results do not depend on it): the autotuner
   times each on the given inputs and keeps the fastest (ms_out[4] receives the times).
   pt_batch_capture records the launch sequence for these two buffers and the current parameters
   into a CUDA graph; pt_batch_replay launches that graph on `stream`. */
typedef struct pt_batch pt_batch;
pt_status pt_batch_create(pt_table *t, int n, const int *h, const int *w, pt_batch **out);
void pt_batch_free(pt_batch *b);
pt_status pt_batch_layout(const pt_batch *b, int64_t *pixel_offset, int64_t *patch_offset, int64_t *totals);
pt_status pt_batch_set_tile(pt_batch *b, int patches_per_cta);
int pt_batch_tile(const pt_batch *b);
pt_status pt_batch_lookup(pt_batch *b, const float *d_rgb, double *d_ann, void *stream);
pt_status pt_batch_autotune(pt_batch *b, const float *d_rgb, double *d_ann, void *stream, int *best,
                            float *ms_out);
pt_status pt_batch_capture(pt_batch *b, const float *d_rgb, double *d_ann, void *stream);
pt_status pt_batch_replay(pt_batch *b, void *stream);

/* Diagnostics (no reference counterpart): pt_table_lookup_device with a CUDA event after every
   stage.  stage_ms[6] receives the summed device time of {descriptor, cells, init, choose, pull,
   output}; counters[4] = {choose candidates, choose SSD rows, pull candidates, pull SSD rows}
   (one SSD row = 24 subtractions, multiplications and additions).  Synchronizes the stream. */
pt_status pt_table_lookup_profile(pt_table *t, const float *d_a, int h, int w, double *d_ann,
                                  void *stream, double *stage_ms, uint64_t *counters);

/* Diagnostics (no reference counterpart; the reference prints its own stage times when verbose,
   patchtable.h:2531-2580, 3107-3117): wall-clock milliseconds of the table build's stages, each
   ended with the stream drained.  ms[PT_BUILD_NSTAGES] = {descriptor (upload, descriptor, shifted
   copy), k-coherence, range + partition, populate order (host shuffle), populate + distance
   transform, total}. */
#define PT_BUILD_DESCRIPTOR 0
#define PT_BUILD_KCOHERENCE 1
#define PT_BUILD_PARTITION 2
#define PT_BUILD_SHUFFLE 3
#define PT_BUILD_POPULATE_DT 4
#define PT_BUILD_TOTAL 5
#define PT_BUILD_NSTAGES 6
pt_status pt_table_build_profile(const pt_table *t, double *ms, int n);

/* Diagnostics (no reference counterpart): C = A * B^T in FP32 through the hand-written tcgen05
   BF16 GEMM of the proposal network.  A [M x K], B [N x K] row-major BF16 device arrays (lda, ldb
   multiples of 8; K a multiple of 16; N in {16, 32, 64, 128, 256}); C [M x N] FP32, ldc.
   *err_flag (device int, may be NULL) becomes 1 if a bounded wait inside the kernel gave up. */
pt_status pt_tc_gemm_f32(const void *A, int lda, const void *B, int ldb, float *C, int ldc, int M, int N,
                         int K, int *err_flag, void *stream);

/* ---- learned proposal (no reference counterpart) ----

   A small network proposes, for every query patch, the PT_PROP_TOPK table cells most likely to
   hold its match; their stored patches are scored by the same exact SSD as every other candidate.
   The network (16 -> 128 -> ReLU -> 128 -> ReLU -> 32) works on tables of at most PT_PROP_DIMS
   grid dimensions: for each dimension it scores the match's bin offset -2..+2 from the query
   patch's own bin (PT_PROP_CLASSES logits); a cell's probability is the product over dimensions.
   BF16 weights and activations, FP32 accumulation, FP32 master weights; every kernel is the
   library's own tcgen05 code.  Device pointers throughout; `stream` is a cudaStream_t (NULL: the
   CUDA default stream), and the calls are asynchronous on it unless stated otherwise.  Calls on
   different streams must be ordered by the caller. */
#define PT_PROP_IN 16
#define PT_PROP_HIDDEN 128
#define PT_PROP_OUT 32
#define PT_PROP_DIMS 6
#define PT_PROP_CLASSES 5
#define PT_PROP_TOPK 8

typedef struct pt_proposal pt_proposal;

/* New network with He-initialised weights drawn from seed; threshold 0.5. */
pt_status pt_proposal_create(uint32_t seed, pt_proposal **out);
void pt_proposal_free(pt_proposal *net);
/* Length of the FP32 parameter vector: W1 [128 x 16], b1, W2 [128 x 128], b2, W3 [32 x 128], b3. */
int pt_proposal_num_params(void);
pt_status pt_proposal_get_params(pt_proposal *net, float *host);
/* Replaces the parameters (host FP32) and resets the optimiser state. */
pt_status pt_proposal_set_params(pt_proposal *net, const float *host);
/* Patches whose most probable cell has probability below threshold keep the plain candidates
   (table cell + k-coherence); with kcoh_confident the confident ones also try k-coherence. */
pt_status pt_proposal_configure(pt_proposal *net, float threshold, int kcoh_confident);
/* Training batch: X [B x 16] BF16 features and labels [B x 8] bytes from pt_table_proposal_samples;
   B a positive multiple of 64.  One AdamW step (lr, decoupled weight decay wd); *loss (may be
   NULL; if given, the call synchronises) receives the batch's mean cross-entropy summed over the
   grid dimensions. */
pt_status pt_proposal_train_step(pt_proposal *net, const void *X, const uint8_t *labels, int B, float lr,
                                 float wd, float *loss, void *stream);
/* Mean loss and the FP32 gradient (host, pt_proposal_num_params floats) of a batch, no update. */
pt_status pt_proposal_gradient(pt_proposal *net, const void *X, const uint8_t *labels, int B, float *loss,
                               float *grad_host, void *stream);
/* logits [B x 32] FP32 of X [B x 16] BF16 (three GEMM launches); synchronises. */
pt_status pt_proposal_forward(pt_proposal *net, const void *X, int B, float *logits, void *stream);
/* Waits for the stream and reports a tensor-core wait that gave up (PT_TIMEOUT). */
pt_status pt_proposal_sync(pt_proposal *net, void *stream);

/* Training samples from a query image d_a (device h x w x 3) and an NNF d_ann of it against this
   table (device doubles, pt_table_lookup layout): X [(h-7)(w-7) x 16] BF16 features and labels
   [(h-7)(w-7) x 8] bytes (per grid dimension: offset class | valid-below << 3 | valid-above << 5,
   0xFF when unused; byte 6 = 1 when the match's bin lies within the 5 x ... x 5 window). */
pt_status pt_table_proposal_samples(pt_table *t, const float *d_a, int h, int w, const double *d_ann,
                                    void *X, uint8_t *labels, void *stream);
/* Fused inference only: cand [(h-7)(w-7) x 8] table entries of the proposed cells (-1 where fewer
   are valid), conf [(h-7)(w-7)] probability of the best cell, logits (may be NULL) [.. x 32]. */
pt_status pt_table_proposal_infer(pt_table *t, pt_proposal *net, const float *d_a, int h, int w,
                                  int32_t *cand, float *conf, float *logits, void *stream);
/* pt_table_lookup with the network's proposals in place of the table candidate (and, unless
   configured otherwise, of k-coherence) for confident patches; same buffers and result layout. */
pt_status pt_table_lookup_learned(pt_table *t, pt_proposal *net, const float *a, int h, int w,
                                  double *ann_out, double *seconds);
pt_status pt_table_lookup_learned_device(pt_table *t, pt_proposal *net, const float *d_a, int h, int w,
                                         double *d_ann, void *stream);
/* Diagnostics: as pt_table_lookup_profile, with stage_ms[7] (the 7th stage is the network) and
   counters[6] (the 5th counts confident patches, the 6th their proposals). */
pt_status pt_table_lookup_learned_profile(pt_table *t, pt_proposal *net, const float *d_a, int h, int w,
                                          double *d_ann, void *stream, double *stage_ms, uint64_t *counters);

/* Diagnostics: the learned query with proposals supplied by the caller instead of the network
   (d_cand: P x PT_PROP_TOPK table entries, -1 = none; d_conf: P confidences; patches with
   d_conf >= threshold use them), e.g. the plain method's own converged matches, which bounds what
   any proposal network could gain.  Outputs as pt_table_lookup_learned_profile. */
pt_status pt_table_lookup_proposed_profile(pt_table *t, const float *d_a, int h, int w, const int32_t *d_cand,
                                           const float *d_conf, float threshold, int kcoh_confident, double *d_ann,
                                           void *stream, double *stage_ms, uint64_t *counters);

/* Diagnostics: number of breadth-first levels the last DT build ran. */
int pt_table_dt_levels(const pt_table *t);

/* ---- introspection (parity tests); shapes as in the reference members patchtable.h:1487-1549 ---- */

/* Grid dimension count; nslices receives PT_MAX_DIMS entries; *ncells the table size. */
int pt_table_shape(const pt_table *t, int *nslices, int64_t *ncells);
/* table (ncells int32, row-major over nslices, values XY_TO_INT(x+7, y+7)). */
pt_status pt_table_get_cells(const pt_table *t, int32_t *out);
/* Descriptor of every b patch, (h-7) x (w-7) x ndims, i.e. wh0 without its padding. */
pt_status pt_table_get_descriptor(const pt_table *t, float *out);
/* Partition of dimension dim: centers/lsizes/rsizes (nslices[dim] floats each),
   to_bin (16384 int32), mmr = {min_val, max_val, range} (patchtable.h:1131-1145). */
pt_status pt_table_get_partition(const pt_table *t, int dim, float *centers, float *lsizes,
                                 float *rsizes, int32_t *to_bin, float *mmr);
/* k-coherence set (patchtable.h:1520): (h-7) x (w-7) x kcoherence packed positions and dists. */
pt_status pt_table_get_kcoherence(const pt_table *t, int32_t *pos, float *dist);
/* Number of cells seeded by populate (table_add_count, patchtable.h:1539). */
int64_t pt_table_add_count(const pt_table *t);

/* Descriptor of an RGB image as the query computes it: (h-7) x (w-7) x ndims floats. */
pt_status pt_descriptor(const pt_params *p, const float *rgb, int h, int w, float *out);

/* Bound on every wait inside this library's device kernels (no reference counterpart; the
   reference has no device waits): a grid-barrier wait of the table build gives up after `polls`
   polls (about 0.1 us each), every block of the launch then leaves, and the call returns
   PT_TIMEOUT with the device still usable.  Process-wide; returns the previous bound.  A negative
   value restores the default, 2^24 polls (seconds).  0 makes any wait give up at once, which the
   tests use to exercise the error path. */
int64_t pt_set_spin_limit(int64_t polls);

/* Cap on the device memory this library holds at once (no reference counterpart): an allocation
   that would pass `bytes` fails as if the device were full and the call returns PT_OOM, leaving
   earlier tables intact.  Process-wide; returns the previous cap; a negative value removes the
   cap (the default).  Lets an application share the GPU with a fixed budget, and lets the tests
   drive the out-of-memory path without exhausting the device.  pt_device_bytes_in_use gives the
   bytes the library currently holds (the zero-allocation query's static array is not counted). */
int64_t pt_set_device_alloc_limit(int64_t bytes);
int64_t pt_device_bytes_in_use(void);

/* Host threads that widen the downloaded NNF to float64 in pt_table_lookup (no reference
   counterpart; the reference's lookup writes its float64 field directly, patchtable.h:3500): the
   GPU sends 8 bytes per patch (packed position, float distance) and these threads write the
   24-byte records into the caller's buffer while later rows are still computed.  n = 0 restores
   the default, min(8, hardware threads); n < 0 turns the host widening off (the GPU writes the
   float64 records and they are copied as they are: three times the bytes over PCIe, no host
   work).  Returns the previous count (-1 when widening was off).  A lookup already widening
   finishes with the threads it started with. */
int pt_set_host_threads(int n);

/* Specialised query kernels (no reference counterpart): the choose of a pass that has only the
   table step, and the pull of a schedule with one neighbour candidate, run as variants compiled
   without the other steps (fewer registers, more resident warps); their results are bit-identical
   to the general kernels'.  on = 0 runs the general kernels everywhere, which the tests use to
   compare the two; returns the previous setting (default 1).  Process-wide. */
int pt_set_lean_kernels(int on);
/* Bytes the last pt_table_lookup on this table copied host -> device and device -> host. */
pt_status pt_table_last_transfer(const pt_table *t, int64_t *h2d_bytes, int64_t *d2h_bytes);

/* Device kernel launches issued by this thread since the last reset (evidence counter). */
int64_t pt_kernel_launch_count(void);
void pt_kernel_launch_count_reset(void);

const char *pt_last_error(void);
const char *pt_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PATCHTABLE_B200_H */
