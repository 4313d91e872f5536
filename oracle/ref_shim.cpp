/* C entry points into the reference's OWN PatchTable implementation (oracle test
   infrastructure, never part of the product).

   This file is compiled together with the unmodified reference sources
   (patchtable/patchtable.cpp, solver/{array,util,timer,pfm}.cpp, headers patchtable/patchtable.h,
   gck.h, dt_downsample.h, patch_pca.h) and the third-party stand-ins in oracle/stubs/.  It only
   adds a C ABI so Python tests and the CPU baseline can drive the reference in memory:

     ptref_create   -> PatchTable<>(&params, b, allowed)       patchtable.h:4397-4424
     ptref_lookup   -> PatchTable<>::lookup(a, ann, ann_prev)  patchtable.h:4448-4468
     ptref_*        -> read-only views of the built table's members (table, wh0, partition,
                       k-coherence set) for parity checks, patchtable.h:1487-1549.

   Private members are reached by compiling the reference header with `private` defined as
   `public`; no reference source is changed. */
#include <algorithm>
#include <memory>
#include <unordered_map>
#include <unordered_set>
#include <vector>
#include <string>
#include <sstream>
#include <iostream>
#include <fstream>
#include <set>
#include <map>
#include <cstring>
#include <cstdint>
#include <cmath>
#include <functional>
#include <omp.h>
#define private public
#include "patchtable.h"
#undef private

namespace {

struct RefTable {
    PatchTableParams *p;
    PatchTable<float, float, int32_t> *t;
    int h, w;
};

template<int D>
PatchTableFixedN<float, float, D, int32_t> *fixed(RefTable *r);

#define PTREF_FIXED(D) \
    template<> PatchTableFixedN<float, float, D, int32_t> *fixed<D>(RefTable *r) { return r->t->p##D; }
PTREF_FIXED(3) PTREF_FIXED(4) PTREF_FIXED(5) PTREF_FIXED(6) PTREF_FIXED(7) PTREF_FIXED(8)
PTREF_FIXED(9) PTREF_FIXED(10) PTREF_FIXED(11) PTREF_FIXED(12) PTREF_FIXED(13) PTREF_FIXED(14) PTREF_FIXED(15)

/* Calls f(fixed table) for the table's compile-time dimension count. */
#define PTREF_DISPATCH(r, BODY) \
    switch ((r)->t->gck_dims) { \
        case 3: { auto T = fixed<3>(r); BODY; } break; \
        case 4: { auto T = fixed<4>(r); BODY; } break; \
        case 5: { auto T = fixed<5>(r); BODY; } break; \
        case 6: { auto T = fixed<6>(r); BODY; } break; \
        case 7: { auto T = fixed<7>(r); BODY; } break; \
        case 8: { auto T = fixed<8>(r); BODY; } break; \
        case 9: { auto T = fixed<9>(r); BODY; } break; \
        case 10: { auto T = fixed<10>(r); BODY; } break; \
        case 11: { auto T = fixed<11>(r); BODY; } break; \
        case 12: { auto T = fixed<12>(r); BODY; } break; \
        case 13: { auto T = fixed<13>(r); BODY; } break; \
        case 14: { auto T = fixed<14>(r); BODY; } break; \
        case 15: { auto T = fixed<15>(r); BODY; } break; \
        default: return -1; \
    }

}  // namespace

extern "C" {

void ptref_srand(unsigned seed) { srand(seed); }

int ptref_rand() { return rand(); }

void ptref_set_threads(int n) { omp_set_num_threads(n); }

/* Parses switches exactly like the reference CLI: PatchTableParams(argc, argv) with argv[0] the
   program name (patchtable.cpp:167-373, 384-387). */
void *ptref_params_new(const char *switches) {
    std::vector<std::string> toks;
    std::istringstream in(switches ? switches : "");
    std::string tok;
    while (in >> tok) toks.push_back(tok);
    std::vector<const char *> argv;
    argv.push_back("patchtable");
    for (auto &t : toks) argv.push_back(t.c_str());
    PatchTableParams *p = new PatchTableParams((int) argv.size(), argv.data());
    /* PatchTableParams does not parse these two; the CLI's match command reads -is_descriptor
       itself (patchtable_main.cpp:240-242) and analogy.cpp:853 sets descriptor_padded. */
    for (size_t i = 0; i + 1 < toks.size(); i++) {
        if (toks[i] == "-is_descriptor") p->is_descriptor = atoi(toks[i + 1].c_str()) != 0;
        if (toks[i] == "-descriptor_padded") p->descriptor_padded = atoi(toks[i + 1].c_str()) != 0;
    }
    return p;
}

void ptref_params_free(void *p) { delete (PatchTableParams *) p; }

/* Scalar parameter access by name, for tests that compare the parsed defaults and presets. */
int ptref_params_get(void *pv, const char *name, double *out) {
    PatchTableParams *p = (PatchTableParams *) pv;
    std::string n(name);
#define F(x) if (n == #x) { *out = (double) p->x; return 0; }
    F(limit) F(threads) F(ndims) F(nchroma) F(ntables) F(dt_algo) F(dt_iters) F(query_step)
    F(grid_ndims) F(prop_dist) F(do_prop) F(do_rs) F(spatial) F(patch_w) F(coherence_spatial)
    F(coherence_temporal) F(kcoherence) F(kcoherence_min_dist) F(kcoherence_iter)
    F(kcoherence_step) F(prop_iters) F(flann_reset_step) F(flann_build_step) F(query_iters) F(triangle_factor)
    F(populate_random) F(populate_nearest) F(partition_step) F(run_dt) F(do_table_lookup)
    F(is_descriptor) F(descriptor_padded) F(allowed_index) F(recalc_dist_temporal) F(sanitize_input) F(init_random)
    F(dim_algo) F(colorspace) F(convert_colorspace) F(flann_checks) F(flann_eps) F(table_ratio)
    F(verbose) F(randomize_dt) F(incoherence) F(lookup_algo) F(kcoherence_algo)
    F(pca_samples) F(pca_subtract_mean) F(pca_mean)
#undef F
    return -1;
}

int ptref_params_nslices(void *pv, int *out, int cap) {
    PatchTableParams *p = (PatchTableParams *) pv;
    int n = (int) p->nslices.size();
    for (int i = 0; i < n && i < cap; i++) out[i] = p->nslices[i];
    return n;
}

/* Builds the reference table on image b (h x w x 3 float RGB in [0,1], row-major).
   allowed (may be NULL) is (h-7) x (w-7) int32.  Returns NULL on failure. */
void *ptref_create(const char *switches, const float *b, int h, int w, int channels,
                   const int32_t *allowed, int verbose, double *seconds) {
    RefTable *r = new RefTable();
    r->p = (PatchTableParams *) ptref_params_new(switches);
    r->p->verbose = verbose;
    r->h = h; r->w = w;
    Array<float> B(h, w, channels);
    memcpy(B.data, b, sizeof(float) * (size_t) h * w * channels);
    Array<int32_t> *A = NULL;
    if (allowed) {
        A = new Array<int32_t>(h - r->p->patch_w + 1, w - r->p->patch_w + 1);
        memcpy(A->data, allowed, sizeof(int32_t) * (size_t) A->nelems);
    }
    double T0 = wall_time();
    r->t = new PatchTable<float, float, int32_t>(r->p, B, A);
    if (seconds) *seconds = wall_time() - T0;
    delete A;
    return r;
}

void ptref_free(void *rv) {
    RefTable *r = (RefTable *) rv;
    delete r->t;
    delete r->p;
    delete r;
}

/* Runs PatchTable::lookup; ann_out receives (ha-7) x (wa-7) x 3 doubles.  ann_prev may be NULL. */
double ptref_lookup(void *rv, const float *a, int h, int w, int channels, double *ann_out,
                    const double *ann_prev) {
    RefTable *r = (RefTable *) rv;
    Array<float> A(h, w, channels);
    memcpy(A.data, a, sizeof(float) * (size_t) h * w * channels);
    Array<double> ann;
    Array<double> *prev = NULL;
    int pw = r->p->patch_w;
    int eh = h - pw + 1, ew = w - pw + 1;
    if (r->p->is_descriptor) {                         /* get_padded_descriptor, patchtable.h:2498-2507 */
        eh = r->p->descriptor_padded ? h - 2 * (pw - 1) : h;
        ew = r->p->descriptor_padded ? w - 2 * (pw - 1) : w;
    }
    if (ann_prev) {
        prev = new Array<double>(eh, ew, 3);
        memcpy(prev->data, ann_prev, sizeof(double) * (size_t) prev->nelems);
    }
    double s = r->t->lookup(A, ann, prev);
    memcpy(ann_out, ann.data, sizeof(double) * (size_t) ann.nelems);
    delete prev;
    return s;
}

int ptref_ndims(void *rv) { return ((RefTable *) rv)->t->gck_dims; }

/* Table shape: returns number of grid dims, fills nslices (cap entries). */
int ptref_table_shape(void *rv, int *nslices, int cap) {
    RefTable *r = (RefTable *) rv;
    int n = 0;
    PTREF_DISPATCH(r, { n = (int) T->table.sizes.size(); for (int i = 0; i < n && i < cap; i++) nslices[i] = T->table.sizes[i]; });
    return n;
}

int ptref_table_add_count(void *rv) {
    RefTable *r = (RefTable *) rv;
    int n = 0;
    PTREF_DISPATCH(r, { n = T->table_add_count; });
    return n;
}

int ptref_get_table(void *rv, int32_t *out) {
    RefTable *r = (RefTable *) rv;
    PTREF_DISPATCH(r, { memcpy(out, T->table.data, sizeof(int32_t) * (size_t) T->table.nelems); });
    return 0;
}

/* wh0 is (h+7) x (w+7) x ndims. */
int ptref_get_wh0(void *rv, float *out) {
    RefTable *r = (RefTable *) rv;
    PTREF_DISPATCH(r, { memcpy(out, T->wh0.data, sizeof(float) * (size_t) T->wh0.nelems); });
    return 0;
}

/* Partition of dimension dim: centers/lsizes/rsizes (nslices each), to_bin (16384),
   mmr = {min_val, max_val, range}. */
int ptref_get_partition(void *rv, int dim, float *centers, float *lsizes, float *rsizes,
                        int32_t *to_bin, float *mmr) {
    RefTable *r = (RefTable *) rv;
    PTREF_DISPATCH(r, {
        auto *L = T->part->L[dim];
        for (size_t i = 0; i < L->centers.size(); i++) { centers[i] = L->centers[i]; lsizes[i] = L->lsizes[i]; rsizes[i] = L->rsizes[i]; }
        for (size_t i = 0; i < L->to_bin.size(); i++) to_bin[i] = L->to_bin[i];
        mmr[0] = L->min_val; mmr[1] = L->max_val; mmr[2] = L->range;
    });
    return 0;
}

/* k-coherence set: beh x bew x k of (packed position, float distance). */
int ptref_get_kcoherence(void *rv, int32_t *pos, float *dist) {
    RefTable *r = (RefTable *) rv;
    PTREF_DISPATCH(r, {
        size_t n = (size_t) T->kcoherence_set.nelems;
        for (size_t i = 0; i < n; i++) { pos[i] = T->kcoherence_set.data[i].first; dist[i] = T->kcoherence_set.data[i].second; }
    });
    return 0;
}

/* gck() on an h x w x 3 image: out is (h+7) x (w+7) x (n + 2*nchroma). gck.h:1956 */
int ptref_gck(const float *in, int h, int w, int n, int nchroma, float *out) {
    Array<float> I(h, w, 3);
    memcpy(I.data, in, sizeof(float) * (size_t) h * w * 3);
    Array<float> O;
    gck<float, float>(I, O, n, nchroma, 8);
    memcpy(out, O.data, sizeof(float) * (size_t) O.nelems);
    return 0;
}

/* Array::rgb2yuv, solver/array.h:1116-1134. */
int ptref_rgb2yuv(const float *in, int h, int w, float *out) {
    Array<float> I(h, w, 3), O;
    memcpy(I.data, in, sizeof(float) * (size_t) h * w * 3);
    I.rgb2yuv(O);
    memcpy(out, O.data, sizeof(float) * (size_t) h * w * 3);
    return 0;
}

/* scale_slices_to_limit, patchtable.cpp:611-642. */
int ptref_scale_slices(const int *in, int n, double limit, int *out) {
    std::vector<int> v(in, in + n);
    std::vector<int> r = scale_slices_to_limit(v, limit);
    for (int i = 0; i < n; i++) out[i] = r[i];
    return 0;
}

}  // extern "C"
