/* CPU restatement of the reference PatchTable build + query path.

   TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
   leg load this library, and only as the checker.  It restates, step by step and in the same
   floating-point order, the reference functions cited beside each routine (paths are relative
   to the reference project root).  Its results are pinned against the reference's own sources
   compiled in oracle/_ref (tests/test_oracle_vs_ref.py).

   Deliberate stand-in: the k-coherence nearest-neighbour search uses the exact search of
   oracle/knn_exact.h in place of FLANN (FLANN is neither vendored nor version-pinned).

   All arithmetic is float unless the reference uses double; the file is compiled with
   -ffp-contract=off so no multiply-add is fused. */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <vector>
#include "knn_exact.h"
#include "pca_jacobi.h"
#include "gck_steps.h"

using std::vector;

namespace {

const int PW = 8;                 /* patch width: TABLE_PATCH_W, patchtable.h:48 */
const int NMAP = 16384;           /* PATCH_PARTITION_NMAP, patchtable.h:216 */
const int UNUSED = (1 << 30) - 1; /* TABLE_UNUSED, patchtable.h:109-112 */
const double DIST_INF = 100000;   /* DIST_INFINITY, patchtable.h:173 */

inline int xy_to_int(int x, int y) { return x | (y << 16); }   /* patchtable.h:163-165 */
inline int int_to_x(int v) { return v & 65535; }
inline int int_to_y(int v) { return v >> 16; }

}  // namespace

extern "C" {

/* The subset of PatchTableParams (patchtable_params.h:23-161) that the build/query path reads. */
typedef struct {
    int ndims, nchroma, grid_ndims;
    double limit;
    int nslices[16], n_nslices;       /* explicit -nslices, n_nslices == 0 means automatic */
    int partition_step;
    int populate_random;
    int run_dt, dt_algo, dt_iters;    /* dt_algo: 1 prop, 2 brute, 4 downsample, 5 hybrid, 6 euclidean */
    int kcoherence, kcoherence_min_dist, kcoherence_step, kcoherence_iter;
    int flann_reset_step, flann_build_step;
    double triangle_factor;
    int prop_iters, query_step, do_prop, prop_dist;
    double coherence_spatial, coherence_temporal;
    int do_table_lookup, do_rs, spatial;
    int allowed_index;
    int recalc_dist_temporal, sanitize_input, init_random;
    int convert_colorspace;
    int is_descriptor, descriptor_padded;   /* descriptor mode: b and a are ndims-channel images */
    int ntables;                            /* further tables at limit / table_ratio^i */
    double table_ratio;
    int dim_algo, pca_samples, pca_subtract_mean, pca_mean;   /* dim_algo 1: PCA descriptor */
    int colorspace;                         /* 0 YUV, 1 Lab (when convert_colorspace) */
} orc_params;

}

namespace {

/* ------------------------------------------------------------------------------------------
   Colour conversion: ARRAY_RGB2YUV, solver/array.h:1116-1127.  The constants are double, the
   pixel is float, the sum is evaluated left to right in double and stored as float.
   ------------------------------------------------------------------------------------------ */
void rgb2yuv(const float *in, int n, float *out) {
    for (int i = 0; i < n; i++) {
        float R = in[3 * i], G = in[3 * i + 1], B = in[3 * i + 2];
        out[3 * i + 0] = (float) (0.299 * R + 0.587 * G + 0.114 * B);
        out[3 * i + 1] = (float) (-0.14713 * R + -0.28886 * G + 0.436 * B);
        out[3 * i + 2] = (float) (0.615 * R + -0.51499 * G + -0.10001 * B);
    }
}

/* ------------------------------------------------------------------------------------------
   Colour conversion -colorspace lab: Array::rgb2lab = rgb2xyz then xyz2lab (solver/array.h:
   1213-1292, D50 white, Bruce Lindbloom's formulas) with the powers read from PowTable<float,
   1024> (solver/array.h:221-237): entry i holds (float) pow((i + 0.5) / 1024, p), p stored as a
   float, and a value v reads entry int(v * 1024.0f) clamped to the table.  Constants are double,
   pixels float, as in the reference.
   ------------------------------------------------------------------------------------------ */
struct PowTab {
    float t[1024];
    explicit PowTab(float p) {
        for (int i = 0; i < 1024; i++) t[i] = (float) pow((i + 0.5) / 1024 * (double) 1.0f, (double) p);
    }
    float operator()(float v) const {
        int i = (int) (v * 1024.0f);
        if (i < 0) i = 0; else if (i >= 1024) i = 1023;
        return t[i];
    }
};

void rgb2lab(const float *in, int n, float *out) {
    static const PowTab p24(2.4f), p13((float) (1.0 / 3.0));
    for (int k = 0; k < n; k++) {
        float c[3];
        for (int j = 0; j < 3; j++) {
            float v = in[3 * k + j];
            c[j] = (v <= 0.04045) ? (float) (v / 12.92) : p24((float) ((v + 0.055) / 1.055));
        }
        float X = (float) (0.4360747 * c[0] + 0.3850649 * c[1] + 0.1430804 * c[2]);
        float Y = (float) (0.2225045 * c[0] + 0.7168786 * c[1] + 0.0606169 * c[2]);
        float Z = (float) (0.0139322 * c[0] + 0.0971045 * c[1] + 0.7141733 * c[2]);
        float xr = (float) (X / 0.9642), yr = (float) (Y / 1.0000), zr = (float) (Z / 0.8249);
        float fx = (xr > 0.008856) ? p13(xr) : (float) ((903.3 * xr + 16) / 116);
        float fy = (yr > 0.008856) ? p13(yr) : (float) ((903.3 * yr + 16) / 116);
        float fz = (zr > 0.008856) ? p13(zr) : (float) ((903.3 * zr + 16) / 116);
        out[3 * k + 0] = 116 * fy - 16;
        out[3 * k + 1] = 500 * (fx - fy);
        out[3 * k + 2] = 200 * (fy - fz);
    }
}

/* The colour conversion of get_padded_descriptor (patchtable.h:2510-2522). */
void convert_color(const orc_params &p, const float *in, int n, float *out) {
    if (!p.convert_colorspace) memcpy(out, in, sizeof(float) * 3 * (size_t) n);
    else if (p.colorspace == 1) rgb2lab(in, n, out);
    else rgb2yuv(in, n, out);
}

/* ------------------------------------------------------------------------------------------
   Gray-code kernels: gck_8<float,float,n,nchroma>, patchtable/gck.h:29-1950 (generated by
   gck.py:84-517).  Output is (h+7) x (w+7) x (n + 2*nchroma) "full" convolution.
   ------------------------------------------------------------------------------------------ */
void gck8(const float *in, int h, int w, int n, int nchroma, float *out) {
    const int rpad = PW / 2, lpad = rpad - 1, lread = rpad, rread = lpad, pad = lpad + rpad;
    const int OH = h + pad, OW = w + pad, OC = n + nchroma * 2;
    vector<float> temp((size_t) OH * OW * 3);
    auto in_zero = [&](int y, int x, int c) -> float {
        if (y < 0 || y >= h || x < 0 || x >= w) return 0.0f;
        return in[((size_t) y * w + x) * 3 + c];
    };
    auto T = [&](int y, int x, int c) -> float & { return temp[((size_t) y * OW + x) * 3 + c]; };
    auto T_zero = [&](int y, int x, int c) -> float {
        if (y < 0 || y >= OH || x < 0 || x >= OW) return 0.0f;
        return temp[((size_t) y * OW + x) * 3 + c];
    };
    auto O = [&](int y, int x, int c) -> float & { return out[((size_t) y * OW + x) * OC + c]; };
    auto O_zero = [&](int y, int x, int c) -> float {
        if (y < 0 || y >= OH || x < 0 || x >= OW) return 0.0f;
        return out[((size_t) y * OW + x) * OC + c];
    };
    /* Horizontal running box sum (gck.h:52-152): temp(y,x) = temp(y,x-1) + in(y-3, x) - in(y-3, x-8). */
    for (int y = 0; y < OH; y++) {
        int ysrc = y - lpad;
        for (int c = 0; c < 3; c++) T(y, 0, c) = in_zero(ysrc, 0, c);
        for (int x = 1; x < OW; x++) {
            int xsrc = x - lpad;
            for (int c = 0; c < 3; c++)
                T(y, x, c) = T(y, x - 1, c) + in_zero(ysrc, xsrc + rread, c) - in_zero(ysrc, xsrc - lread - 1, c);
        }
    }
    /* Vertical running box sum (gck.h:160-205).  The reference always writes three channels here;
       with nchroma 0 the first kernel owns one, the extra two land in slots the recurrence below
       overwrites before reading (or, with fewer than three output channels, past the array's
       end), so only the first kernel's own channels are written. */
    const int nc0 = nchroma > 0 ? 3 : 1;
    for (int x = 0; x < OW; x++)
        for (int c = 0; c < nc0; c++) O(0, x, c) = T(rread, x, c);
    for (int y = 1; y < OH; y++)
        for (int x = 0; x < OW; x++)
            for (int c = 0; c < nc0; c++)
                O(y, x, c) = O(y - 1, x, c) + T_zero(y + rread, x, c) - T_zero(y - lread - 1, x, c);
    /* Snake-order recurrences for kernels 1..n-1 (gck.h:215-1950, gck.py:364-420):
       out_i(p) = s*out_i(p-d) + out_{i-1}(p) + s*out_{i-1}(p-d), evaluated left to right. */
    auto c0 = [&](int k) { return k < nchroma ? k * 3 : nchroma * 3 + (k - nchroma); };
    for (int y = 0; y < OH; y++) {
        for (int x = 0; x < OW; x++) {
            for (int i = 1; i < n; i++) {
                int horiz = ORC_GCK_STEPS[i - 1][0], d = ORC_GCK_STEPS[i - 1][1];
                float s = (float) ORC_GCK_STEPS[i - 1][2];
                int yp = horiz ? y : y - d, xp = horiz ? x - d : x;
                int nc = i < nchroma ? 3 : 1;
                for (int c = 0; c < nc; c++) {
                    float a = s * O_zero(yp, xp, c0(i) + c);
                    float b = O(y, x, c0(i - 1) + c);
                    float e = s * O_zero(yp, xp, c0(i - 1) + c);
                    O(y, x, c0(i) + c) = a + b + e;
                }
            }
        }
    }
}

/* ------------------------------------------------------------------------------------------
   Exact patch distance: patch_dist_exact<float,8,3>, patchtable.h:330-373 (SSE path).  Four
   lane sums over 8 rows x 6 chunks of 4 floats, lanes added 0+1+2+3 at the end.
   ------------------------------------------------------------------------------------------ */
float patch_dist_exact(const float *a, int a_w, int ax, int ay, const float *b, int b_w, int bx, int by) {
    float lane[4] = {0, 0, 0, 0};
    for (int dy = 0; dy < PW; dy++) {
        const float *arow = a + ((size_t) (ay + dy) * a_w + ax) * 3;
        const float *brow = b + ((size_t) (by + dy) * b_w + bx) * 3;
        float d[6][4];
        for (int nn = 0; nn < 6; nn++)
            for (int q = 0; q < 4; q++) {
                float t = arow[nn * 4 + q] - brow[nn * 4 + q];
                d[nn][q] = t * t;
            }
        for (int q = 0; q < 4; q++)
            lane[q] = lane[q] + d[0][q] + d[1][q] + d[2][q] + d[3][q] + d[4][q] + d[5][q];
    }
    return lane[0] + lane[1] + lane[2] + lane[3];
}

/* ------------------------------------------------------------------------------------------
   One-dimensional partition: PatchPartition1D, patchtable.h:1131-1326 (non-regular grid,
   randomize = false).
   ------------------------------------------------------------------------------------------ */
struct Partition1D {
    vector<int> to_bin;
    vector<float> centers, lsizes, rsizes;
    float min_val, max_val, range;
    int nslices;

    /* get_bin, patchtable.h:1298-1325. */
    int get_bin(float v) const {
        int idx = (int) ((v - min_val) * (float) (NMAP - 1) / range);
        if (idx < 0) idx = 0;
        else if (idx >= NMAP) idx = NMAP - 1;
        return to_bin[idx];
    }
};

/* ------------------------------------------------------------------------------------------
   Descriptor-mode distance: patch_dist_approx<float, TABLE_NCHANNELS>, patchtable.h:376-437
   (TABLE_SSE).  Four lanes from the first four floats (also with 3 dimensions, where the fourth
   float is whatever follows in memory); with exactly 8, 12 or 16 dimensions further blocks of
   four are added lane-wise and the lanes summed 0+1+2+3, otherwise the lanes are summed first
   and the remaining dimensions added one by one.
   ------------------------------------------------------------------------------------------ */
float patch_dist_approx(const float *avec, const float *bvec, int nd) {
    float l[4];
    for (int q = 0; q < 4; q++) { float d = avec[q] - bvec[q]; l[q] = d * d; }
    if (nd == 8 || nd == 12 || nd == 16 || nd == 20) {
        for (int n = 1; n < nd / 4; n++)
            for (int q = 0; q < 4; q++) { float d = avec[4 * n + q] - bvec[4 * n + q]; l[q] = l[q] + d * d; }
        return l[0] + l[1] + l[2] + l[3];
    }
    float s = l[0] + l[1] + l[2] + l[3];
    for (int i = 4; i < nd; i++) { float d = avec[i] - bvec[i]; s += d * d; }
    return s;
}

/* get_padded_descriptor in descriptor mode, patchtable.h:2498-2507: an unpadded H x W x nd input
   goes to offset (7, 7) of a zeroed (H+14) x (W+14) x nd image (copy_rect); a padded input is that
   image already.  vh x vw is the virtual image whose patches are the input's pixels
   (TABLE_IMG_HEIGHT / TABLE_IMG_WIDTH, patchtable.h:2489-2490). */
void padded_input(const orc_params &p, const float *in, int H, int W, vector<float> &wh, int &vh, int &vw) {
    const int nd = p.ndims;
    if (p.descriptor_padded) {
        wh.assign(in, in + (size_t) H * W * nd);
        vh = H - 7; vw = W - 7;
        return;
    }
    const int WH = H + 14, WW = W + 14;
    wh.assign((size_t) WH * WW * nd, 0.0f);
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++)
            for (int c = 0; c < nd; c++) wh[((size_t) (y + 7) * WW + (x + 7)) * nd + c] = in[((size_t) y * W + x) * nd + c];
    vh = H + 7; vw = W + 7;
}

/* -dim_algo pca basis (see pca_fit). */
const int PCA_D = PW * PW * 3;

struct Pca {
    vector<float> mean;     /* PCA_D */
    vector<float> basis;    /* ndims x PCA_D */
};

struct Table {
    orc_params p;
    int h, w;                   /* b size */
    int nd;                     /* descriptor dims */
    int gnd;                    /* grid dims */
    vector<float> b0;           /* h x w x 3 RGB */
    vector<float> wh0;          /* (h+7) x (w+7) x nd */
    vector<int> allowed;        /* (h-7) x (w-7), empty if none */
    vector<int> nslices;
    vector<int64_t> stride;
    int64_t ncells = 0;
    vector<int32_t> table;
    vector<Partition1D> part;
    int table_add_count = 0;
    int kc_max_knn = 0;         /* longest neighbour list the k-coherence search asked for */
    int kc_h = 0, kc_w = 0;
    vector<int32_t> kc_pos;     /* kc_h x kc_w x kcoherence */
    vector<float> kc_dist;
    vector<float> min_val, max_val, range;
    /* Scratch reused across lookups, like lookup_buffer/lookup_wh (patchtable.h:1507-1509). */
    vector<float> lookup_wh;
    /* ntables > 1: the further tables (tables, patchtable.h:1491) */
    vector<std::unique_ptr<Table>> subs;
    /* -dim_algo pca: the basis fitted on b (PatchTableFixedN::pca) */
    Pca pca;

    int WW() const { return w + 7; }
    float whv(int y, int x, int i) const { return wh0[((size_t) y * WW() + x) * nd + i]; }
    bool is_allowed(int py, int px) const {
        return allowed.empty() || allowed[(size_t) py * (w - 7) + px] == p.allowed_index;
    }
};

/* get_padded_descriptor for RGB input (patchtable.h:2492-2546): YUV then gck. */
void padded_descriptor(const orc_params &p, const float *rgb, int h, int w, vector<float> &wh) {
    vector<float> yuv((size_t) h * w * 3);
    convert_color(p, rgb, h * w, yuv.data());
    wh.assign((size_t) (h + 7) * (w + 7) * p.ndims, 0.0f);
    gck8(yuv.data(), h, w, p.ndims - p.nchroma * 2, p.nchroma, wh.data());
}

/* ------------------------------------------------------------------------------------------
   -dim_algo pca, patch_pca.h.  cv::PCA(DATA_AS_ROW, maxComponents = ndims) is restated in
   pca_jacobi.h (sample mean or zero mean, covariance, cyclic Jacobi eigenvectors); the same
   header stands in for OpenCV in the reference build, so the reference's own sampling and
   projection (patch_pca.h:14-113) run there and pin this restatement by digest.
   ------------------------------------------------------------------------------------------ */
/* The 192-vector the reference builds for the patch at (ax, ay) (extract_patches and
   apply_patch_pca, patch_pca.h:30-37, 87-96): for row dy, column dx and channel c it reads
   arow[dx] [c], where arow points at float 0 of pixel (ax, ay + dy) of the interleaved image, so
   entry (dy, dx, c) is float dx + c of that row -- floats 0..9, i.e. the first three pixels and a
   third, not pixel dx.  Restated as written, since the descriptor values depend on it. */
inline void pca_patch_vector(const float *img, int w, int ax, int ay, float *v) {
    int k = 0;
    for (int dy = 0; dy < PW; dy++) {
        const float *arow = img + ((size_t) (ay + dy) * w + ax) * 3;
        for (int dx = 0; dx < PW; dx++)
            for (int c = 0; c < 3; c++) v[k++] = arow[dx + c];
    }
}

/* extract_patches + get_patch_pca, patch_pca.h:14-52, on the colour-converted image: sample i is
   the patch at (rand() % (w-7), rand() % (h-7)). */
void pca_fit(const orc_params &p, const float *img, int h, int w, Pca &out) {
    const int n = p.pca_samples, aew = w - PW + 1, aeh = h - PW + 1;
    vector<float> X((size_t) n * PCA_D);
    for (int i = 0; i < n; i++) {
        int ax = rand() % aew;
        int ay = rand() % aeh;
        pca_patch_vector(img, w, ax, ay, &X[(size_t) i * PCA_D]);
    }
    const vector<float> zero(PCA_D, 0.0f);
    pt_pca_jacobi_fit(X.data(), n, PCA_D, !p.pca_subtract_mean, zero.data(), p.ndims, out.mean, out.basis);
}

/* apply_patch_pca, patch_pca.h:54-110 (pca_mean off): channel k of the patch at (x, y) goes to
   wh(y+7, x+7, k); the projection sums (v_j - mean_j) * basis_kj in j order, in float. */
void pca_apply(const orc_params &p, const Pca &pca, const float *img, int h, int w, vector<float> &wh) {
    const int nd = p.ndims, WW = w + PW - 1;
    wh.assign((size_t) (h + PW - 1) * WW * nd, 0.0f);
    vector<float> v(PCA_D);
    for (int ay = 0; ay + PW <= h; ay++)
        for (int ax = 0; ax + PW <= w; ax++) {
            pca_patch_vector(img, w, ax, ay, v.data());
            pt_pca_project(v.data(), PCA_D, pca.mean.data(), pca.basis.data(), nd,
                           &wh[((size_t) (ay + PW - 1) * WW + ax + PW - 1) * nd]);
        }
}

/* scale_slices_to_limit, patchtable.cpp:611-642 (product and multiply: solver/util.cpp:186-205). */
vector<int> scale_slices_to_limit(vector<int> nslices, double limit) {
    auto product = [](const vector<int> &L) { double a = 1.0; for (int v : L) a *= v; return a; };
    if (limit > 0) {
        vector<int> nslices0(nslices);
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

void build_kcoherence(Table &t);
void dt_prop(Table &t);
void dt_prop1(Table &t);
void dt_unmask(Table &t);
void dt_downsample(Table &t);
void dt_euclidean(Table &t);
void dt_brute(Table &t);

/* PatchTableFixedN constructor, patchtable.h:2584-3373, default path (no product quantisation,
   no k-means, TABLE_POPULATE_FAST).  With TABLE_POPULATE_FAST (patchtable.h:37) populate never
   reaches add_patch (patchtable.h:3127-3159), so populate_nearest has no effect and randomize_dt
   collects no adjacency: do_after_dt (patchtable.h:1831-1866) finds every set empty and changes
   no cell.  Neither switch is read here. */
Table *build(const orc_params &p, const float *b, int h, int w, const int32_t *allowed, const float *wh0_in) {
    const int h_in = h, w_in = w;
    Table *t = new Table();
    t->p = p;
    t->nd = p.ndims;
    t->gnd = p.grid_ndims < 0 ? p.ndims : p.grid_ndims;
    if (p.is_descriptor) {
        /* b is h x w x ndims descriptors (the caller sets ndims = channels, nchroma = 0 as the
           reference's constructor does, patchtable.h:4398-4401); b0 is unused. */
        int vh, vw;
        padded_input(p, b, h, w, t->wh0, vh, vw);
        h = vh; w = vw;
    } else {
        t->b0.assign(b, b + (size_t) h * w * 3);
        if (p.dim_algo == 1) {                           /* reduce_dim, patchtable.h:1709-1713 */
            vector<float> img((size_t) h * w * 3);
            convert_color(p, b, h * w, img.data());
            pca_fit(p, img.data(), h, w, t->pca);
            if (!wh0_in) pca_apply(p, t->pca, img.data(), h, w, t->wh0);
        } else if (!wh0_in) {
            padded_descriptor(p, b, h, w, t->wh0);
        }
        if (wh0_in) t->wh0.assign(wh0_in, wh0_in + (size_t) (h + 7) * (w + 7) * p.ndims);
    }
    t->h = h; t->w = w;
    if (allowed) t->allowed.assign(allowed, allowed + (size_t) (h - 7) * (w - 7));
    const int xmin = 7, ymin = 7, xmax = w, ymax = h;   /* gck_xmin/xmax, patchtable_params.h:14-17 */

    if (p.kcoherence) build_kcoherence(*t);

    /* set_min_max, patchtable.h:1758-1778. */
    int G = t->gnd;
    t->min_val.assign(G, 1e20f);
    t->max_val.assign(G, -1e20f);
    for (int y = ymin; y < ymax; y++)
        for (int x = xmin; x < xmax; x++) {
            if (!t->is_allowed(y - ymin, x - xmin)) continue;
            for (int i = 0; i < G; i++) {
                float v = t->whv(y, x, i);
                t->min_val[i] = std::min(t->min_val[i], v);
                t->max_val[i] = std::max(t->max_val[i], v);
            }
        }
    t->range.resize(G);
    for (int i = 0; i < G; i++) t->range[i] = t->max_val[i] - t->min_val[i];

    /* set_default_nslices, patchtable.h:1780-1810 (TABLE_SIZE_STDDEV == 0). */
    vector<int> ns(G);
    if (p.n_nslices == 0) {
        float max_range = t->range[0];
        for (int i = 1; i < G; i++) if (t->range[i] > max_range) max_range = t->range[i];
        double scale = 200.0 / max_range;
        for (int i = 0; i < G; i++) ns[i] = (int) (t->range[i] * scale);
    } else {
        for (int i = 0; i < G; i++) ns[i] = p.nslices[i];
    }
    t->nslices = scale_slices_to_limit(ns, p.limit);

    /* PatchPartition, patchtable.h:1355-1396: patches sampled every partition_step. */
    vector<int> patches;
    for (int y = ymin; y < ymax; y += p.partition_step)
        for (int x = xmin; x < xmax; x += p.partition_step)
            if (t->is_allowed(y - ymin, x - xmin)) patches.push_back(xy_to_int(x, y));
    t->part.resize(G);
    for (int c = 0; c < G; c++) {
        Partition1D &P = t->part[c];
        int ncs = t->nslices[c];
        P.nslices = ncs;
        /* Sorting by channel value; only values at quantile positions are read, so the
           (unstable) order of equal values does not matter (patchtable.h:1172-1176). */
        vector<float> vals(patches.size());
        for (size_t i = 0; i < patches.size(); i++) vals[i] = t->whv(int_to_y(patches[i]), int_to_x(patches[i]), c);
        std::sort(vals.begin(), vals.end());
        P.min_val = t->min_val[c];
        P.max_val = t->max_val[c];
        P.range = P.max_val - P.min_val;
        P.centers.resize(ncs); P.lsizes.resize(ncs); P.rsizes.resize(ncs);
        int N = (int) vals.size();
        for (int i = 0; i < ncs; i++) {            /* patchtable.h:1193-1201 */
            int idx1 = (N - 1) * i / ncs;
            int idx2 = (N - 1) * (i + 1) / ncs;
            float cell_max = vals[idx2], cell_min = vals[idx1];
            P.centers[i] = (cell_min + cell_max) / 2;
        }
        for (int i = 0; i < ncs; i++) {            /* patchtable.h:1203-1215 */
            float prev_center = (i - 1 >= 0) ? P.centers[i - 1] : P.min_val;
            float next_center = (i + 1 < ncs) ? P.centers[i + 1] : P.max_val;
            P.lsizes[i] = P.centers[i] - prev_center;
            if (i - 1 >= 0) P.lsizes[i] /= 2;
            P.rsizes[i] = next_center - P.centers[i];
            if (i + 1 < ncs) P.rsizes[i] /= 2;
        }
        P.to_bin.resize(NMAP);                      /* patchtable.h:1219-1256 */
        int icenter = 0;
        for (int i = 0; i < NMAP; i++) {
            double coord = P.min_val + (i + 0.5) * P.range / NMAP;
            while (coord > P.centers[icenter]) {
                if (icenter + 1 < ncs) icenter++;
                else break;
            }
            int prev_c = icenter - 1;
            if (prev_c < 0) prev_c = 0;
            int next_c = icenter;
            if (next_c == 0) next_c++;
            if (ncs == 1) next_c = prev_c = 0;
            double mid = (P.centers[prev_c] + P.centers[next_c]) / 2.0;
            P.to_bin[i] = (coord < mid) ? prev_c : next_c;
        }
    }

    /* Table shape and strides: Array<itype>::resize(nslices), row-major (solver/array.h:262-294). */
    t->stride.assign(G, 1);
    t->ncells = 1;
    for (int i = G - 1; i >= 0; i--) { t->stride[i] = t->ncells; t->ncells *= t->nslices[i]; }
    t->table.assign((size_t) t->ncells, UNUSED);

    /* Populate, TABLE_POPULATE_INNER_BLOCK with populate_random (patchtable.h:3121-3159):
       std::random_shuffle of the allowed patch list, first visitor of a cell wins. */
    vector<int> order;
    for (int y = ymin; y < ymax; y++)
        for (int x = xmin; x < xmax; x++)
            if (t->is_allowed(y - ymin, x - xmin)) order.push_back(xy_to_int(x, y));
    if (p.populate_random) {
        /* libstdc++ random_shuffle(first, last): for i in 1..n-1, j = rand() % (i + 1), swap. */
        for (size_t i = 1; i < order.size(); i++) {
            size_t j = (size_t) (rand() % (int) (i + 1));
            if (i != j) std::swap(order[i], order[j]);
        }
    }
    for (int pos : order) {
        int x = int_to_x(pos), y = int_to_y(pos);
        int64_t cell = 0;
        for (int i = 0; i < G; i++) cell += (int64_t) t->part[i].get_bin(t->whv(y, x, i)) * t->stride[i];
        if (t->table[cell] == UNUSED) { t->table[cell] = xy_to_int(x, y); t->table_add_count++; }
    }

    /* Distance transform (patchtable.h:3254-3298). */
    bool zeros_filled = false;
    if (p.run_dt) {
        if (p.dt_algo == 1) { dt_prop(*t); zeros_filled = (p.dt_iters <= 0); }
        else if (p.dt_algo == 2) { dt_brute(*t); zeros_filled = true; }
        else if (p.dt_algo == 4) { dt_downsample(*t); zeros_filled = true; }
        else if (p.dt_algo == 5) { dt_prop1(*t); dt_downsample(*t); dt_unmask(*t); zeros_filled = true; }
        else if (p.dt_algo == 6) { dt_euclidean(*t); zeros_filled = true; }
        else { fprintf(stderr, "oracle: dt_algo %d is not restated\n", p.dt_algo); abort(); }
    }
    if (!zeros_filled) {                            /* fill_zeros, patchtable.h:2063-2079 */
        int vfill = xy_to_int(PW - 1, PW - 1);
        if (!t->allowed.empty()) {
            bool found = false;
            for (int y = ymin; y < ymax && !found; y++)
                for (int x = xmin; x < xmax; x++)
                    if (t->is_allowed(y - ymin, x - xmin)) { vfill = xy_to_int(x, y); found = true; break; }
        }
        for (auto &v : t->table) if (v == UNUSED) v = vfill;
    }
    /* Further tables, patchtable.h:3359-3371: the same b at limit int(limit / table_ratio^i),
       without k-coherence, each drawing its own populate order from rand() in turn. */
    for (int i = 1; i < p.ntables; i++) {
        orc_params pc = p;
        pc.limit = (double) (int) (pc.limit * (1.0 / pow(p.table_ratio, i)));
        pc.kcoherence = 0;
        pc.ntables = 1;
        t->subs.emplace_back(build(pc, b, h_in, w_in, allowed, nullptr));
    }
    return t;
}

/* do_dt_prop, patchtable.h:2081-2165, with PropEdge labels (patchtable.h:1435-1468). */
void dt_prop(Table &t) {
    int G = t.gnd;
    struct Elem { int64_t grid_index; int32_t table_value; uint8_t label; };
    vector<Elem> cur, nxt;
    for (int64_t j = 0; j < t.ncells; j++)
        if (t.table[j] != UNUSED) cur.push_back(Elem{j, t.table[j], 0});
    int nlabels = 1 + G * 2;
    struct Edge { int dim, dir, label; };
    auto mk = [&](int dim, int dir) { return Edge{dim, dir, 2 * dim + 1 + (dir + 1) / 2}; };
    vector<vector<Edge>> next_label;
    vector<Edge> next0;
    for (int i = 0; i < G; i++) { next0.push_back(mk(i, -1)); next0.push_back(mk(i, 1)); }
    next_label.push_back(next0);
    for (int i = 0; i < G; i++)
        for (int dir = -1; dir <= 1; dir += 2) {
            vector<Edge> nx;
            nx.push_back(mk(i, dir));
            for (int j = i + 1; j < G; j++) { nx.push_back(mk(j, -1)); nx.push_back(mk(j, 1)); }
            next_label.push_back(nx);
        }
    (void) nlabels;
    for (int iter = 0;; iter++) {
        if (t.p.dt_iters > 0 && iter > t.p.dt_iters) break;
        if (cur.empty()) break;
        nxt.clear();
        for (const Elem &e : cur) {
            for (const Edge &E : next_label[e.label]) {
                int64_t gp = e.grid_index + E.dir * t.stride[E.dim];
                if (gp >= 0 && gp < t.ncells && t.table[gp] == UNUSED) {
                    int64_t dp = (e.grid_index / t.stride[E.dim]) % t.nslices[E.dim] + E.dir;
                    if (dp >= 0 && dp < t.nslices[E.dim]) {
                        t.table[gp] = e.table_value;
                        nxt.push_back(Elem{gp, e.table_value, (uint8_t) E.label});
                    }
                }
            }
        }
        cur.swap(nxt);
    }
}

const int HI_MASK = 1 << 30;       /* TABLE_HI_MASK, patchtable.h:109-112 */

/* do_dt_prop1, patchtable.h:2306-2325.  Cells are visited in increasing index; each populated
   cell without the high bit writes its value, with the high bit set, into every adjacent cell
   that is still unused.  An unused cell therefore ends up with the value of its
   lowest-indexed populated neighbour. */
void dt_prop1(Table &t) {
    int G = t.gnd;
    for (int64_t j = 0; j < t.ncells; j++) {
        int32_t v = t.table[j];
        if (v == UNUSED || (v & HI_MASK)) continue;
        for (int i = 0; i < G; i++) {
            int64_t c = (j / t.stride[i]) % t.nslices[i];
            if (c > 0 && t.table[j - t.stride[i]] == UNUSED) t.table[j - t.stride[i]] = v | HI_MASK;
            if (c + 1 < t.nslices[i] && t.table[j + t.stride[i]] == UNUSED) t.table[j + t.stride[i]] = v | HI_MASK;
        }
    }
}

/* unmask_table, patchtable.h:2332-2336. */
void dt_unmask(Table &t) {
    for (auto &v : t.table) v &= HI_MASK - 1;
}

namespace {

/* One level of the downsample pyramid: sizes and row-major strides (dimension 0 slowest, like
   Array's layout). */
struct Level {
    vector<int> size;
    vector<int64_t> stride;
    vector<int32_t> v;
    void shape(const vector<int> &s) {
        size = s;
        stride.assign(s.size(), 1);
        int64_t n = 1;
        for (int d = (int) s.size() - 1; d >= 0; d--) { stride[d] = n; n *= s[d]; }
        v.assign((size_t) n, UNUSED);
    }
};

/* Coordinates of flat index j. */
void coords_of(int64_t j, const Level &L, vector<int> &c) {
    for (size_t d = 0; d < L.size.size(); d++) c[d] = (int) ((j / L.stride[d]) % L.size[d]);
}

}  // namespace

/* do_dt_downsample, patchtable.h:2339-2358, with dt_downsample / dt_upsample (the generated
   dt_downsample.h).  Each coarser level halves every size (rounding up) until all sizes are 1;
   a coarse cell takes the first of its up to 2^G children, in lexicographic order with
   dimension 0 slowest, that holds a value without the high bit, or stays unused.  Going back
   down, every unused fine cell copies its parent. */
void dt_downsample(Table &t) {
    int G = t.gnd;
    vector<Level> pyr(1);
    pyr[0].size = t.nslices;
    pyr[0].stride = t.stride;
    pyr[0].v = t.table;
    vector<int> c(G), cc(G);
    for (;;) {
        const Level &hi = pyr.back();
        bool unit = true;
        for (int s : hi.size) unit = unit && s == 1;
        if (unit) break;
        vector<int> ls(G);
        for (int d = 0; d < G; d++) ls[d] = (hi.size[d] + 1) / 2;
        Level lo;
        lo.shape(ls);
        for (int64_t j = 0; j < (int64_t) lo.v.size(); j++) {
            coords_of(j, lo, c);
            /* odometer over the children, last dimension fastest */
            for (int d = 0; d < G; d++) cc[d] = 2 * c[d];
            int32_t found = UNUSED;
            for (;;) {
                int64_t hj = 0;
                for (int d = 0; d < G; d++) hj += cc[d] * hi.stride[d];
                int32_t v = hi.v[hj];
                if (!(v & HI_MASK) && v != UNUSED) { found = v; break; }
                int d = G - 1;
                for (; d >= 0; d--) {
                    if (++cc[d] < std::min(2 * c[d] + 2, hi.size[d])) break;
                    cc[d] = 2 * c[d];
                }
                if (d < 0) break;
            }
            lo.v[j] = found;
        }
        pyr.push_back(std::move(lo));
    }
    for (size_t k = pyr.size() - 1; k >= 1; k--) {
        const Level &lo = pyr[k];
        Level &hi = pyr[k - 1];
        for (int64_t j = 0; j < (int64_t) hi.v.size(); j++) {
            if (hi.v[j] != UNUSED) continue;
            coords_of(j, hi, c);
            int64_t lj = 0;
            for (int d = 0; d < G; d++) lj += (c[d] / 2) * lo.stride[d];
            hi.v[j] = lo.v[lj];
        }
    }
    t.table = pyr[0].v;
}

/* do_dt_euclidean + euclidean_dt, patchtable.h:4244-4340: the Felzenszwalb-Huttenlocher
   lower envelope of parabolas, one dimension after another, in single precision.  Distances
   start at 1E20 for unused cells and 0 for populated ones; the nearest cell's value is carried
   along in place, so a cell whose parabola lies before it reads the value already moved there
   in the same line (index_array, patchtable.h:4265). */
void dt_euclidean(Table &t) {
    int G = t.gnd;
    const float INF_F = (float) 1E20;
    vector<float> dist((size_t) t.ncells);
    for (int64_t j = 0; j < t.ncells; j++) dist[j] = t.table[j] == UNUSED ? INF_F : 0.0f;
    int maxn = 0;
    for (int d = 0; d < G; d++) maxn = std::max(maxn, t.nslices[d]);
    /* The reference squares ints (curNo*curNo); its build wraps them at 32 bits, which matters
       from 46341 cells along one dimension on. */
    auto sq = [](int x) { return (float) (int32_t) ((uint32_t) x * (uint32_t) x); };
    vector<float> f(maxn), dd(maxn), z(maxn + 1);
    vector<int> v(maxn);
    vector<int32_t> idx(maxn);
    for (int dim = 0; dim < G; dim++) {
        int n = t.nslices[dim];
        int64_t st = t.stride[dim];
        for (int64_t base = 0; base < t.ncells; base++) {
            if ((base / st) % n != 0) continue;          /* one line per start cell with coord 0 */
            for (int q = 0; q < n; q++) { f[q] = dist[base + q * st]; idx[q] = t.table[base + q * st]; }
            int k = 0;
            v[0] = 0; z[0] = -INF_F; z[1] = INF_F;
            for (int q = 1; q < n; q++) {
                float s = ((f[q] + sq(q)) - (f[v[k]] + sq(v[k]))) / (float) (2 * q - 2 * v[k]);
                while (s <= z[k]) {
                    k--;
                    s = ((f[q] + sq(q)) - (f[v[k]] + sq(v[k]))) / (float) (2 * q - 2 * v[k]);
                }
                k++;
                v[k] = q; z[k] = s; z[k + 1] = INF_F;
            }
            k = 0;
            for (int q = 0; q < n; q++) {
                while (z[k + 1] < (float) q) k++;
                dd[q] = sq(q - v[k]) + f[v[k]];
                idx[q] = idx[v[k]];
            }
            for (int q = 0; q < n; q++) { dist[base + q * st] = dd[q]; t.table[base + q * st] = idx[q]; }
        }
    }
}

/* do_dt_brute, patchtable.h:2364-2413: every cell takes, over the whole valid patch region of b
   (the allowed mask is not consulted), the patch nearest the cell under patch_dist_to_grid<0>
   (patchtable.h:1403-1425) with TABLE_INFINITY_NORM: the largest over grid dimensions of
   |wh - centre| / (rsize when wh - centre > 0, else lsize), maxima taken as (a > b ? a : b).
   The first patch in raster order seeds the search and a later one replaces it only when
   strictly nearer, so ties keep the earliest. */
void dt_brute(Table &t) {
    const int G = t.gnd;
    vector<int> gi(G);
    for (int64_t j = 0; j < t.ncells; j++) {
        for (int i = 0; i < G; i++) gi[i] = (int) ((j / t.stride[i]) % t.nslices[i]);
        auto dist = [&](int x, int y) {
            float ans = 0;
            for (int i = 0; i < G; i++) {
                const Partition1D &P = t.part[i];
                float delta = t.whv(y, x, i) - P.centers[gi[i]];
                float sz = delta > 0 ? P.rsizes[gi[i]] : P.lsizes[gi[i]];
                delta = std::fabs(delta) / sz;
                ans = ans > delta ? ans : delta;
            }
            return ans;
        };
        int xb = PW - 1, yb = PW - 1;
        float db = dist(xb, yb);
        for (int y = PW - 1; y < t.h; y++)
            for (int x = PW - 1; x < t.w; x++) {
                float d = dist(x, y);
                if (d < db) { db = d; xb = x; yb = y; }
            }
        t.table[j] = xy_to_int(xb, yb);
    }
}

/* k-coherence with the FLANN path, patchtable.h:2653-2869 (TABLE_KCOHERENCE_TRIANGLE,
   kcoherence_algo flann, incoherence off).  The vectors is_valid / matched_* live across the
   patch loop exactly as in the reference, so entries past the early break keep the values the
   previous patch left in them (patchtable.h:2675-2677, 2793-2796). */
void build_kcoherence(Table &t) {
    const orc_params &p = t.p;
    const int xmin = 7, ymin = 7, xmax = t.w, ymax = t.h;
    int bew = xmax - xmin, beh = ymax - ymin;
    int K = p.kcoherence, nd = t.nd;
    t.kc_h = beh; t.kc_w = bew;
    t.kc_pos.assign((size_t) beh * bew * K, 0);
    t.kc_dist.assign((size_t) beh * bew * K, 0.0f);
    /* build_flann_index_func, patchtable.h:822-861. */
    vector<float> train;
    vector<int> index_to_pos;
    for (int y = ymin; y < ymax; y += p.flann_build_step)
        for (int x = xmin; x < xmax; x += p.flann_build_step) {
            if (!t.is_allowed(y - ymin, x - xmin)) continue;
            for (int i = 0; i < nd; i++) train.push_back(t.whv(y, x, i));
            index_to_pos.push_back(xy_to_int(x - xmin, y - ymin));
        }
    ptoracle::ExactKnn index(train.data(), (int) index_to_pos.size(), nd);
    int knn0 = K + 1;
    vector<float> q(nd);
    vector<bool> is_valid(knn0);
    vector<int> matched_indices(knn0);
    vector<float> matched_dists(knn0);
    vector<ptoracle::KnnResult> res;
    int prev_knn = knn0;
    int min_dist2 = p.kcoherence_min_dist * p.kcoherence_min_dist;
    vector<std::pair<float, std::pair<int, int>>> triples;
    for (int y = ymin; y < ymax; y += p.kcoherence_step) {
        for (int x = xmin; x < xmax; x += p.kcoherence_step) {
            if (!t.is_allowed(y - ymin, x - xmin)) continue;
            int yk = (y - ymin) / p.kcoherence_step, xk = (x - xmin) / p.kcoherence_step;
            for (int i = 0; i < nd; i++) q[i] = t.whv(y, x, i);
            int knn = (x / p.kcoherence_step) % p.flann_reset_step == 0 ? knn0 : prev_knn;
            while (1) {
                is_valid.resize(knn);
                matched_indices.resize(knn);
                matched_dists.resize(knn);
                index.query(q.data(), knn, res);
                if ((int) res.size() < knn) { fprintf(stderr, "oracle: k-coherence needs more points\n"); abort(); }
                for (int i = 0; i < knn; i++) { matched_indices[i] = index_to_pos[res[i].idx]; matched_dists[i] = res[i].dist; }
                int nvalid = 0;
                for (int i = 0; i < knn; i++) {
                    int bx = int_to_x(matched_indices[i]), by = int_to_y(matched_indices[i]);
                    int dx = bx + xmin - x, dy = by + ymin - y;
                    is_valid[i] = dx * dx + dy * dy >= min_dist2;
                    if (is_valid[i]) { nvalid++; if (nvalid >= K) break; }
                }
                if (nvalid < K) { knn *= 2; continue; }
                /* Exact distance of each match to this patch, then sort (dist, pos, valid). */
                for (int i = 0; i < knn; i++) {
                    int v = matched_indices[i];
                    if (p.is_descriptor)   /* TABLE_PREPARE_B_DIST / TABLE_LOOKUP_PATCH_DIST, patchtable.h:310-320 */
                        matched_dists[i] = patch_dist_approx(&t.wh0[((size_t) y * t.WW() + x) * nd],
                                                             &t.wh0[((size_t) (int_to_y(v) + 7) * t.WW() + int_to_x(v) + 7) * nd], nd);
                    else
                        matched_dists[i] = patch_dist_exact(t.b0.data(), t.w, x - xmin, y - ymin, t.b0.data(), t.w, int_to_x(v), int_to_y(v));
                }
                triples.resize(knn);
                for (int i = 0; i < knn; i++) triples[i] = std::make_pair(matched_dists[i], std::make_pair(matched_indices[i], (int) is_valid[i]));
                std::sort(triples.begin(), triples.end());
                for (int i = 0; i < knn; i++) {
                    matched_dists[i] = triples[i].first;
                    matched_indices[i] = triples[i].second.first;
                    is_valid[i] = triples[i].second.second;
                }
                int cv = 0;
                for (int i = 0; i < knn; i++) {
                    if (is_valid[i]) {
                        size_t o = ((size_t) yk * t.kc_w + xk) * K + cv;
                        t.kc_pos[o] = xy_to_int(int_to_x(matched_indices[i]), int_to_y(matched_indices[i]));
                        t.kc_dist[o] = matched_dists[i];
                        cv++;
                        if (cv >= K) break;
                    }
                }
                break;
            }
            prev_knn = knn;
            t.kc_max_knn = std::max(t.kc_max_knn, knn);
        }
    }
}

/* lookup_templated<is_descriptor, use_allowed_patches>, patchtable.h:3468-4217.  In descriptor
   mode a is ah x aw x ndims descriptors, every distance is patch_dist_approx of the two padded
   descriptor vectors and propagation scores candidates one by one instead of through the
   summed-area table (patchtable.h:3943, 4043-4060). */
double lookup(Table &t, const float *a, int ah, int aw, double *ann, const double *ann_prev,
              const float *coh_sv) {
    const orc_params &p = t.p;
    vector<float> &a_wh = t.lookup_wh;
    const bool desc = p.is_descriptor;
    if (desc) {
        padded_input(p, a, ah, aw, a_wh, ah, aw);
    } else if (p.dim_algo == 1) {
        vector<float> img((size_t) ah * aw * 3);
        convert_color(p, a, ah * aw, img.data());
        pca_apply(p, t.pca, img.data(), ah, aw, a_wh);
    } else {
        padded_descriptor(p, a, ah, aw, a_wh);
    }
    const int nd = t.nd, G = t.gnd;
    const int awhw = aw + 7;
    double prop_scale = 1.0 / (1 + p.coherence_spatial);
    double temporal_scale = 1.0 / (1 + p.coherence_temporal);
    int ann_h = ah - PW + 1, ann_w = aw - PW + 1;
    int b0_ew = t.w - PW + 1, b0_eh = t.h - PW + 1;
    int a_w = aw, a_h = ah, b_w = t.w, b_h = t.h;
    bool use_allowed = !t.allowed.empty();
    auto ANN = [&](int y, int x, int c) -> double & { return ann[((size_t) y * ann_w + x) * 3 + c]; };
    auto dist = [&](int ax, int ay, int bx, int by) {
        if (desc)
            return patch_dist_approx(&a_wh[((size_t) (ay + 7) * awhw + ax + 7) * nd],
                                     &t.wh0[((size_t) (by + 7) * t.WW() + bx + 7) * nd], nd);
        return patch_dist_exact(a, aw, ax, ay, t.b0.data(), t.w, bx, by);
    };
    vector<float> lookup_dist_orig;
    if (p.init_random) {                                  /* patchtable.h:3522-3537 */
        for (int y = 0; y < ann_h; y++)
            for (int x = 0; x < ann_w; x++) {
                int xs = rand() % b0_ew, ys = rand() % b0_eh;
                ANN(y, x, 0) = xs; ANN(y, x, 1) = ys; ANN(y, x, 2) = dist(x, y, xs, ys);
            }
    } else if (!ann_prev) {                               /* patchtable.h:3538-3547 */
        for (int y = 0; y < ann_h; y++)
            for (int x = 0; x < ann_w; x++) {
                ANN(y, x, 0) = b0_ew + 1;
                ANN(y, x, 1) = 0;        /* left uninitialised by the reference; never read when do_table_lookup */
                ANN(y, x, 2) = DIST_INF;
            }
    } else {                                              /* patchtable.h:3548-3585 */
        lookup_dist_orig.assign((size_t) ann_h * ann_w, 0.0f);
        for (int y = 0; y < ann_h; y++)
            for (int x = 0; x < ann_w; x++) {
                const double *pp = &ann_prev[((size_t) y * ann_w + x) * 3];
                int xs = (int) pp[0], ys = (int) pp[1];
                if (p.sanitize_input) {
                    if (xs < 0) xs = 0; else if (xs >= b0_ew) xs = b0_ew - 1;
                    if (ys < 0) ys = 0; else if (ys >= b0_eh) ys = b0_eh - 1;
                }
                ANN(y, x, 0) = xs; ANN(y, x, 1) = ys;
                if (p.recalc_dist_temporal) {
                    float dc = dist(x, y, xs, ys);
                    double ts = coh_sv ? (double) coh_sv[(size_t) y * ann_w + x] : temporal_scale;
                    float v = (float) (dc * ts);
                    lookup_dist_orig[(size_t) y * ann_w + x] = v;
                    ANN(y, x, 2) = v;
                } else {
                    ANN(y, x, 2) = pp[2] * temporal_scale;
                }
            }
    }
    const int dx_table[8] = {-1, 0, 1, -1, 1, -1, 0, 1};
    const int dy_table[8] = {-1, -1, -1, 0, 0, 1, 1, 1};
    bool do_rs_or_spatial = p.do_rs || p.spatial;
    int prop_w = (p.query_step + p.prop_dist) * 2 + 1;
    int sat_w = PW + prop_w + 1 - 1;
    int sat_w_nopad = sat_w - 1;
    const int pw1 = PW - 1;
    for (int prop_iter = 0; prop_iter < p.prop_iters; prop_iter++) {
        bool reverse = prop_iter % 2;
        bool do_lookup = prop_iter == 0 && p.do_table_lookup;
        bool do_kcoh = p.kcoherence > 0 && (p.kcoherence_iter < 0 || p.kcoherence_iter == prop_iter);
        for (int y0 = 0; y0 < ann_h; y0 += p.query_step) {
            int y = reverse ? (ann_h - 1 - y0) : y0;
            vector<float> sat((size_t) sat_w * sat_w, 0.0f);
            for (int x0 = 0; x0 < ann_w; x0 += p.query_step) {
                int x = reverse ? (ann_w - 1 - x0) : x0;
                int xbest = (int) ANN(y, x, 0);
                int ybest = (int) ANN(y, x, 1);
                float dbest = (float) (ANN(y, x, 2) * prop_scale);
                if (do_lookup) {                          /* patchtable.h:3641-3709 */
                    const float *wh_p = &a_wh[((size_t) (y + pw1) * awhw + (x + pw1)) * nd];
                    int64_t idx = 0;
                    for (int i = 0; i < G; i++) idx += (int64_t) t.part[i].get_bin(wh_p[i]) * t.stride[i];
                    int v = t.table[idx];
                    int xs = int_to_x(v) - pw1, ys = int_to_y(v) - pw1;
                    if (xs != xbest || ys != ybest) {
                        float dc = dist(x, y, xs, ys);
                        if (dc < dbest) { dbest = dc; xbest = xs; ybest = ys; }
                    }
                    int xprev = xs, yprev = ys;          /* further tables, patchtable.h:3711-3735 */
                    for (const auto &u : t.subs) {
                        int64_t idx1 = 0;
                        for (int i = 0; i < G; i++) idx1 += (int64_t) u->part[i].get_bin(wh_p[i]) * u->stride[i];
                        int v1 = u->table[idx1];
                        int xs1 = int_to_x(v1) - pw1, ys1 = int_to_y(v1) - pw1;
                        if ((xs1 != xbest || ys1 != ybest) && (xs1 != xprev || ys1 != yprev)) {
                            float dc = dist(x, y, xs1, ys1);
                            if (dc < dbest) { dbest = dc; xbest = xs1; ybest = ys1; }
                        }
                        xprev = xs1; yprev = ys1;
                    }
                }
                if (do_kcoh) {                            /* patchtable.h:3750-3851 */
                    int ks = p.kcoherence_step;
                    const int32_t *kp = &t.kc_pos[((size_t) (ybest / ks) * t.kc_w + (xbest / ks)) * p.kcoherence];
                    const float *kd = &t.kc_dist[((size_t) (ybest / ks) * t.kc_w + (xbest / ks)) * p.kcoherence];
                    int kdx = 0, kdy = 0;
                    if (ks > 1) { kdx = xbest % ks; kdy = ybest % ks; }
                    for (int k = 0; k < p.kcoherence; k++) {
                        float k_dist = kd[k];
                        if (k_dist >= p.triangle_factor * dbest) break;
                        int v = kp[k];
                        int xs = int_to_x(v), ys = int_to_y(v);
                        if (ks > 1) {
                            xs += kdx; ys += kdy;
                            if (xs >= b0_ew) xs = b0_ew - 1;
                            if (ys >= b0_eh) ys = b0_eh - 1;
                        }
                        float dc = dist(x, y, xs, ys);
                        if (dc < dbest) { dbest = dc; xbest = xs; ybest = ys; }
                    }
                }
                if (do_rs_or_spatial) {                   /* patchtable.h:3854-3905 */
                    if (p.spatial) {
                        int symin = ybest - p.spatial, symax = ybest + p.spatial + 1;
                        int sxmin = xbest - p.spatial, sxmax = xbest + p.spatial + 1;
                        int xb0 = xbest, yb0 = ybest;
                        if (symin < 0) symin = 0; else if (symax > b0_eh) symax = b0_eh;
                        if (sxmin < 0) sxmin = 0; else if (sxmax > b0_ew) sxmax = b0_ew;
                        for (int ys = symin; ys < symax; ys++)
                            for (int xs = sxmin; xs < sxmax; xs++)
                                if ((xs != xb0 || ys != yb0) && (!use_allowed || t.is_allowed(ys, xs))) {
                                    float dc = dist(x, y, xs, ys);
                                    if (dc < dbest) { dbest = dc; xbest = xs; ybest = ys; }
                                }
                    } else {
                        int r = rand() & 7;
                        int xs = xbest + dx_table[r], ys = ybest + dy_table[r];
                        if (xs >= 0 && xs < b0_ew && ys >= 0 && ys < b0_eh && (!use_allowed || t.is_allowed(ys, xs))) {
                            float dc = dist(x, y, xs, ys);
                            if (dc < dbest) { dbest = dc; xbest = xs; ybest = ys; }
                        }
                    }
                }
                if (p.do_prop) {                          /* patchtable.h:3908-4145 */
                    int ax_shift = x - p.query_step, ay_shift = y - p.query_step;
                    int bx_shift = xbest - p.query_step, by_shift = ybest - p.query_step;
                    int dy_min = 0, dy_max = sat_w_nopad, dx_min = 0, dx_max = sat_w_nopad;
                    if (ax_shift + dx_min < 0) dx_min = -ax_shift;
                    else if (ax_shift + dx_max > a_w) dx_max = a_w - ax_shift;
                    if (ay_shift + dy_min < 0) dy_min = -ay_shift;
                    else if (ay_shift + dy_max > a_h) dy_max = a_h - ay_shift;
                    if (bx_shift + dx_min < 0) dx_min = -bx_shift;
                    else if (bx_shift + dx_max > b_w) dx_max = b_w - bx_shift;
                    if (by_shift + dy_min < 0) dy_min = -by_shift;
                    else if (by_shift + dy_max > b_h) dy_max = b_h - by_shift;
                    if (!desc && (dx_min > 0 || dy_min > 0)) {
                        if (dx_min > 0)
                            for (int dy = dy_min > 0 ? dy_min - 1 : dy_min; dy < dy_max; dy++) sat[(size_t) (dy + 1) * sat_w + dx_min] = 0;
                        if (dy_min > 0)
                            for (int dx = dx_min; dx < dx_max; dx++) sat[(size_t) dy_min * sat_w + dx + 1] = 0;
                    }
                    for (int dy = dy_min; dy < dy_max && !desc; dy++) {
                        const float *a_row = a + ((size_t) (ay_shift + dy) * aw + ax_shift) * 3;
                        const float *b_row = t.b0.data() + ((size_t) (by_shift + dy) * t.w + bx_shift) * 3;
                        float *sat_row = &sat[(size_t) (dy + 1) * sat_w + 1];
                        float *sat_row_prev = &sat[(size_t) dy * sat_w + 1];
                        float row_sum = 0;
                        for (int dx = dx_min; dx < dx_max; dx++) {
                            const float *ap = a_row + dx * 3, *bp = b_row + dx * 3;
                            float d0 = ap[0] - bp[0], d1 = ap[1] - bp[1], d2 = ap[2] - bp[2];
                            row_sum += d0 * d0 + d1 * d1 + d2 * d2;
                            sat_row[dx] = row_sum + sat_row_prev[dx];
                        }
                    }
                    int dy_max_patch = dy_max - PW + 1, dx_max_patch = dx_max - PW + 1;
                    bool missing = false;
                    for (int dy = dy_min; dy < dy_max_patch; dy++) {
                        const float *s1 = &sat[(size_t) dy * sat_w];
                        const float *s2 = &sat[(size_t) (dy + PW) * sat_w];
                        int ys = dy + by_shift;
                        for (int dx = dx_min; dx < dx_max_patch; dx++) {
                            int xs = dx + bx_shift;
                            if (use_allowed && !t.is_allowed(ys, xs)) { missing = true; continue; }
                            int dx2 = dx + PW;
                            float dc = desc ? dist(ax_shift + dx, ay_shift + dy, xs, ys)
                                            : s1[dx] - s1[dx2] - s2[dx] + s2[dx2];
                            double *ap = &ANN(ay_shift + dy, ax_shift + dx, 0);
                            if (dc < ap[2]) { ap[0] = xs; ap[1] = ys; ap[2] = dc; }
                        }
                    }
                    if (dx_max < sat_w_nopad || dy_max < sat_w_nopad || missing) {   /* patchtable.h:4086-4145 */
                        int dy_start, dy_end, dx_start, dx_end;
                        if (missing) {
                            dx_start = 0; dx_end = p.query_step * 2;
                            dy_start = 0; dy_end = p.query_step * 2;
                            if (ax_shift + dx_start < 0) dx_start = -ax_shift;
                            if (ay_shift + dy_start < 0) dy_start = -ay_shift;
                            if (ax_shift + dx_end > ann_w) dx_end = ann_w - ax_shift;
                            if (ay_shift + dy_end > ann_h) dy_end = ann_h - ay_shift;
                        } else if (reverse) {
                            dx_start = 0; dx_end = p.query_step;
                            dy_start = 0; dy_end = p.query_step;
                            if (ax_shift + dx_start < 0) dx_start = -ax_shift;
                            if (ay_shift + dy_start < 0) dy_start = -ay_shift;
                        } else {
                            dx_start = p.query_step; dx_end = p.query_step * 2;
                            dy_start = p.query_step; dy_end = p.query_step * 2;
                            if (ax_shift + dx_end > ann_w) dx_end = ann_w - ax_shift;
                            if (ay_shift + dy_end > ann_h) dy_end = ann_h - ay_shift;
                        }
                        for (int dy = dy_start; dy < dy_end; dy++) {
                            int ys = ybest + (ay_shift + dy) - y;
                            if (ys < 0) ys = 0; else if (ys >= b0_eh) ys = b0_eh - 1;
                            for (int dx = dx_start; dx < dx_end; dx++) {
                                double *ap = &ANN(ay_shift + dy, ax_shift + dx, 0);
                                if (ap[2] == DIST_INF) {
                                    int xs = xbest + (ax_shift + dx) - x;
                                    if (xs < 0) xs = 0; else if (xs >= b0_ew) xs = b0_ew - 1;
                                    if (use_allowed)
                                        while (!t.is_allowed(ys, xs)) { xs = rand() % b0_ew; ys = rand() % b0_eh; }
                                    float dc = dist(ax_shift + dx, ay_shift + dy, xs, ys);
                                    ap[2] = dc; ap[0] = xs; ap[1] = ys;
                                }
                            }
                        }
                    }
                } else {
                    ANN(y, x, 0) = xbest; ANN(y, x, 1) = ybest; ANN(y, x, 2) = dbest;
                }
            }
        }
    }
    if (ann_prev && p.coherence_temporal != 0.0) {       /* patchtable.h:4178-4193 */
        for (int y = 0; y < ann_h; y++)
            for (int x = 0; x < ann_w; x++) {
                double *ap = &ANN(y, x, 0);
                const double *pp = &ann_prev[((size_t) y * ann_w + x) * 3];
                if (ap[0] == pp[0] && ap[1] == pp[1]) {
                    if ((p.recalc_dist_temporal && ap[2] == lookup_dist_orig[(size_t) y * ann_w + x]) ||
                        (!p.recalc_dist_temporal && ap[2] == pp[2] * temporal_scale))
                        ap[2] /= temporal_scale;
                }
            }
    }
    return 0.0;
}

}  // namespace

extern "C" {

void orc_srand(unsigned s) { srand(s); }

void orc_rgb2yuv(const float *in, int h, int w, float *out) { rgb2yuv(in, h * w, out); }

void orc_rgb2lab(const float *in, int h, int w, float *out) { rgb2lab(in, h * w, out); }

void orc_gck(const float *yuv, int h, int w, int n, int nchroma, float *out) { gck8(yuv, h, w, n, nchroma, out); }

/* patch_dist_approx of two descriptor vectors. */
float orc_patch_dist_approx(const float *a, const float *b, int nd) { return patch_dist_approx(a, b, nd); }

/* Padded descriptor of an RGB image: (h+7) x (w+7) x ndims. */
void orc_descriptor(const orc_params *p, const float *rgb, int h, int w, float *out) {
    vector<float> wh;
    padded_descriptor(*p, rgb, h, w, wh);
    memcpy(out, wh.data(), sizeof(float) * wh.size());
}

float orc_patch_dist(const float *a, int aw, int ax, int ay, const float *b, int bw, int bx, int by) {
    return patch_dist_exact(a, aw, ax, ay, b, bw, bx, by);
}

void orc_scale_slices(const int *in, int n, double limit, int *out) {
    vector<int> r = scale_slices_to_limit(vector<int>(in, in + n), limit);
    for (int i = 0; i < n; i++) out[i] = r[i];
}

/* wh0 may be NULL (computed from b) or a (h+7) x (w+7) x ndims descriptor to build from. */
void *orc_build(const orc_params *p, const float *b, int h, int w, const int32_t *allowed, const float *wh0) {
    return build(*p, b, h, w, allowed, wh0);
}

void orc_free(void *t) { delete (Table *) t; }

/* Further table i of an ntables > 1 build (owned by t), or NULL. */
void *orc_subtable(void *tv, int i) {
    Table *t = (Table *) tv;
    return i >= 0 && i < (int) t->subs.size() ? t->subs[i].get() : nullptr;
}

int orc_table_shape(void *tv, int *nslices, long long *ncells) {
    Table *t = (Table *) tv;
    for (int i = 0; i < t->gnd; i++) nslices[i] = t->nslices[i];
    *ncells = t->ncells;
    return t->gnd;
}

int orc_table_add_count(void *tv) { return ((Table *) tv)->table_add_count; }
int orc_kc_max_knn(void *tv) { return ((Table *) tv)->kc_max_knn; }

void orc_get_table(void *tv, int32_t *out) {
    Table *t = (Table *) tv;
    memcpy(out, t->table.data(), sizeof(int32_t) * t->table.size());
}

void orc_get_wh0(void *tv, float *out) {
    Table *t = (Table *) tv;
    memcpy(out, t->wh0.data(), sizeof(float) * t->wh0.size());
}

void orc_get_partition(void *tv, int dim, float *centers, float *lsizes, float *rsizes, int32_t *to_bin, float *mmr) {
    Table *t = (Table *) tv;
    const Partition1D &P = t->part[dim];
    for (int i = 0; i < P.nslices; i++) { centers[i] = P.centers[i]; lsizes[i] = P.lsizes[i]; rsizes[i] = P.rsizes[i]; }
    for (int i = 0; i < NMAP; i++) to_bin[i] = P.to_bin[i];
    mmr[0] = P.min_val; mmr[1] = P.max_val; mmr[2] = P.range;
}

void orc_get_kcoherence(void *tv, int32_t *pos, float *dist) {
    Table *t = (Table *) tv;
    memcpy(pos, t->kc_pos.data(), sizeof(int32_t) * t->kc_pos.size());
    memcpy(dist, t->kc_dist.data(), sizeof(float) * t->kc_dist.size());
}

/* ann_out: (ah-7) x (aw-7) x 3 doubles [x, y, dist]; in descriptor mode a is ah x aw x ndims and
   ann_out ah x aw x 3 (padded: (ah-14) x (aw-14) x 3).  ann_prev / coh_sv may be NULL. */
void orc_lookup(void *tv, const float *a, int ah, int aw, double *ann_out, const double *ann_prev, const float *coh_sv) {
    lookup(*(Table *) tv, a, ah, aw, ann_out, ann_prev, coh_sv);
}

}  // extern "C"
