/* Patch descriptor kernel: RGB -> (RGBA copy, YUV, Walsh-Hadamard projections of every 8x8 patch).

   Replaces get_padded_descriptor (patchtable/patchtable.h:2492-2546): ARRAY_RGB2YUV
   (solver/array.h:1116-1127) followed by gck_8 (patchtable/gck.h:29-1950).  The reference
   evaluates the projections with running sums along rows and columns; this kernel computes each
   patch's projections directly from a shared-memory tile, so there is no sequential dependency
   and every output is an independent 8-term sum per pass.  Values agree with the reference to
   float rounding (the reference's running sums drift along long rows).

   One CTA owns a 64 x 8 block of patches.  It loads the (8+7) x (64+7) pixel region once with
   coalesced loads, converts it to YUV in double precision exactly as the reference does (double
   constants, left-to-right sum, rounded to float), applies each needed horizontal sign vector
   per row, then each vertical sign vector per patch, and writes the descriptor as ndims floats
   padded to a 32- or 64-byte record.  The same pass writes the RGBA (float4) copy of the image
   used by the distance kernels. */
#include <cuda_runtime.h>
#include <cstdio>
#include <mutex>

#include "pt_bins.cuh"
#include "pt_internal.h"
#include "wh_tables.h"
#include "pt_kernels.h"

namespace {

constexpr int TW = 64, TH = 8;            /* patches per CTA */
constexpr int RW = TW + 7, RH = TH + 7;   /* pixel region per CTA */
constexpr int RWP = RW + 1;               /* padded smem row */
constexpr int NT = 256;

/* The table step fused into the query's descriptor pass: each patch's cell (get_bin over the grid
   dimensions, exactly as k_table_cand computes it from stored descriptors) and its entry
   tcand[p] = table[cell], so the plain query never stores or re-reads its descriptors. */
struct CellPlan {
    int G;
    float min_val[PT_DESC_MAX], range[PT_DESC_MAX];
    long long stride[PT_DESC_MAX];
    const int *to_bin;
    const int *table;
    int *tcand;
};

struct DescPlan {
    int nd;                               /* output channels */
    int ncombo;                           /* distinct (plane, horizontal vector) filters */
    int combo_plane[PT_DESC_MAX];
    signed char combo_h[PT_DESC_MAX][8];
    int ch_combo[PT_DESC_MAX];
    signed char ch_v[PT_DESC_MAX][8];
    /* the same signs as +-1.0f: a fused multiply-add by +-1 rounds exactly like the add or
       subtract it stands for, and reads the sign straight from the parameter bank */
    float combo_hf[PT_DESC_MAX][8];
    float ch_vf[PT_DESC_MAX][8];
};


__device__ __forceinline__ void yuv_exact(float R, float G, float B, float &Y, float &U, float &V) {
    /* ARRAY_RGB2YUV, solver/array.h:1124-1126: double constants x float pixels, summed left to
       right in double, stored as float.  Explicit _rn intrinsics keep the compiler from fusing. */
    double r = R, g = G, b = B;
    Y = __double2float_rn(__dadd_rn(__dadd_rn(__dmul_rn(0.299, r), __dmul_rn(0.587, g)), __dmul_rn(0.114, b)));
    U = __double2float_rn(__dadd_rn(__dadd_rn(__dmul_rn(-0.14713, r), __dmul_rn(-0.28886, g)), __dmul_rn(0.436, b)));
    V = __double2float_rn(__dadd_rn(__dadd_rn(__dmul_rn(0.615, r), __dmul_rn(-0.51499, g)), __dmul_rn(-0.10001, b)));
}


/* -colorspace lab: Array::rgb2lab (solver/array.h:1246-1256) = rgb2xyz (:1213-1244) then xyz2lab
   (:1264-1292), whose powers come from PowTable (solver/array.h:221-237): 1024 entries
   table[i] = (float) pow((i + 0.5) / 1024, p) for p = (float) 2.4 and (float) (1/3), read at
   int(v * 1024.0f) clamped to the table.  The tables are filled once per device from the host
   C library's pow, the arithmetic around them is the reference's double / float mix. */
__device__ float g_lab_pow[2][PT_LAB_N];

__device__ __forceinline__ float lab_tab(int t, float v) {
    int i = __float2int_rz(__fmul_rn(v, (float) PT_LAB_N));
    i = i < 0 ? 0 : (i >= PT_LAB_N ? PT_LAB_N - 1 : i);
    return g_lab_pow[t][i];
}

__device__ __forceinline__ float srgb_linear(float c) {
    const double cd = c;
    if (cd <= 0.04045) return __double2float_rn(__ddiv_rn(cd, 12.92));
    return lab_tab(0, __double2float_rn(__ddiv_rn(__dadd_rn(cd, 0.055), 1.055)));
}

__device__ __forceinline__ float lab_f(float r) {
    if ((double) r > 0.008856) return lab_tab(1, r);
    return __double2float_rn(__ddiv_rn(__dadd_rn(__dmul_rn(903.3, (double) r), 16.0), 116.0));
}

__device__ __forceinline__ void lab_exact(float R, float G, float B, float &L, float &A, float &Bo) {
    const double r = srgb_linear(R), g = srgb_linear(G), b = srgb_linear(B);
    const float X = __double2float_rn(__dadd_rn(__dadd_rn(__dmul_rn(0.4360747, r), __dmul_rn(0.3850649, g)), __dmul_rn(0.1430804, b)));
    const float Y = __double2float_rn(__dadd_rn(__dadd_rn(__dmul_rn(0.2225045, r), __dmul_rn(0.7168786, g)), __dmul_rn(0.0606169, b)));
    const float Z = __double2float_rn(__dadd_rn(__dadd_rn(__dmul_rn(0.0139322, r), __dmul_rn(0.0971045, g)), __dmul_rn(0.7141733, b)));
    const float fx = lab_f(__double2float_rn(__ddiv_rn((double) X, 0.9642)));
    const float fy = lab_f(__double2float_rn(__ddiv_rn((double) Y, 1.0)));
    const float fz = lab_f(__double2float_rn(__ddiv_rn((double) Z, 0.8249)));
    L = __fsub_rn(__fmul_rn(116.0f, fy), 16.0f);
    A = __fmul_rn(500.0f, __fsub_rn(fx, fy));
    Bo = __fmul_rn(200.0f, __fsub_rn(fy, fz));
}

/* The colour-converted pixels under a 64 x 8 block of patches with top-left patch (x0, y0), as
   3 planes of RH x RWP floats; the block also writes the RGBA copy of the pixels it owns. */
__device__ __forceinline__ void stage_pix(float *pix, const float *__restrict__ rgb, int h, int w, int convert,
                                          float4 *__restrict__ rgba, int eh, int ew, int x0, int y0) {
    const int tid = threadIdx.x;
    const bool last_col = x0 + TW >= ew, last_row = y0 + TH >= eh;
    const int own_x1 = last_col ? w : x0 + TW, own_y1 = last_row ? h : y0 + TH;
    for (int i = tid; i < RH * RW; i += NT) {
        int r = i / RW, c = i % RW;
        int gy = y0 + r, gx = x0 + c;
        float R = 0.f, G = 0.f, B = 0.f;
        if (gy < h && gx < w) {
            const float *p = rgb + ((size_t) gy * w + gx) * 3;
            R = __ldg(p); G = __ldg(p + 1); B = __ldg(p + 2);
            if (rgba && gy < own_y1 && gx < own_x1) rgba[(size_t) gy * w + gx] = make_float4(R, G, B, 0.f);
        }
        float Y = R, U = G, V = B;
        if (convert == PT_COLOR_YUV) yuv_exact(R, G, B, Y, U, V);
        else if (convert == PT_COLOR_LAB) lab_exact(R, G, B, Y, U, V);
        pix[(0 * RH + r) * RWP + c] = Y;
        pix[(1 * RH + r) * RWP + c] = U;
        pix[(2 * RH + r) * RWP + c] = V;
    }
}

/* A patch's descriptor: its table entry (CELLS) and / or its store record (desc set). */
template<bool CELLS>
__device__ __forceinline__ void emit_patch(const float (&out)[PT_DESC_MAX], size_t p, const CellPlan *cp, int *tcand,
                                           float *desc, int ds) {
    if (CELLS) {
        long long cell = 0;
#pragma unroll
        for (int d = 0; d < PT_DESC_MAX; d++)
            if (d < cp->G) cell += (long long) pt_get_bin(cp->min_val[d], cp->range[d], cp->to_bin + d * PT_NMAP, out[d]) * cp->stride[d];
        tcand[p] = __ldg(cp->table + cell);
    }
    if (desc == nullptr) return;
    float4 *dst = reinterpret_cast<float4 *>(desc + p * ds);
#pragma unroll
    for (int q = 0; q < PT_DESC_MAX / 4; q++)
        if (q < ds / 4) dst[q] = make_float4(out[4 * q], out[4 * q + 1], out[4 * q + 2], out[4 * q + 3]);
}

/* One 64 x 8 block of patches with top-left patch (x0, y0).  With CELLS the table entry of each
   patch's cell is written to cp.tcand (and the descriptor only where desc is set). */
template<bool CELLS = false>
__device__ __forceinline__ void desc_tile(const DescPlan &c_plan, float *smem, const float *__restrict__ rgb, int h, int w,
                                          int convert, float4 *__restrict__ rgba, float *__restrict__ desc, int ds, int eh,
                                          int ew, int x0, int y0, const CellPlan *cp = nullptr, int *tcand = nullptr) {
    float *pix = smem;                               /* 3 planes x RH x RWP */
    float *hs = smem + 3 * RH * RWP;                 /* ncombo x RH x TW */
    const int tid = threadIdx.x;
    stage_pix(pix, rgb, h, w, convert, rgba, eh, ew, x0, y0);
    __syncthreads();

    /* horizontal filters: each item is 4 consecutive outputs of one row, read as a 12-float window
       (three 16-byte shared loads) and summed tap by tap in the filter's order */
    const int ncombo = c_plan.ncombo;
    constexpr int HQ = TW / 4;                         /* 4-output items per row */
    for (int m = 0; m < ncombo; m++) {                /* one filter at a time: its signs stay in registers */
        float sg[8];
#pragma unroll
        for (int b = 0; b < 8; b++) sg[b] = c_plan.combo_hf[m][b];
        const float *plane = pix + c_plan.combo_plane[m] * RH * RWP;
        float *dst = hs + m * RH * TW;
        for (int i = tid; i < RH * HQ; i += NT) {
            const int r = i / HQ, j0 = (i % HQ) * 4;
            const float4 *row = reinterpret_cast<const float4 *>(plane + r * RWP + j0);
            const float4 u0 = row[0], u1 = row[1], u2 = row[2];
            const float x[11] = {u0.x, u0.y, u0.z, u0.w, u1.x, u1.y, u1.z, u1.w, u2.x, u2.y, u2.z};
            float o[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                float acc = 0.f;
#pragma unroll
                for (int b = 0; b < 8; b++) acc = __fmaf_rn(sg[b], x[q + b], acc);
                o[q] = acc;
            }
            *reinterpret_cast<float4 *>(dst + r * TW + j0) = make_float4(o[0], o[1], o[2], o[3]);
        }
    }
    __syncthreads();

    /* vertical filters: each thread takes two vertically adjacent patches of one column and reads
       the 9 filtered rows under them once per channel */
    const int nd = c_plan.nd;
    for (int i = tid; i < TW * (TH / 2); i += NT) {
        const int pj = i % TW, pi = 2 * (i / TW);
        const int px = x0 + pj, py = y0 + pi;
        if (px >= ew || py >= eh || (!CELLS && desc == nullptr)) continue;
        const bool two = py + 1 < eh;
        float out0[PT_DESC_MAX], out1[PT_DESC_MAX];
#pragma unroll
        for (int c = 0; c < PT_DESC_MAX; c++) {
            out0[c] = out1[c] = 0.f;
            if (c < nd) {
                const float *col = hs + (c_plan.ch_combo[c] * RH + pi) * TW + pj;
                float y[9];
#pragma unroll
                for (int a = 0; a < 9; a++) y[a] = col[a * TW];
                float s0 = 0.f, s1 = 0.f;
#pragma unroll
                for (int a = 0; a < 8; a++) {
                    s0 = __fmaf_rn(c_plan.ch_vf[c][a], y[a], s0);
                    s1 = __fmaf_rn(c_plan.ch_vf[c][a], y[a + 1], s1);
                }
                out0[c] = s0;
                out1[c] = s1;
            }
        }
        emit_patch<CELLS>(out0, (size_t) py * ew + px, cp, tcand, desc, ds);
        if (two) emit_patch<CELLS>(out1, (size_t) (py + 1) * ew + px, cp, tcand, desc, ds);
    }
}

/* Four CTAs per SM (64 registers; shared memory sized to the plan's filters): the kernel is
   issue-bound and the extra warps fill the barrier gaps (0.105 -> 0.093 ms at 1080p). */
__global__ void __launch_bounds__(NT, 4)
k_descriptor(const DescPlan c_plan, const float *__restrict__ rgb, int h, int w, int convert,
             float4 *__restrict__ rgba, float *__restrict__ desc, int ds, int eh, int ew, int ty0) {
    extern __shared__ __align__(16) float smem[];
    desc_tile(c_plan, smem, rgb, h, w, convert, rgba, desc, ds, eh, ew, blockIdx.x * TW, (blockIdx.y + ty0) * TH);
}

__global__ void __launch_bounds__(NT, 4)
k_descriptor_cells(const DescPlan c_plan, const CellPlan cp, const float *__restrict__ rgb, int h, int w, int convert,
                   float4 *__restrict__ rgba, int eh, int ew, int ty0) {
    extern __shared__ __align__(16) float smem[];
    desc_tile<true>(c_plan, smem, rgb, h, w, convert, rgba, nullptr, 0, eh, ew, blockIdx.x * TW, (blockIdx.y + ty0) * TH, &cp,
                    cp.tcand);
}

/* Persistent descriptor pass over the 64 x 8 tiles of every image of a batch (images, RGBA
   copies and descriptors concatenated), the tiles handed out by a work counter; with CELLS the
   table entries of the patches' cells are written instead of the descriptors. */
template<bool CELLS>
__global__ void __launch_bounds__(NT, 4)
k_descriptor_batch(const DescPlan c_plan, const CellPlan cp, const PtBatchImage *__restrict__ imgs, int n, long long ntiles,
                   const float *__restrict__ rgb, int convert, float4 *__restrict__ rgba, float *__restrict__ desc, int ds,
                   unsigned long long *work) {
    extern __shared__ __align__(16) float smem[];
    __shared__ long long s_next;
    /* tiles go out one at a time; a CTA claims its next tile when it starts the current one and
       reads the claim after it, so the counter's round trip overlaps the work */
    if (threadIdx.x == 0) s_next = (long long) atomicAdd(work, 1ull);
    __syncthreads();
    long long t = s_next;
    while (t < ntiles) {
        long long claim = 0;
        if (threadIdx.x == 0) claim = (long long) atomicAdd(work, 1ull);
        int lo = 0, hi = n - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(&imgs[mid].tile_off) <= t) lo = mid; else hi = mid - 1;
        }
        const PtBatchImage &g = imgs[lo];
        const long long lt = t - g.tile_off;
        const int tpr = (g.ew + TW - 1) / TW;
        desc_tile<CELLS>(c_plan, smem, rgb + 3 * g.pix_off, g.h, g.w, convert, rgba ? rgba + g.pix_off : nullptr,
                         CELLS ? nullptr : desc + g.patch_off * ds, ds, g.eh, g.ew, (int) (lt % tpr) * TW, (int) (lt / tpr) * TH,
                         &cp, CELLS ? cp.tcand + g.patch_off : nullptr);
        __syncthreads();                                 /* the next tile reuses the shared memory and s_next */
        if (threadIdx.x == 0) s_next = claim;
        __syncthreads();
        t = s_next;
    }
}

/* -dim_algo pca projection (apply_patch_pca, patch_pca.h:60-110): descriptor channel k of a
   patch = sum over the patch's 192 values v_j of (v_j - mean_j) * basis[k][j], accumulated in j
   order with separately rounded products and sums.  Value j = (dy * 8 + dx) * 3 + c is float
   dx + c of the interleaved patch row dy, as the reference reads it (its row pointer advances by
   dx floats, patch_pca.h:87-96): pixel (dx + c) / 3 of the first four, channel (dx + c) % 3.
   Each thread projects two patches of the block (rows pi and pi + 4) so that every basis load serves both;
   all lanes read the same basis word, a broadcast. */
__global__ void __launch_bounds__(NT)
k_pca(const float *__restrict__ rgb, int h, int w, int convert, float4 *__restrict__ rgba,
      const float *__restrict__ mean, const float *__restrict__ basis, int ncomp, float *__restrict__ desc, int ds,
      int eh, int ew) {
    __shared__ float pix[3 * RH * RWP];
    const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
    stage_pix(pix, rgb, h, w, convert, rgba, eh, ew, x0, y0);
    __syncthreads();
    const int pj = threadIdx.x % TW, pi = threadIdx.x / TW;        /* pi in 0..3 */
    float acc[2][PT_DESC_MAX];
#pragma unroll
    for (int k = 0; k < PT_DESC_MAX; k++) acc[0][k] = acc[1][k] = 0.f;
#pragma unroll 1
    for (int dy = 0; dy < 8; dy++)
#pragma unroll 1
        for (int dx = 0; dx < 8; dx++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const int j = (dy * 8 + dx) * 3 + c;
                const float mj = __ldg(mean + j);
                const int f = dx + c, fc = f % 3, fx = f / 3;        /* float f of the row: pixel fx, channel fc */
                const float d0 = __fsub_rn(pix[(fc * RH + pi + dy) * RWP + pj + fx], mj);
                const float d1 = __fsub_rn(pix[(fc * RH + pi + 4 + dy) * RWP + pj + fx], mj);
#pragma unroll
                for (int k = 0; k < PT_DESC_MAX; k++) {
                    if (k < ncomp) {
                        const float bk = __ldg(basis + k * PT_PCA_DIM + j);
                        acc[0][k] = __fadd_rn(acc[0][k], __fmul_rn(d0, bk));
                        acc[1][k] = __fadd_rn(acc[1][k], __fmul_rn(d1, bk));
                    }
                }
            }
#pragma unroll
    for (int u = 0; u < 2; u++) {
        const int py = y0 + pi + 4 * u, px = x0 + pj;
        if (py >= eh || px >= ew) continue;
        float *o = desc + ((size_t) py * ew + px) * ds;
#pragma unroll
        for (int k = 0; k < PT_DESC_MAX; k++)
            if (k < ds) o[k] = k < ncomp ? acc[u][k] : 0.f;
    }
}

}  // namespace

/* Builds the per-channel plan for n = ndims - 2*nchroma kernels (gck.h channel map,
   gck.py:386-389): kernel k < nchroma has Y, U, V channels at 3k..3k+2, the others one Y
   channel at 3*nchroma + (k - nchroma). */
static pt_status make_plan(int ndims, int nchroma, DescPlan &plan) {
    int n = ndims - 2 * nchroma;
    if (ndims < 1 || ndims > PT_DESC_MAX || nchroma < 0 || nchroma > 3 || n < 1 || n > 64 || n < nchroma)
        return pt_fail(PT_UNSUPPORTED, "descriptor: ndims=%d nchroma=%d not supported on the GPU path (ndims <= %d)",
                       ndims, nchroma, PT_DESC_MAX);
    memset(&plan, 0, sizeof(plan));
    plan.nd = ndims;
    auto combo_of = [&](int plane, int k) {
        for (int m = 0; m < plan.ncombo; m++) {
            bool same = plan.combo_plane[m] == plane;
            for (int b = 0; b < 8 && same; b++) same = plan.combo_h[m][b] == PT_WH_H[k][b];
            if (same) return m;
        }
        int m = plan.ncombo++;
        plan.combo_plane[m] = plane;
        for (int b = 0; b < 8; b++) { plan.combo_h[m][b] = PT_WH_H[k][b]; plan.combo_hf[m][b] = PT_WH_H[k][b] > 0 ? 1.f : -1.f; }
        return m;
    };
    for (int k = 0; k < n; k++) {
        int nc = k < nchroma ? 3 : 1;
        int c0 = k < nchroma ? 3 * k : 3 * nchroma + (k - nchroma);
        for (int c = 0; c < nc; c++) {
            int ch = c0 + c;
            plan.ch_combo[ch] = combo_of(c, k);
            for (int a = 0; a < 8; a++) { plan.ch_v[ch][a] = PT_WH_V[k][a]; plan.ch_vf[ch][a] = PT_WH_V[k][a] > 0 ? 1.f : -1.f; }
        }
    }
    return PT_OK;
}

pt_status pt_descriptor_check(int ndims, int nchroma) {
    DescPlan plan;
    return make_plan(ndims, nchroma, plan);
}

size_t pt_descriptor_smem(int ndims) {
    (void) ndims;
    return sizeof(float) * (3 * RH * RWP + PT_DESC_MAX * RH * TW);
}

pt_status pt_launch_descriptor(int ndims, int nchroma, const float *rgb, int h, int w, int convert, float4 *rgba,
                               float *desc, int ds, cudaStream_t st) {
    return pt_launch_descriptor_rows(ndims, nchroma, rgb, h, w, convert, rgba, desc, ds, 0, (h - 7 + TH - 1) / TH, st);
}

pt_status pt_launch_descriptor_rows(int ndims, int nchroma, const float *rgb, int h, int w, int convert, float4 *rgba,
                                    float *desc, int ds, int trow0, int trows, cudaStream_t st) {
    if (convert == PT_COLOR_LAB) PT_TRY(pt_lab_tables_ready());
    int eh = h - 7, ew = w - 7;
    DescPlan plan;
    PT_TRY(make_plan(ndims, nchroma, plan));
    if (eh < 1 || ew < 1) return pt_fail(PT_BAD_ARG, "image %dx%d is smaller than one 8x8 patch", w, h);
    static bool attr = false;
    size_t smem = sizeof(float) * (3 * RH * RWP + plan.ncombo * RH * TW);
    if (!attr) {
        PT_CUDA(cudaFuncSetAttribute(k_descriptor, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) pt_descriptor_smem(0)));
        attr = true;
    }
    const int ntr = (eh + TH - 1) / TH;
    if (trow0 < 0 || trows < 1 || trow0 + trows > ntr)
        return pt_fail(PT_BAD_ARG, "descriptor tile rows [%d, %d) outside 0..%d", trow0, trow0 + trows, ntr);
    dim3 grid((ew + TW - 1) / TW, trows);
    k_descriptor<<<grid, NT, smem, st>>>(plan, rgb, h, w, convert, rgba, desc, ds, eh, ew, trow0);
    PT_LAUNCHED();
    return PT_OK;
}

pt_status pt_launch_descriptor_cells(int ndims, int nchroma, const float *rgb, int h, int w, int convert, float4 *rgba,
                                     const PtBins &bins, const int *to_bin, const int *table, int *tcand, int trow0,
                                     int trows, cudaStream_t st) {
    if (convert == PT_COLOR_LAB) PT_TRY(pt_lab_tables_ready());
    int eh = h - 7, ew = w - 7;
    DescPlan plan;
    PT_TRY(make_plan(ndims, nchroma, plan));
    if (eh < 1 || ew < 1) return pt_fail(PT_BAD_ARG, "image %dx%d is smaller than one 8x8 patch", w, h);
    if (bins.G < 1 || bins.G > ndims) return pt_fail(PT_BAD_ARG, "grid dims %d outside 1..%d", bins.G, ndims);
    CellPlan cp;
    memset(&cp, 0, sizeof(cp));
    cp.G = bins.G;
    for (int d = 0; d < bins.G; d++) { cp.min_val[d] = bins.min_val[d]; cp.range[d] = bins.range[d]; cp.stride[d] = bins.stride[d]; }
    cp.to_bin = to_bin;
    cp.table = table;
    cp.tcand = tcand;
    static bool attr = false;
    size_t smem = sizeof(float) * (3 * RH * RWP + plan.ncombo * RH * TW);
    if (!attr) {
        PT_CUDA(cudaFuncSetAttribute(k_descriptor_cells, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) pt_descriptor_smem(0)));
        attr = true;
    }
    const int ntr = (eh + TH - 1) / TH;
    if (trow0 < 0 || trows < 1 || trow0 + trows > ntr)
        return pt_fail(PT_BAD_ARG, "descriptor tile rows [%d, %d) outside 0..%d", trow0, trow0 + trows, ntr);
    dim3 grid((ew + TW - 1) / TW, trows);
    k_descriptor_cells<<<grid, NT, smem, st>>>(plan, cp, rgb, h, w, convert, rgba, eh, ew, trow0);
    PT_LAUNCHED();
    return PT_OK;
}

namespace {

template<bool CELLS>
pt_status launch_descriptor_batch(int ndims, int nchroma, const CellPlan &cp, const PtBatchImage *imgs, int n,
                                  long long ntiles, const float *rgb, int convert, float4 *rgba, float *desc, int ds,
                                  unsigned long long *work, cudaStream_t st) {
    if (convert == PT_COLOR_LAB) PT_TRY(pt_lab_tables_ready());
    DescPlan plan;
    PT_TRY(make_plan(ndims, nchroma, plan));
    if (ntiles <= 0) return PT_OK;
    /* shared memory for this plan's filters only, as the single-image pass sizes it */
    const size_t smem = sizeof(float) * (3 * RH * RWP + plan.ncombo * RH * TW);
    static int nsm = 0;
    static size_t per_smem[PT_DESC_MAX + 1] = {};
    static int per_n[PT_DESC_MAX + 1] = {};
    if (!nsm) {
        int dev = 0;
        PT_CUDA(cudaGetDevice(&dev));
        PT_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        PT_CUDA(cudaFuncSetAttribute(k_descriptor_batch<CELLS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int) pt_descriptor_smem(0)));
    }
    const int slot = plan.ncombo;
    if (per_smem[slot] != smem) {
        int per = 0;
        PT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_descriptor_batch<CELLS>, NT, smem));
        per_n[slot] = per < 1 ? 1 : per;
        per_smem[slot] = smem;
    }
    const long long g = (long long) per_n[slot] * nsm;
    PT_CUDA(cudaMemsetAsync(work, 0, sizeof(unsigned long long), st));
    k_descriptor_batch<CELLS><<<(unsigned) (ntiles < g ? ntiles : g), NT, smem, st>>>(plan, cp, imgs, n, ntiles, rgb, convert,
                                                                                     rgba, desc, ds, work);
    PT_LAUNCHED();
    return PT_OK;
}

}  // namespace

pt_status pt_launch_descriptor_cells_batch(int ndims, int nchroma, const PtBatchImage *imgs, int n, long long ntiles,
                                           const float *rgb, int convert, float4 *rgba, const PtBins &bins, const int *to_bin,
                                           const int *table, int *tcand, unsigned long long *work, cudaStream_t st) {
    if (bins.G < 1 || bins.G > ndims) return pt_fail(PT_BAD_ARG, "grid dims %d outside 1..%d", bins.G, ndims);
    CellPlan cp;
    memset(&cp, 0, sizeof(cp));
    cp.G = bins.G;
    for (int d = 0; d < bins.G; d++) { cp.min_val[d] = bins.min_val[d]; cp.range[d] = bins.range[d]; cp.stride[d] = bins.stride[d]; }
    cp.to_bin = to_bin;
    cp.table = table;
    cp.tcand = tcand;
    return launch_descriptor_batch<true>(ndims, nchroma, cp, imgs, n, ntiles, rgb, convert, rgba, nullptr, 0, work, st);
}

namespace {

/* get_padded_descriptor in descriptor mode (patchtable.h:2498-2507): an unpadded input sits at
   offset 7 of a zero-padded (H+14) x (W+14) image, a padded input is that image already, and the
   patch at (x, y) is pixel (x+7, y+7) of it.  With 3 dimensions slot 3 holds the next pixel's
   first channel, the value the reference's four-float load picks up (pt_descdist.cuh). */
__global__ void k_desc_input(const float *__restrict__ in, int H, int W, int nd, int padded, int ew, int eh,
                             float *desc, int ds) {
    const long long p = blockIdx.x * (long long) NT + threadIdx.x;
    if (p >= (long long) ew * eh) return;
    const int x = (int) (p % ew), y = (int) (p / ew);
    const int off = padded ? 0 : 7;
    auto at = [&](int py, int px, int c) -> float {
        const int iy = py - off, ix = px - off;
        return (iy >= 0 && iy < H && ix >= 0 && ix < W) ? __ldg(in + ((size_t) iy * W + ix) * nd + c) : 0.0f;
    };
    float *o = desc + p * ds;
    for (int c = 0; c < ds; c++) {
        float v = 0.0f;
        if (c < nd) v = at(y + 7, x + 7, c);
        else if (nd == 3 && c == 3) v = at(y + 7, x + 8, 0);
        o[c] = v;
    }
}

}  // namespace

pt_status pt_launch_descriptor_input(const float *in, int H, int W, int nd, int padded, float *desc, int ds,
                                     cudaStream_t st) {
    const int ew = padded ? W - 14 : W, eh = padded ? H - 14 : H;
    if (ew < 1 || eh < 1) return pt_fail(PT_BAD_ARG, "descriptor image %dx%d has no patches", W, H);
    if (nd < 3 || nd > ds || ds > PT_DESC_MAX) return pt_fail(PT_UNSUPPORTED, "descriptor dimensions %d outside 3..%d", nd, PT_DESC_MAX);
    const long long P = (long long) ew * eh;
    k_desc_input<<<(unsigned) ((P + NT - 1) / NT), NT, 0, st>>>(in, H, W, nd, padded, ew, eh, desc, ds);
    PT_LAUNCHED();
    return PT_OK;
}

pt_status pt_launch_pca(const float *rgb, int h, int w, int convert, float4 *rgba, const float *mean, const float *basis,
                        int ncomp, float *desc, int ds, cudaStream_t st) {
    if (convert == PT_COLOR_LAB) PT_TRY(pt_lab_tables_ready());
    const int ew = w - 7, eh = h - 7;
    if (ew < 1 || eh < 1) return pt_fail(PT_BAD_ARG, "image %dx%d is smaller than one 8x8 patch", w, h);
    if (ncomp < 1 || ncomp > ds || ds > PT_DESC_MAX) return pt_fail(PT_UNSUPPORTED, "PCA with %d components", ncomp);
    dim3 grid((ew + TW - 1) / TW, (eh + TH - 1) / TH);
    k_pca<<<grid, NT, 0, st>>>(rgb, h, w, convert, rgba, mean, basis, ncomp, desc, ds, eh, ew);
    PT_LAUNCHED();
    return PT_OK;
}

/* Fills the PowTable stand-ins of -colorspace lab on the current device (once per device). */
pt_status pt_lab_tables_ready() {
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    PT_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 64 && done[dev]) return PT_OK;
    float tab[2][PT_LAB_N];
    pt_lab_pow_tables(tab);
    PT_CUDA(cudaMemcpyToSymbol(g_lab_pow, tab, sizeof(tab)));
    if (dev < 64) done[dev] = true;
    return PT_OK;
}
