/* Zero-allocation query entry point: pt_table_lookup_device_noalloc.

   Some callers of this library must not allocate device memory while they run queries: a video
   or image-analogy frame loop with a fixed per-frame latency budget (cudaMalloc and cudaFree
   synchronise the whole device and can stall for milliseconds), or an application that hands
   the GPU's memory to its own allocator at start-up, so that any further cudaMalloc from a
   library fails.  For them this entry point runs the same query kernels as
   pt_table_lookup_device but takes every intermediate buffer from one file-scope device array,
   so a call allocates nothing.

   Limits and behaviour:
     * query images of at most PT_NOALLOC_MAX_PIXELS (262144) pixels, e.g. 512 x 512, and tables
       with ndims <= 8; larger requests fail with PT_BAD_ARG / PT_UNSUPPORTED;
     * the array costs 20 MiB of device memory on every GPU that loads the library, held until
       the process exits;
     * all calls share the array: calls that overlap on the GPU (different streams, threads or
       tables at the same time) race on it and must be serialised by the caller;
     * the first call on a device resolves the array's device address (cudaGetSymbolAddress);
       make that first call before any stream capture.
   The query state is rewritten from scratch on every call, so the contents left by the previous
   call never reach the result. */
#include <cuda_runtime.h>

#include <mutex>

#include "patchtable_b200.h"
#include "pt_internal.h"
#include "pt_kernels.h"

namespace {

constexpr size_t kMaxPixels = PT_NOALLOC_MAX_PIXELS;
/* per pixel: RGBA copy (16 B) + descriptor record (32 B) + table candidate (4 B)
   + four position buffers (16 B) + three distance buffers (12 B) */
constexpr size_t kBytesPerPixel = 16 + 32 + 4 + 16 + 12;
constexpr size_t kScratchBytes = kMaxPixels * kBytesPerPixel;

static __device__ __align__(256) unsigned char pt_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch[kMaxDevices] = {nullptr};

/* Device address of the scratch array on the current device, resolved once per device. */
pt_status scratch_address(void **out) {
    int dev = 0;
    PT_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return pt_fail(PT_UNSUPPORTED, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, pt_noalloc_scratch);
        if (e != cudaSuccess)
            return pt_fail(PT_CUDA_ERR, "cudaGetSymbolAddress(pt_noalloc_scratch): %s", cudaGetErrorString(e));
        g_scratch[dev] = p;
    }
    *out = g_scratch[dev];
    return PT_OK;
}

}  // namespace

extern "C" pt_status pt_table_lookup_device_noalloc(pt_table *t, const float *d_a, int h, int w, double *d_ann,
                                                    void *stream) {
    if (!t || !d_a || !d_ann) return pt_fail(PT_BAD_ARG, "null argument");
    if (h < 8 || w < 8) return pt_fail(PT_BAD_ARG, "image %dx%d is smaller than one 8x8 patch", w, h);
    if ((long long) h * w > (long long) kMaxPixels)
        return pt_fail(PT_BAD_ARG, "image %dx%d has %lld pixels; the zero-allocation lookup handles at most %lld",
                       w, h, (long long) h * w, (long long) kMaxPixels);
    PtTableView v;
    PT_TRY(pt_table_view(t, &v));
    if (v.ds != 8) return pt_fail(PT_UNSUPPORTED, "the zero-allocation lookup handles ndims <= 8 (table has %d)", v.p.ndims);
    void *base = nullptr;
    PT_TRY(scratch_address(&base));
    cudaStream_t st = (cudaStream_t) stream;
    const pt_params &p = v.p;
    const size_t N = kMaxPixels;
    unsigned char *s = (unsigned char *) base;
    float4 *rgba = (float4 *) s;            s += N * 16;
    float *desc = (float *) s;              s += N * 32;
    int *tcand = (int *) s;                 s += N * 4;
    int *pos0 = (int *) s;                  s += N * 4;
    int *pos1 = (int *) s;                  s += N * 4;
    int *chpos = (int *) s;                 s += N * 4;
    int *kcdone = (int *) s;                s += N * 4;
    float *d0 = (float *) s;                s += N * 4;
    float *d1 = (float *) s;                s += N * 4;
    float *chd = (float *) s;
    int *pos[2] = {pos0, pos1};
    float *dd[2] = {d0, d1};

    long long P = (long long) (h - 7) * (w - 7);
    int n = (int) P;
    PT_TRY(pt_launch_descriptor(p.ndims, p.nchroma, d_a, h, w, pt_color_mode(p), rgba, desc, 8, st));
    PT_TRY(pt_launch_table_candidates(v.bins, desc, 8, P, v.to_bin, v.table, tcand, st));
    QuerySetup qs;
    qs.aw = w; qs.ah = h; qs.bw = v.w; qs.bh = v.h;
    qs.prop_scale = 1.0 / (1 + p.coherence_spatial);
    qs.triangle_factor = p.triangle_factor;
    qs.kcoherence = p.kcoherence;
    qs.kc_try = p.gpu_kc_max;
    qs.kcoherence_step = p.kcoherence_step;
    qs.spatial = p.spatial;
    qs.do_rs = p.do_rs;
    qs.radius = p.query_step + p.prop_dist;
    if (qs.radius > 2) qs.radius = 2;
    qs.b1 = v.b_rgba1;
    qs.pull_max = p.gpu_pull_max;
    qs.tile = p.gpu_tile;
    qs.allowed = v.allowed;
    qs.allowed_index = p.allowed_index;
    qs.stream = st;
    PT_TRY(pt_launch_init(n, pt_xy(v.w - 7 + 1, 0), (float) PT_DIST_INF, pos[0], dd[0], st));
    int passes = pt_default_passes(p);
    int jump = pt_default_jump(p, passes);
    int cur = 0;
    for (int i = 0; i < passes; i++) {
        bool do_table = i == 0 && p.do_table_lookup;
        QuerySetup qi = qs;
        qi.pass = i;
        if (!pt_pass_kcoh(p, i, passes)) qi.kcoherence = 0;
        const int use_done = i > 0 && pt_pass_kcoh(p, i - 1, passes);
        PT_TRY(pt_launch_choose(qi, n, rgba, v.b_rgba, pos[cur], dd[cur], tcand, v.kcoh, do_table, chpos, chd,
                                kcdone, use_done, nullptr, st));
        if (p.do_prop) {
            QuerySetup qp = qs;
            qp.step = pt_pass_step(i, passes, jump);
            PT_TRY(pt_launch_pull(qp, n, rgba, v.b_rgba, pos[cur], dd[cur], chpos, chd, pos[1 - cur], dd[1 - cur],
                                  nullptr, st));
            cur = 1 - cur;
        } else {
            PT_CUDA(cudaMemcpyAsync(pos[cur], chpos, sizeof(int) * n, cudaMemcpyDeviceToDevice, st));
            PT_CUDA(cudaMemcpyAsync(dd[cur], chd, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
        }
    }
    PT_TRY(pt_launch_output(n, pos[cur], dd[cur], d_ann, st));
    return PT_OK;
}
