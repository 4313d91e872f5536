/* Internal declarations shared by the host code and the CUDA kernels of patchtable_b200. */
#pragma once

#include <cstdint>
#include <cstdarg>
#include <vector>
#include <string>

#include "patchtable_b200.h"

#ifdef __CUDACC__
#include <cuda_runtime.h>
#endif

#define PT_NMAP 16384                      /* PATCH_PARTITION_NMAP, patchtable.h:216 */
#define PT_UNUSED ((1 << 30) - 1)          /* TABLE_UNUSED, patchtable.h:109-112 */
#define PT_DIST_INF 100000.0               /* DIST_INFINITY, patchtable.h:173 */
#define PT_PW 8                            /* patch width (TABLE_PATCH_W, patchtable.h:48) */
#define PT_DESC_MAX 16                     /* descriptor dims handled by the GPU path */

/* XY_TO_INT / INT_TO_X / INT_TO_Y, patchtable.h:163-165. */
#ifdef __CUDACC__
#define PT_HD __host__ __device__ __forceinline__
#else
#define PT_HD inline
#endif
PT_HD int pt_xy(int x, int y) { return x | (y << 16); }
PT_HD int pt_x(int v) { return v & 65535; }
PT_HD int pt_y(int v) { return v >> 16; }

/* Records an error message for pt_last_error() and returns the status. */
pt_status pt_fail(pt_status s, const char *fmt, ...);
/* Counts device kernel launches issued by the library (pt_kernel_launch_count). */
void pt_count_launches(int n);
/* Polls after which a device-side wait gives up (pt_set_spin_limit). */
long long pt_spin_limit();
/* Device-allocation accounting of DevBuf (pt_set_device_alloc_limit): admits `bytes` more or
   refuses when the library's live device allocations would exceed the limit. */
bool pt_alloc_admit(size_t bytes);
void pt_alloc_release(size_t bytes);

#define PT_TRY(expr) do { pt_status _s = (expr); if (_s != PT_OK) return _s; } while (0)

#ifdef __CUDACC__
#define PT_CUDA(call) do { cudaError_t _e = (call); if (_e != cudaSuccess) \
    return pt_fail(_e == cudaErrorMemoryAllocation ? PT_OOM : PT_CUDA_ERR, "%s: %s (%s:%d)", #call, \
                   cudaGetErrorString(_e), __FILE__, __LINE__); } while (0)
#define PT_LAUNCHED() do { pt_count_launches(1); cudaError_t _e = cudaGetLastError(); if (_e != cudaSuccess) \
    return pt_fail(PT_CUDA_ERR, "kernel launch: %s (%s:%d)", cudaGetErrorString(_e), __FILE__, __LINE__); } while (0)
#endif

/* One grid dimension's partition, PatchPartition1D (patchtable.h:1131-1326). */
struct PtPartition {
    std::vector<int> to_bin;
    std::vector<float> centers, lsizes, rsizes;
    float min_val = 0, max_val = 0, range = 0;
    int nslices = 0;
};

#ifdef __CUDACC__
/* A device buffer owned by the table; freed with cudaFree. */
template<class T> struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    DevBuf() {}
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    cudaError_t reserve(size_t count) {
        if (count <= n && p) return cudaSuccess;
        release();
        const size_t bytes = sizeof(T) * (count ? count : 1);
        if (!pt_alloc_admit(bytes)) return cudaErrorMemoryAllocation;
        cudaError_t e = cudaMalloc((void **) &p, bytes);
        if (e == cudaSuccess) { n = count; held = bytes; }
        else { p = nullptr; pt_alloc_release(bytes); }
        return e;
    }
    void release() {
        if (p) { cudaFree(p); pt_alloc_release(held); }
        p = nullptr; n = 0; held = 0;
    }
private:
    size_t held = 0;
};

/* Page-locked host memory owned by a table (download staging); freed with cudaFreeHost. */
template<class T> struct PinnedBuf {
    T *p = nullptr;
    size_t n = 0;
    PinnedBuf() {}
    PinnedBuf(const PinnedBuf &) = delete;
    PinnedBuf &operator=(const PinnedBuf &) = delete;
    ~PinnedBuf() { if (p) cudaFreeHost(p); }
    cudaError_t reserve(size_t count) {
        if (count <= n && p) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr; n = 0;
        cudaError_t e = cudaMallocHost((void **) &p, sizeof(T) * (count ? count : 1));
        if (e == cudaSuccess) n = count;
        else p = nullptr;
        return e;
    }
};
#endif

/* pt_host.cpp: ann[3i .. 3i+2] = (x, y, dist) of pos[i] / dist[i] for i < n, in float64, split
   across the library's host threads (pt_set_host_threads). */
void pt_expand_nnf(const int *pos, const float *dist, long long n, double *ann);
/* false when pt_set_host_threads(n < 0) asked for float64 records written on the GPU instead. */
bool pt_host_widen();
/* dst[0 .. n) = src[0 .. n), split across the same host threads (staging a pageable query image
   in page-locked memory). */
void pt_host_copy(float *dst, const float *src, size_t n);
