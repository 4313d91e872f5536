/* Descriptor-mode patch distance: patch_dist_approx<float, TABLE_NCHANNELS> with TABLE_SSE
   (patchtable/patchtable.h:376-437).

   The first four squared differences form four lanes.  With exactly 8, 12 or 16 dimensions every
   further block of four is added lane-wise and the lanes are summed 0+1+2+3 at the end; with any
   other count the four lanes are summed first and the remaining dimensions are added one by one.
   Every operation is rounded on its own (no fused multiply-add), as in the SSE code.

   Vectors hold up to 16 floats, padded with the layout of the table's descriptor store: 8 floats
   per patch for up to 8 dimensions, 16 beyond.  With 3 dimensions the reference still loads four
   floats -- its fourth lane reads the next pixel's first channel -- so the descriptor store keeps
   that value in slot 3 and the lane sees it here as well. */
#pragma once

#include <cuda_runtime.h>

__device__ __forceinline__ float pt_sqd(float a, float b) {
    const float t = __fsub_rn(a, b);
    return __fmul_rn(t, t);
}

/* a: the query vector in registers (slots >= the store width are never read); b: 16-byte aligned
   store entry; nd: descriptor dimensions (3..16). */
__device__ __forceinline__ float pt_desc_dist(const float4 (&a)[4], const float4 *__restrict__ b, int nd) {
    const float4 b0 = __ldg(b);
    float l0 = pt_sqd(a[0].x, b0.x), l1 = pt_sqd(a[0].y, b0.y), l2 = pt_sqd(a[0].z, b0.z), l3 = pt_sqd(a[0].w, b0.w);
    if (nd == 8 || nd == 12 || nd == 16) {
#pragma unroll
        for (int n = 1; n < 4; n++) {
            if (4 * n >= nd) break;
            const float4 bn = __ldg(b + n);
            l0 = __fadd_rn(l0, pt_sqd(a[n].x, bn.x));
            l1 = __fadd_rn(l1, pt_sqd(a[n].y, bn.y));
            l2 = __fadd_rn(l2, pt_sqd(a[n].z, bn.z));
            l3 = __fadd_rn(l3, pt_sqd(a[n].w, bn.w));
        }
        return __fadd_rn(__fadd_rn(__fadd_rn(l0, l1), l2), l3);
    }
    float s = __fadd_rn(__fadd_rn(__fadd_rn(l0, l1), l2), l3);
#pragma unroll
    for (int n = 1; n < 4; n++) {
        if (4 * n >= nd) break;
        const float4 bn = __ldg(b + n);
        s = __fadd_rn(s, pt_sqd(a[n].x, bn.x));
        if (4 * n + 1 < nd) s = __fadd_rn(s, pt_sqd(a[n].y, bn.y));
        if (4 * n + 2 < nd) s = __fadd_rn(s, pt_sqd(a[n].z, bn.z));
        if (4 * n + 3 < nd) s = __fadd_rn(s, pt_sqd(a[n].w, bn.w));
    }
    return s;
}

/* Loads a store entry of ds floats (8 or 16) into registers. */
__device__ __forceinline__ void pt_desc_load(const float4 *__restrict__ v, int ds, float4 (&a)[4]) {
    a[0] = __ldg(v);
    a[1] = __ldg(v + 1);
    if (ds > 8) { a[2] = __ldg(v + 2); a[3] = __ldg(v + 3); }
    else a[2] = a[3] = make_float4(0.f, 0.f, 0.f, 0.f);
}
