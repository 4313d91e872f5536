/* Bin lookup shared by the table build, the query and the proposal network. */
#pragma once

#include <climits>
#include <cuda_runtime.h>

#include "pt_internal.h"

/* float -> int conversion with x86 cvttss2si semantics (NaN and out-of-range give INT_MIN), as
   the reference's `int idx = (v-min_val)*(NMAP-1)/range` compiles on x86-64. */
__device__ __forceinline__ int pt_cvtt_x86(float f) {
    if (!(f >= -2147483648.0f && f < 2147483648.0f)) return INT_MIN;
    return __float2int_rz(f);
}

/* PatchPartition1D::get_bin, patchtable.h:1298-1325, bit-exact (no fused operations); to_bin_d is
   the dimension's PT_NMAP-entry lookup table. */
__device__ __forceinline__ int pt_get_bin(float min_val, float range, const int *__restrict__ to_bin_d, float v) {
    float t = __fdiv_rn(__fmul_rn(__fsub_rn(v, min_val), (float) (PT_NMAP - 1)), range);
    int idx = pt_cvtt_x86(t);
    if (idx < 0) idx = 0;
    else if (idx >= PT_NMAP) idx = PT_NMAP - 1;
    return __ldg(to_bin_d + idx);
}
