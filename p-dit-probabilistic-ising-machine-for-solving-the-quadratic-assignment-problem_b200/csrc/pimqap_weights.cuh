// pimqap_weights.cuh - the binary32 weight function of the one-shot update rule.
#pragma once

#include <cuda_runtime.h>

namespace pimqap {

// 2^x in binary32 for x <= 0: Cody-Waite reduction x = k + f (k = rint(x), |f| <= 1/2, f
// exact), the degree-7 Taylor polynomial of 2^f = e^(f ln 2) (coefficients (ln 2)^m / m!
// rounded to binary32) by Horner's rule with fused multiply-adds, then scaling by 2^k (two
// multiplies below 2^-126, so a subnormal result is rounded once).  Each step is a single
// correctly rounded IEEE operation with no contraction left to the compiler, so a C
// restatement with fmaf returns the same bits.  Error below 1 ulp over the normal range;
// 0 for x <= -150.
__device__ __forceinline__ float exp2f_neg(float x) {
    if (!(x > -150.0f)) return 0.0f;
    x = fminf(x, 0.0f);
    const float k = rintf(x);
    const float f = __fsub_rn(x, k);
    float p = 0x1.ffcbfcp-17f;
    p = __fmaf_rn(p, f, 0x1.430912p-13f);
    p = __fmaf_rn(p, f, 0x1.5d87fep-10f);
    p = __fmaf_rn(p, f, 0x1.3b2ab6p-7f);
    p = __fmaf_rn(p, f, 0x1.c6b08ep-5f);
    p = __fmaf_rn(p, f, 0x1.ebfbe0p-3f);
    p = __fmaf_rn(p, f, 0x1.62e430p-1f);
    p = __fmaf_rn(p, f, 1.0f);
    const int ki = (int)k;
    if (ki >= -126) return __fmul_rn(p, __int_as_float((ki + 127) << 23));
    return __fmul_rn(__fmul_rn(p, __int_as_float((ki + 191) << 23)), 0x1p-64f);
}

// The threshold of a one-shot proposal: word 0 of the update's Philox block as an odd
// multiple of 2^-24, in (0, 1).
__device__ __forceinline__ float oneshot_uniform(unsigned int w0) {
    return __fmul_rn(__uint2float_rn(((w0 >> 9) << 1) | 1u), 0x1p-24f);
}

}  // namespace pimqap
