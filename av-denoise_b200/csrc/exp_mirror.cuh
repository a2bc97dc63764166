// The exponential of the exact NLMeans path and the bilateral prefilter, evaluated with separately
// rounded operations in a fixed order so that a CPU evaluation of the same steps gives the same
// bits. Written from the mathematics:
//   n = rint(x * log2(e)), r = x - n*ln2 by Cody and Waite's two-constant reduction (ln2 split
//   into a 16-bit head, so n*head is exact, and the float nearest the remainder), |r| <= ln2/2;
//   e^r by its degree-7 Taylor polynomial (coefficients 1/k!) in Horner form with fused
//   multiply-adds, which truncates below 0.1 ulp on the reduced range;
//   e^x = e^r * 2^n, the power of two built from its exponent bits.
// x below -87 (a subnormal result) and NaN give 0; x above 88 overflows to +inf once n reaches 128.
// Within 1 ulp of the exponential over the weights' range.
#pragma once

#include <cuda_runtime.h>

namespace avd {

__device__ __forceinline__ float exp_mirror(float x) {
    constexpr float kLog2e = 1.44269502162933349609375f;      // float(log2(e))
    constexpr float kLn2Hi = 0.693145751953125f;              // ln2 to 16 bits
    constexpr float kLn2Lo = 1.428606765330187045037746e-06f;  // float(ln2 - kLn2Hi)
    if (!(x >= -87.0f)) return 0.0f;
    const float n = rintf(__fmul_rn(x, kLog2e));
    float r = __fmaf_rn(n, -kLn2Hi, x);
    r = __fmaf_rn(n, -kLn2Lo, r);
    float p = 1.0f / 5040.0f;
    p = __fmaf_rn(p, r, 1.0f / 720.0f);
    p = __fmaf_rn(p, r, 1.0f / 120.0f);
    p = __fmaf_rn(p, r, 1.0f / 24.0f);
    p = __fmaf_rn(p, r, 1.0f / 6.0f);
    p = __fmaf_rn(p, r, 0.5f);
    p = __fmaf_rn(p, r, 1.0f);
    p = __fmaf_rn(p, r, 1.0f);
    const int e = static_cast<int>(n) + 127;
    const float scale = e >= 255 ? __int_as_float(0x7f800000) : __int_as_float(e << 23);
    return __fmul_rn(p, scale);
}

}  // namespace avd
