// The logarithm and the two-argument arctangent of the colour grain gains, evaluated with
// separately rounded float operations in a fixed order so that a CPU evaluation of the same steps
// gives the same bits (the exponential is exp_mirror.cuh's). Written from the mathematics:
//
//   log_mirror    x = m 2^e with m in [sqrt(1/2), sqrt(2)], ln m = 2 atanh(s) for s = (m-1)/(m+1)
//                 by the series 2s (1 + s^2/3 + s^4/5 + ... + s^10/11) (|s| <= 0.172, so the first
//                 omitted term is below 1e-10 relative), plus e ln2 with ln2 split into a 16-bit
//                 head and a tail.
//   atan2_mirror  octant reduction to t = min/max in [0, 1], t > tan(pi/12) folded by
//                 atan t = pi/6 + atan((t sqrt3 - 1) / (t + sqrt3)), atan u by its Taylor series to
//                 u^13 (|u| <= 0.268, first omitted term below 1e-9 relative), then the octant and
//                 quadrant restored.
// Both lie within 2 ulp of the true functions over the gains' ranges.
#pragma once

#include <cuda_runtime.h>

#include "exp_mirror.cuh"

namespace avd {

// For finite x > 0.
__device__ __forceinline__ float log_mirror(float x) {
    constexpr float kLn2Hi = 0.693145751953125f;
    constexpr float kLn2Lo = 1.428606765330187045037746e-06f;
    constexpr float kSqrt2 = 1.41421356237309504880f;
    uint32_t b = __float_as_uint(x);
    int e = 0;
    if (b < 0x00800000u) {  // subnormal: bring it into the normal range
        x = __fmul_rn(x, 16777216.0f);
        b = __float_as_uint(x);
        e = -24;
    }
    e += static_cast<int>(b >> 23) - 127;
    float m = __uint_as_float((b & 0x007FFFFFu) | 0x3F800000u);
    if (m > kSqrt2) {
        m = __fmul_rn(m, 0.5f);
        e += 1;
    }
    const float s = __fdiv_rn(__fsub_rn(m, 1.0f), __fadd_rn(m, 1.0f));
    const float z = __fmul_rn(s, s);
    float p = 1.0f / 11.0f;
    p = __fadd_rn(__fmul_rn(p, z), 1.0f / 9.0f);
    p = __fadd_rn(__fmul_rn(p, z), 1.0f / 7.0f);
    p = __fadd_rn(__fmul_rn(p, z), 1.0f / 5.0f);
    p = __fadd_rn(__fmul_rn(p, z), 1.0f / 3.0f);
    p = __fmul_rn(p, z);
    const float lm = __fmul_rn(__fadd_rn(s, __fmul_rn(s, p)), 2.0f);
    const float fe = static_cast<float>(e);
    return __fadd_rn(__fmul_rn(fe, kLn2Hi), __fadd_rn(__fmul_rn(fe, kLn2Lo), lm));
}

__device__ __forceinline__ float atan2_mirror(float y, float x) {
    constexpr float kTan15 = 0.267949192431122706f;
    constexpr float kSqrt3 = 1.73205080756887729f;
    constexpr float kPi6 = 0.523598775598298873f;
    constexpr float kPi2 = 1.57079632679489662f;
    constexpr float kPi = 3.14159265358979324f;
    const float ax = fabsf(x), ay = fabsf(y);
    const bool swap = ay > ax;
    const float num = swap ? ax : ay, den = swap ? ay : ax;
    float t = den > 0.0f ? __fdiv_rn(num, den) : 0.0f;
    float base = 0.0f;
    if (t > kTan15) {
        t = __fdiv_rn(__fsub_rn(__fmul_rn(t, kSqrt3), 1.0f), __fadd_rn(t, kSqrt3));
        base = kPi6;
    }
    const float z = __fmul_rn(t, t);
    float q = 1.0f / 13.0f;
    q = __fsub_rn(__fmul_rn(q, z), 1.0f / 11.0f);
    q = __fadd_rn(__fmul_rn(q, z), 1.0f / 9.0f);
    q = __fsub_rn(__fmul_rn(q, z), 1.0f / 7.0f);
    q = __fadd_rn(__fmul_rn(q, z), 1.0f / 5.0f);
    q = __fsub_rn(__fmul_rn(q, z), 1.0f / 3.0f);
    q = __fadd_rn(__fmul_rn(q, z), 1.0f);
    float a = __fadd_rn(base, __fmul_rn(t, q));
    if (swap) a = __fsub_rn(kPi2, a);
    if (signbit(x)) a = __fsub_rn(kPi, a);
    return signbit(y) ? -a : a;
}

}  // namespace avd
