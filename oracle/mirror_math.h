// CPU ORACLE - test infrastructure only (see nlm_oracle.cpp for the rules it follows).
//
// The transcendental functions of the colour grain gains, evaluated with separately rounded float
// operations in a fixed order, so that the CUDA kernels (csrc/mirror_math.cuh, the same steps) give
// the same bits. Each is written from the mathematics:
//
//   exp_mirror    Cody and Waite's reduction x = n ln2 + r (ln2 split into a 16-bit head), e^r by
//                 its degree-7 Taylor polynomial in Horner form with fused multiply-adds, scaled by
//                 2^n from the exponent bits (the same steps as the exact NLMeans path's).
//   log_mirror    x = m 2^e with m in [sqrt(1/2), sqrt(2)], ln m = 2 atanh(s) for s = (m-1)/(m+1)
//                 by the series 2s (1 + s^2/3 + s^4/5 + ... + s^10/11) (|s| <= 0.172, so the first
//                 omitted term is below 1e-10 relative), plus e ln2 with ln2 split into a 16-bit
//                 head and a tail.
//   atan2_mirror  octant reduction to t = min/max in [0, 1], t > tan(pi/12) folded by
//                 atan t = pi/6 + atan((t sqrt3 - 1) / (t + sqrt3)), atan u by its Taylor series to
//                 u^13 (|u| <= 0.268, first omitted term below 1e-9 relative), then the octant and
//                 quadrant restored.
// Each lies within a few ulp of the true function over the ranges the gains use; the reference
// evaluates the same functions in f32 on its device, within a few ulp of these.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

namespace mirror {

inline float from_bits(uint32_t b) {
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}
inline uint32_t to_bits(float f) {
    uint32_t b;
    std::memcpy(&b, &f, 4);
    return b;
}

inline float exp_mirror(float x) {
    constexpr float kLog2e = 1.44269502162933349609375f;
    constexpr float kLn2Hi = 0.693145751953125f;
    constexpr float kLn2Lo = 1.428606765330187045037746e-06f;
    if (!(x >= -87.0f)) return 0.0f;
    const float n = std::nearbyint(x * kLog2e);
    float r = std::fma(n, -kLn2Hi, x);
    r = std::fma(n, -kLn2Lo, r);
    float p = 1.0f / 5040.0f;
    p = std::fma(p, r, 1.0f / 720.0f);
    p = std::fma(p, r, 1.0f / 120.0f);
    p = std::fma(p, r, 1.0f / 24.0f);
    p = std::fma(p, r, 1.0f / 6.0f);
    p = std::fma(p, r, 0.5f);
    p = std::fma(p, r, 1.0f);
    p = std::fma(p, r, 1.0f);
    const int e = static_cast<int>(n) + 127;
    const float scale = e >= 255 ? from_bits(0x7f800000u) : from_bits(static_cast<uint32_t>(e) << 23);
    return p * scale;
}

// For finite x > 0.
inline float log_mirror(float x) {
    constexpr float kLn2Hi = 0.693145751953125f;
    constexpr float kLn2Lo = 1.428606765330187045037746e-06f;
    constexpr float kSqrt2 = 1.41421356237309504880f;
    uint32_t b = to_bits(x);
    int e = 0;
    if (b < 0x00800000u) {  // subnormal: bring it into the normal range
        x = x * 16777216.0f;
        b = to_bits(x);
        e = -24;
    }
    e += static_cast<int>(b >> 23) - 127;
    float m = from_bits((b & 0x007FFFFFu) | 0x3F800000u);
    if (m > kSqrt2) {
        m = m * 0.5f;
        e += 1;
    }
    const float s = (m - 1.0f) / (m + 1.0f);
    const float z = s * s;
    float p = 1.0f / 11.0f;
    p = p * z + 1.0f / 9.0f;
    p = p * z + 1.0f / 7.0f;
    p = p * z + 1.0f / 5.0f;
    p = p * z + 1.0f / 3.0f;
    p = p * z;
    const float lm = (s + s * p) * 2.0f;
    const float fe = static_cast<float>(e);
    return fe * kLn2Hi + (fe * kLn2Lo + lm);
}

inline float atan2_mirror(float y, float x) {
    constexpr float kTan15 = 0.267949192431122706f;
    constexpr float kSqrt3 = 1.73205080756887729f;
    constexpr float kPi6 = 0.523598775598298873f;
    constexpr float kPi2 = 1.57079632679489662f;
    constexpr float kPi = 3.14159265358979324f;
    const float ax = std::fabs(x), ay = std::fabs(y);
    const bool swap = ay > ax;
    const float num = swap ? ax : ay, den = swap ? ay : ax;
    float t = den > 0.0f ? num / den : 0.0f;
    float base = 0.0f;
    if (t > kTan15) {
        t = (t * kSqrt3 - 1.0f) / (t + kSqrt3);
        base = kPi6;
    }
    const float z = t * t;
    float q = 1.0f / 13.0f;
    q = q * z - 1.0f / 11.0f;
    q = q * z + 1.0f / 9.0f;
    q = q * z - 1.0f / 7.0f;
    q = q * z + 1.0f / 5.0f;
    q = q * z - 1.0f / 3.0f;
    q = q * z + 1.0f;
    float a = base + t * q;
    if (swap) a = kPi2 - a;
    if (std::signbit(x)) a = kPi - a;
    return std::signbit(y) ? -a : a;
}

}  // namespace mirror
