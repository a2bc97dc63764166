// The colour cell table of the grain gains: its layout, a block's cell, and the value of a table at
// a colour interpolated between the 8 nearest cell centres (av-denoise-core/src/noise/colour.rs:24-81,
// noise/kernels/colour.rs:57-97, noise/kernels/colour_fit.rs:88-262). Every operation is rounded on
// its own, in the oracle's order (oracle/colour_oracle.cpp), so both give the same bits.
//
// A table holds one value per cell: 16 brightness bins of 16 codes, each with one neutral cell and
// 5 saturation levels (edges 6, 12, 20, 30, 44 codes of chroma magnitude) of 12 hue sectors.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "mirror_math.cuh"

namespace avd {
namespace colour {

constexpr int kBrightnessBins = 16;
constexpr float kBrightnessStep = 16.0f;
constexpr int kHueBins = 12;
constexpr int kLevels = 6;  // neutral, then 5 saturation levels
constexpr int kPerBrightness = 1 + 5 * kHueBins;
constexpr int kCells = kBrightnessBins * kPerBrightness;  // 976
constexpr int kMeanFields = 3;
constexpr float kChromaCentre = 128.0f;
constexpr float kPi = 3.14159265358979324f;
constexpr float kTau = 6.28318530717958648f;

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

__device__ __forceinline__ float saturation_of(float cb, float cr) {
    return __fsqrt_rn(__fadd_rn(__fmul_rn(cb, cb), __fmul_rn(cr, cr)));
}

__device__ __forceinline__ uint32_t brightness_bin(float luma) {
    const float scaled = floorf(__fdiv_rn(luma, kBrightnessStep));
    return static_cast<uint32_t>(clampf(scaled, 0.0f, static_cast<float>(kBrightnessBins - 1)));
}

// colour.rs:57-83 (`colour_cell`).
__device__ __forceinline__ uint32_t colour_cell(float luma, float cb, float cr) {
    const uint32_t brightness = brightness_bin(luma);
    const float s = saturation_of(cb, cr);
    const uint32_t level = (s >= 6.0f ? 1u : 0u) + (s >= 12.0f ? 1u : 0u) + (s >= 20.0f ? 1u : 0u) +
                           (s >= 30.0f ? 1u : 0u) + (s >= 44.0f ? 1u : 0u);
    const float turn = __fdiv_rn(__fadd_rn(atan2_mirror(cr, cb), kPi), kTau);
    const float raw_sector = floorf(__fmul_rn(turn, static_cast<float>(kHueBins)));
    const uint32_t sector = static_cast<uint32_t>(fmaxf(raw_sector, 0.0f)) % kHueBins;
    const uint32_t coloured = 1u + (max(level, 1u) - 1u) * kHueBins + sector;
    return brightness * kPerBrightness + (level == 0 ? 0u : coloured);
}

__device__ __forceinline__ float between(float v, float lo, float hi) {
    return __fdiv_rn(__fsub_rn(v, lo), __fsub_rn(hi, lo));
}

// colour_fit.rs:96-113: the fractional index along the saturation centres 3, 9, 16, 25, 37, 51.
__device__ __forceinline__ float saturation_position(float s) {
    const float step1 = between(s, 3.0f, 9.0f);
    const float step2 = __fadd_rn(1.0f, between(s, 9.0f, 16.0f));
    const float step3 = __fadd_rn(2.0f, between(s, 16.0f, 25.0f));
    const float step4 = __fadd_rn(3.0f, between(s, 25.0f, 37.0f));
    const float step5 = __fadd_rn(4.0f, between(s, 37.0f, 51.0f));
    const float upper4 = s < 37.0f ? step4 : step5;
    const float upper3 = s < 25.0f ? step3 : upper4;
    const float upper2 = s < 16.0f ? step2 : upper3;
    return clampf(s < 9.0f ? step1 : upper2, 0.0f, 5.0f);
}

__device__ __forceinline__ uint32_t table_index(uint32_t brightness, uint32_t level, uint32_t sector) {
    const uint32_t coloured = 1u + (max(level, 1u) - 1u) * kHueBins + sector;
    return brightness * kPerBrightness + (level == 0 ? 0u : coloured);
}

struct TablePosition {
    uint32_t brightness_low, level_low, sector_low;
    float brightness_fraction, level_fraction, hue_fraction;
};

// colour_fit.rs:134-170 (`table_position`).
__device__ __forceinline__ TablePosition table_position(float luma, float cb, float cr) {
    TablePosition p;
    const float bpos = clampf(__fsub_rn(__fdiv_rn(luma, kBrightnessStep), 0.5f), 0.0f,
                              static_cast<float>(kBrightnessBins - 1));
    p.brightness_low = min(static_cast<uint32_t>(floorf(bpos)), static_cast<uint32_t>(kBrightnessBins - 2));
    p.brightness_fraction = __fsub_rn(bpos, static_cast<float>(p.brightness_low));
    const float lpos = saturation_position(saturation_of(cb, cr));
    p.level_low = min(static_cast<uint32_t>(floorf(lpos)), static_cast<uint32_t>(kLevels - 2));
    p.level_fraction = __fsub_rn(lpos, static_cast<float>(p.level_low));
    const float turn = __fdiv_rn(__fadd_rn(atan2_mirror(cr, cb), kPi), kTau);
    const float hpos = __fsub_rn(__fmul_rn(turn, static_cast<float>(kHueBins)), 0.5f);
    const float hfloor = floorf(hpos);
    p.hue_fraction = __fsub_rn(hpos, hfloor);
    p.sector_low = static_cast<uint32_t>(__fadd_rn(hfloor, static_cast<float>(kHueBins))) % kHueBins;
    return p;
}

// colour_fit.rs:172-193 (`table_corner`): corner c's cell and weight.
__device__ __forceinline__ void table_corner(const TablePosition& p, int corner, uint32_t* index, float* weight) {
    const int bs = corner / 4, ls = (corner / 2) % 2, ss = corner % 2;
    const float bw = bs ? p.brightness_fraction : __fsub_rn(1.0f, p.brightness_fraction);
    const float lw = ls ? p.level_fraction : __fsub_rn(1.0f, p.level_fraction);
    const float sw = ss ? p.hue_fraction : __fsub_rn(1.0f, p.hue_fraction);
    *index = table_index(p.brightness_low + bs, p.level_low + ls, (p.sector_low + ss) % kHueBins);
    *weight = __fmul_rn(__fmul_rn(bw, lw), sw);
}

// colour_fit.rs:196-210 (`colour_table_value`).
__device__ __forceinline__ float table_value(const float* table, float luma, float cb, float cr) {
    const TablePosition p = table_position(luma, cb, cr);
    float value = 0.0f;
#pragma unroll
    for (int corner = 0; corner < 8; ++corner) {
        uint32_t index;
        float weight;
        table_corner(p, corner, &index, &weight);
        value = __fadd_rn(value, __fmul_rn(weight, table[index]));
    }
    return value;
}

// colour_fit.rs:212-262 (`colour_gain`, `colour_gain_pair`): the gains of two tables at one colour.
__device__ __forceinline__ void gain_pair(const float* first, const float* second, float luma, float cb, float cr,
                                          float* first_gain, float* second_gain) {
    const TablePosition p = table_position(luma, cb, cr);
    float a = 0.0f, b = 0.0f;
#pragma unroll
    for (int corner = 0; corner < 8; ++corner) {
        uint32_t index;
        float weight;
        table_corner(p, corner, &index, &weight);
        a = __fadd_rn(a, __fmul_rn(weight, __ldg(first + index)));
        b = __fadd_rn(b, __fmul_rn(weight, __ldg(second + index)));
    }
    *first_gain = exp_mirror(a);
    *second_gain = exp_mirror(b);
}

}  // namespace colour
}  // namespace avd
