// CPU ORACLE - test infrastructure only (see nlm_oracle.cpp for the rules it follows).
//
// The colour cell table of the grain gains, shared by the colour and the collaborative-filter
// restatements: its layout (av-denoise-core/src/noise/colour.rs:24-81), a block's cell
// (noise/kernels/colour.rs:57-97) and a table's value at a colour interpolated between the 8
// nearest cell centres (noise/kernels/colour_fit.rs:88-262), every operation rounded on its own.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "mirror_math.h"

namespace colour_table {

using mirror::atan2_mirror;

constexpr float PI_F = 3.14159265358979324f;
constexpr float TAU_F = 6.28318530717958648f;
constexpr int BRIGHTNESS_BINS = 16;
constexpr float BRIGHTNESS_STEP = 16.0f;
constexpr float SAT_EDGES[5] = {6.0f, 12.0f, 20.0f, 30.0f, 44.0f};
constexpr float SAT_CENTRES[6] = {3.0f, 9.0f, 16.0f, 25.0f, 37.0f, 51.0f};
constexpr int HUE_BINS = 12;
constexpr int PER_BRIGHTNESS = 1 + 5 * HUE_BINS;          // 61
constexpr int CELLS = BRIGHTNESS_BINS * PER_BRIGHTNESS;  // 976

inline float clampf(float v, float lo, float hi) { return std::min(std::max(v, lo), hi); }

inline uint32_t brightness_bin(float luma) {
    const float scaled = std::floor(luma / BRIGHTNESS_STEP);
    return static_cast<uint32_t>(clampf(scaled, 0.0f, static_cast<float>(BRIGHTNESS_BINS - 1)));
}

// colour.rs:57-83 (`colour_cell`).
inline uint32_t colour_cell(float luma, float cb, float cr) {
    const uint32_t brightness = brightness_bin(luma);
    const float saturation = std::sqrt(cb * cb + cr * cr);
    uint32_t level = 0;
    for (float edge : SAT_EDGES) level += saturation >= edge ? 1u : 0u;
    const float hue = atan2_mirror(cr, cb);
    const float turn = (hue + PI_F) / TAU_F;
    const float raw_sector = std::floor(turn * static_cast<float>(HUE_BINS));
    const uint32_t sector = static_cast<uint32_t>(std::max(raw_sector, 0.0f)) % HUE_BINS;
    const uint32_t coloured = 1u + (std::max(level, 1u) - 1u) * HUE_BINS + sector;
    return brightness * PER_BRIGHTNESS + (level == 0 ? 0u : coloured);
}

// ---- the table lookup (colour_fit.rs:88-262) ---------------------------------------------------

inline float between(float v, float lo, float hi) { return (v - lo) / (hi - lo); }

inline float saturation_position(float s) {
    const float step1 = between(s, SAT_CENTRES[0], SAT_CENTRES[1]);
    const float step2 = 1.0f + between(s, SAT_CENTRES[1], SAT_CENTRES[2]);
    const float step3 = 2.0f + between(s, SAT_CENTRES[2], SAT_CENTRES[3]);
    const float step4 = 3.0f + between(s, SAT_CENTRES[3], SAT_CENTRES[4]);
    const float step5 = 4.0f + between(s, SAT_CENTRES[4], SAT_CENTRES[5]);
    const float upper4 = s < SAT_CENTRES[4] ? step4 : step5;
    const float upper3 = s < SAT_CENTRES[3] ? step3 : upper4;
    const float upper2 = s < SAT_CENTRES[2] ? step2 : upper3;
    const float position = s < SAT_CENTRES[1] ? step1 : upper2;
    return clampf(position, 0.0f, 5.0f);
}

inline uint32_t table_index(uint32_t brightness, uint32_t level, uint32_t sector) {
    const uint32_t coloured = 1u + (std::max(level, 1u) - 1u) * HUE_BINS + sector;
    return brightness * PER_BRIGHTNESS + (level == 0 ? 0u : coloured);
}

struct Position {
    uint32_t brightness_low, level_low, sector_low;
    float brightness_fraction, level_fraction, hue_fraction;
};

inline Position table_position(float luma, float cb, float cr) {
    Position p;
    const float bpos = clampf(luma / BRIGHTNESS_STEP - 0.5f, 0.0f, static_cast<float>(BRIGHTNESS_BINS - 1));
    p.brightness_low = std::min(static_cast<uint32_t>(std::floor(bpos)), static_cast<uint32_t>(BRIGHTNESS_BINS - 2));
    p.brightness_fraction = bpos - static_cast<float>(p.brightness_low);
    const float saturation = std::sqrt(cb * cb + cr * cr);
    const float lpos = saturation_position(saturation);
    p.level_low = std::min(static_cast<uint32_t>(std::floor(lpos)), 4u);
    p.level_fraction = lpos - static_cast<float>(p.level_low);
    const float hue = atan2_mirror(cr, cb);
    const float hpos = (hue + PI_F) / TAU_F * static_cast<float>(HUE_BINS) - 0.5f;
    const float hfloor = std::floor(hpos);
    p.hue_fraction = hpos - hfloor;
    p.sector_low = static_cast<uint32_t>(hfloor + static_cast<float>(HUE_BINS)) % HUE_BINS;
    return p;
}

inline void table_corner(const Position& p, int corner, uint32_t* index, float* weight) {
    const int bs = corner / 4, ls = (corner / 2) % 2, ss = corner % 2;
    const float bw = bs ? p.brightness_fraction : 1.0f - p.brightness_fraction;
    const float lw = ls ? p.level_fraction : 1.0f - p.level_fraction;
    const float sw = ss ? p.hue_fraction : 1.0f - p.hue_fraction;
    const uint32_t sector = (p.sector_low + ss) % HUE_BINS;
    *index = table_index(p.brightness_low + bs, p.level_low + ls, sector);
    *weight = bw * lw * sw;
}

inline float table_value(const float* table, float luma, float cb, float cr) {
    const Position p = table_position(luma, cb, cr);
    float value = 0.0f;
    for (int corner = 0; corner < 8; ++corner) {
        uint32_t index;
        float weight;
        table_corner(p, corner, &index, &weight);
        value += weight * table[index];
    }
    return value;
}

}  // namespace colour_table
