// CPU ORACLE - test infrastructure only (see nlm_oracle.cpp for the rules it follows).
//
// A C++17 restatement of av-denoise's colour grain gains, in the arithmetic of the CUDA kernels
// (every multiply and add separately rounded, sums in the kernels' order; the transcendental
// functions are the mirrors of mirror_math.h):
//
//   block means     av-denoise-core/src/noise/kernels/colour.rs:187-340 (`noise_colour_means`):
//                   each 16x16 block's mean luma, Cb and Cr on the 8-bit scale, on the luma and the
//                   chroma noise grid; each sum is 64 per-thread strided sums folded in halving
//                   rounds of 32..1.
//   cell sums       colour.rs:342-430 (`noise_colour_accumulate`): each static, measurable block's
//                   count, fixed-point log grain, colour and histogram bin, per channel, into its
//                   colour cell (16 brightness bins x (1 neutral + 5 saturation levels x 12 hue
//                   sectors)), plus the luma calibration or chroma plane records.
//   window          colour.rs:441-470 (`noise_colour_window`): the frames' fixed-point sums decoded
//                   and added oldest first.
//   levels          colour.rs:472-559 (`noise_colour_levels`): each cell's kept blocks under its
//                   ceiling and its mean (luma) or median (chroma) log grain.
//   fit             kernels/colour_fit.rs:341-935 (`noise_colour_fit_base`, `solve_knots`,
//                   `noise_colour_fit_kernel`, `noise_colour_fit_table`, `noise_colour_fit_ceilings`)
//                   and noise/colour.rs:630-680 (`ColourFit::queue`): a 17-knot brightness base by
//                   penalised least squares, a Gaussian-kernel lift of the cells' residuals, the
//                   pulled cell table; a second fit without each cell's blocks above the first
//                   fit's model plus ln 2.
//   gains           colour_fit.rs:937-1125 (`noise_colour_fit_gains`): log gains against the
//                   neutral calibration over the luma noise curve (luma) or the plane's median grain
//                   clamped to 0.4..3 (chroma), ramped in with the evidence.
//   lookup          colour_fit.rs:88-262 (`colour_table_value`, `colour_gain`, `colour_gain_pair`):
//                   the gain at a colour, interpolated between the 8 nearest cell centres.
//
// One deliberate difference, shared with the CUDA kernels: the hue angle, the logarithm and the
// exponential are the mirror functions, and the cell centres' cosines and sines are the correctly
// rounded values at the exact sector angles; the reference evaluates the device's f32 functions,
// within a few ulp of these.

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "colour_table.h"
#include "mirror_math.h"

namespace {

using mirror::atan2_mirror;
using mirror::exp_mirror;
using mirror::log_mirror;
using namespace colour_table;

constexpr int NB = 16;
constexpr float STATIC_GATE = 1.5f / 255.0f;
constexpr float SQRT_2F = 1.41421356237309504880f;
constexpr float LN_2F = 0.693147180559945309f;

// noise/colour.rs:24-176.
constexpr float NEUTRAL_SATURATION = 8.0f;
constexpr int W_COUNT = 0, W_LOG = 1, W_LUMA = 2, W_CB = 3, W_CR = 4, W_HIST = 5;
constexpr int HIST_BINS = 64;
constexpr float LOG_MIN = -3.5f, LOG_STEP = 0.125f;
constexpr float LOG_MAX = LOG_MIN + static_cast<float>(HIST_BINS) * LOG_STEP;
constexpr int CELL_WORDS = W_HIST + HIST_BINS;  // 69
constexpr int LEVEL_FIELDS = 2;
constexpr float CHROMA_CENTRE = 128.0f;
constexpr float LUMA_MIN = 20.0f, LUMA_MAX = 240.0f;
constexpr float LUMA_GRAIN_FLOOR = 0.05f, CHROMA_GRAIN_FLOOR = 0.03f;
constexpr float LOG_FIXED = 2048.0f, MEAN_FIXED = 16.0f;
constexpr int FIT_THREADS = 256;
constexpr int KERNEL_LANES = 8;
constexpr int KNOTS = 17, LAST_KNOT = 16;
constexpr float KNOT_STEP = 255.0f / static_cast<float>(LAST_KNOT);
constexpr float KNOT_PENALTY = 2.0f, RIDGE = 1.0e-5f, MIN_BLOCKS = 8.0f;
constexpr float KERNEL_EXPONENT = -0.5f / (1.0f * 1.0f);
constexpr float KERNEL_LUMA_STEP = 32.0f, KERNEL_CHROMA_STEP = 12.0f;
constexpr float PRIOR_SHARE = 0.002f, PULL = 15.0f, LUMA_DEAD_ZONE = 0.1f;
constexpr float CHROMA_GAIN_MIN = 0.4f, CHROMA_GAIN_MAX = 3.0f;
constexpr float NEUTRAL_RAMP = 256.0f, BLOCK_RAMP = 256.0f;
constexpr int CF_LUMA = 0, CF_CB = 1, CF_CR = 2, CF_WEIGHT = 3, CF_RESIDUAL = 4, CF_FIELDS = 5;
constexpr int P_PRIOR = KNOTS, P_POPULATED = KNOTS + 1, P_BLOCKS = KNOTS + 2, P_LUMA_LOW = KNOTS + 3,
              P_LUMA_HIGH = KNOTS + 4, PLANE_WORDS = KNOTS + 5;
constexpr int QUERIES = 2 * CELLS;
constexpr int HIST_EDGES = HIST_BINS + 1;
constexpr int NORM_RECORDS = BRIGHTNESS_BINS;

// cos and sin of each hue sector's centre angle, -pi + (s + 0.5) pi / 6, correctly rounded.
constexpr float C15 = 0.965925826289068287f, S15 = 0.258819045102520762f, H45 = 0.707106781186547524f;
constexpr float SECTOR_COS[12] = {-C15, -H45, -S15, S15, H45, C15, C15, H45, S15, -S15, -H45, -C15};
constexpr float SECTOR_SIN[12] = {-S15, -H45, -C15, -C15, -H45, -S15, S15, H45, C15, C15, H45, S15};

int record_count(int planes, bool luma) { return planes * CELLS + (luma ? BRIGHTNESS_BINS : planes); }

uint32_t histogram_bin(float log_grain) {
    const float position = std::floor((log_grain - LOG_MIN) / LOG_STEP);
    return static_cast<uint32_t>(clampf(position, 0.0f, static_cast<float>(HIST_BINS - 1)));
}

// Rust's `f32::round`: half away from zero.
int32_t round_fixed(float v) { return static_cast<int32_t>(std::round(v)); }

void add_block(int32_t* cells, int record, float log_grain, float luma, float cb, float cr) {
    int32_t* r = cells + static_cast<int64_t>(record) * CELL_WORDS;
    const float clamped = clampf(log_grain, LOG_MIN, LOG_MAX);
    r[W_COUNT] += 1;
    r[W_LOG] += round_fixed(clamped * LOG_FIXED);
    r[W_LUMA] += round_fixed(luma * MEAN_FIXED);
    r[W_CB] += round_fixed(cb * MEAN_FIXED);
    r[W_CR] += round_fixed(cr * MEAN_FIXED);
    r[W_HIST + histogram_bin(log_grain)] += 1;
}

float read_sample(const uint32_t* plane, int64_t index, int spw, bool is_float) {
    const uint32_t word = plane[index / spw];
    if (is_float) return mirror::from_bits(word);
    const int bits = 32 / spw;
    const uint32_t mask = spw == 1 ? 0xFFFFFFFFu : ((1u << bits) - 1u);
    return static_cast<float>((word >> ((index % spw) * bits)) & mask);
}

// ---- the fit (colour_fit.rs:264-935) ------------------------------------------------------------

void cell_centre(uint32_t cell, float* luma, float* cb, float* cr) {
    const uint32_t brightness = cell / PER_BRIGHTNESS, ring = cell % PER_BRIGHTNESS;
    *luma = (static_cast<float>(brightness) + 0.5f) * BRIGHTNESS_STEP;
    const uint32_t coloured = std::max(ring, 1u) - 1u;
    const uint32_t level = coloured / HUE_BINS + 1u, sector = coloured % HUE_BINS;
    const float saturation = ring == 0 ? 0.0f : SAT_CENTRES[level];
    *cb = saturation * SECTOR_COS[sector];
    *cr = saturation * SECTOR_SIN[sector];
}

float knot_position(float luma) { return clampf(luma / KNOT_STEP, 0.0f, static_cast<float>(LAST_KNOT)); }
uint32_t knot_low(float position) {
    return std::min(static_cast<uint32_t>(std::floor(position)), static_cast<uint32_t>(LAST_KNOT - 1));
}

float brightness_base(const float* header, float luma) {
    const float held = clampf(luma, header[P_LUMA_LOW], header[P_LUMA_HIGH]);
    const float position = knot_position(held);
    const uint32_t low = knot_low(position);
    const float fraction = position - static_cast<float>(low);
    return header[low] + (header[low + 1] - header[low]) * fraction;
}

float shrink(float value, float dead_zone) {
    const float size = std::max(std::fabs(value) - dead_zone, 0.0f);
    return value < 0.0f ? -size : size;
}

// colour.rs:505-559 for cells [first, first + count).
void levels_of(const float* window, const float* ceilings, int first, int count, bool mean_level, float* levels) {
    for (int cell = first; cell < first + count; ++cell) {
        const float* r = window + static_cast<int64_t>(cell) * CELL_WORDS;
        const float ceiling = ceilings[cell];
        float dropped = 0.0f, dropped_log = 0.0f;
        for (int bin = 0; bin < HIST_BINS; ++bin) {
            const float n = r[W_HIST + bin];
            const float low = LOG_MIN + static_cast<float>(bin) * LOG_STEP;
            const float high = low + LOG_STEP;
            const float above = clampf((high - ceiling) / LOG_STEP, 0.0f, 1.0f);
            const float cut = std::max(low, ceiling);
            dropped += n * above;
            dropped_log += n * above * (cut + high) * 0.5f;
        }
        const float kept = std::max(r[W_COUNT] - dropped, 0.0f);
        float level = 0.0f;
        if (mean_level) {
            level = (r[W_LOG] - dropped_log) / std::max(kept, 1.0f);
        } else {
            const float target = kept * 0.5f;
            float below = 0.0f;
            bool found = false;
            for (int bin = 0; bin < HIST_BINS; ++bin) {
                const float n = r[W_HIST + bin];
                const float low = LOG_MIN + static_cast<float>(bin) * LOG_STEP;
                const float high = low + LOG_STEP;
                const float above = clampf((high - ceiling) / LOG_STEP, 0.0f, 1.0f);
                const float share = 1.0f - above;
                const float kept_count = n * share;
                if (!found && below + kept_count >= target && kept_count > 0.0f) {
                    level = low + (target - below) / kept_count * share * LOG_STEP;
                    found = true;
                }
                below += kept_count;
            }
        }
        levels[cell * LEVEL_FIELDS] = kept;
        levels[cell * LEVEL_FIELDS + 1] = kept > 0.0f ? level : 0.0f;
    }
}

// colour_fit.rs:534-686 (`solve_knots`).
void solve_knots(const float* sums, float* knots, float penalty) {
    constexpr int SUM_OFF = KNOTS, SUM_RIGHT = KNOTS + LAST_KNOT;
    float diag[KNOTS], first[KNOTS], second[KNOTS], right[KNOTS];
    for (int k = 0; k < KNOTS; ++k) {
        diag[k] = sums[k];
        right[k] = sums[SUM_RIGHT + k];
        first[k] = k < LAST_KNOT ? sums[SUM_OFF + k] : 0.0f;
        second[k] = 0.0f;
    }
    for (int row = 0; row < KNOTS - 2; ++row) {
        diag[row] += penalty;
        diag[row + 1] += 4.0f * penalty;
        diag[row + 2] += penalty;
        first[row] -= 2.0f * penalty;
        first[row + 1] -= 2.0f * penalty;
        second[row] += penalty;
    }
    float scale[KNOTS];
    for (int k = 0; k < KNOTS; ++k) scale[k] = 1.0f / std::sqrt(std::max(diag[k], 1.0e-30f));
    float ld[KNOTS], l1[KNOTS], l2[KNOTS];
    for (int k = 0; k < KNOTS; ++k) {
        float pivot = 1.0f + RIDGE;
        if (k >= 1) pivot -= l1[k - 1] * l1[k - 1];
        if (k >= 2) pivot -= l2[k - 2] * l2[k - 2];
        const float root = std::sqrt(std::max(pivot, 1.0e-12f));
        ld[k] = root;
        l1[k] = 0.0f;
        l2[k] = 0.0f;
        if (k + 1 < KNOTS) {
            float below = first[k] * scale[k] * scale[k + 1];
            if (k >= 1) below -= l2[k - 1] * l1[k - 1];
            l1[k] = below / root;
        }
        if (k + 2 < KNOTS) l2[k] = second[k] * scale[k] * scale[k + 2] / root;
    }
    float solution[KNOTS], residual[KNOTS];
    for (int k = 0; k < KNOTS; ++k) {
        solution[k] = 0.0f;
        residual[k] = right[k];
    }
    for (int pass = 0; pass < 2; ++pass) {
        float fwd[KNOTS], bwd[KNOTS];
        for (int k = 0; k < KNOTS; ++k) {
            float v = residual[k] * scale[k];
            if (k >= 1) v -= l1[k - 1] * fwd[k - 1];
            if (k >= 2) v -= l2[k - 2] * fwd[k - 2];
            fwd[k] = v / ld[k];
        }
        for (int k = LAST_KNOT; k >= 0; --k) {
            float v = fwd[k];
            if (k + 1 < KNOTS) v -= l1[k] * bwd[k + 1];
            if (k + 2 < KNOTS) v -= l2[k] * bwd[k + 2];
            bwd[k] = v / ld[k];
        }
        for (int k = 0; k < KNOTS; ++k) solution[k] += bwd[k] * scale[k];
        for (int k = 0; k < KNOTS; ++k) {
            const float ridge = RIDGE * diag[k];
            float product = (diag[k] + ridge) * solution[k];
            if (k >= 1) product += first[k - 1] * solution[k - 1];
            if (k >= 2) product += second[k - 2] * solution[k - 2];
            if (k + 1 < KNOTS) product += first[k] * solution[k + 1];
            if (k + 2 < KNOTS) product += second[k] * solution[k + 2];
            residual[k] = right[k] - product;
        }
    }
    for (int k = 0; k < KNOTS; ++k) knots[k] = solution[k];
}

// colour_fit.rs:341-532 (`noise_colour_fit_base`) for one plane.
void fit_base(const float* window, const float* levels, int plane, float* fit_cells, float* header) {
    const int pc = plane * CELLS;
    std::vector<uint32_t> lows(CELLS);
    std::vector<float> fractions(CELLS), weights(CELLS), cell_levels(CELLS);
    float root_p[FIT_THREADS], pop_p[FIT_THREADS], block_p[FIT_THREADS], low_p[FIT_THREADS], high_p[FIT_THREADS];
    for (int t = 0; t < FIT_THREADS; ++t) {
        float root_sum = 0.0f, pop_sum = 0.0f, block_sum = 0.0f, span_low = FLT_MAX, span_high = -FLT_MAX;
        for (int cell = t; cell < CELLS; cell += FIT_THREADS) {
            const float* r = window + static_cast<int64_t>(pc + cell) * CELL_WORDS;
            const float divisor = std::max(r[W_COUNT], 1.0f);
            const float luma = r[W_LUMA] / divisor, cb = r[W_CB] / divisor, cr = r[W_CR] / divisor;
            const float kept = levels[(pc + cell) * LEVEL_FIELDS], level = levels[(pc + cell) * LEVEL_FIELDS + 1];
            const bool populated = kept >= MIN_BLOCKS;
            const float position = knot_position(luma);
            const uint32_t low = knot_low(position);
            const float weight = populated ? kept : 0.0f;
            lows[cell] = low;
            fractions[cell] = position - static_cast<float>(low);
            weights[cell] = weight;
            cell_levels[cell] = level;
            root_sum += std::sqrt(weight);
            pop_sum += populated ? 1.0f : 0.0f;
            block_sum += kept;
            if (populated) {
                span_low = std::min(span_low, luma);
                span_high = std::max(span_high, luma);
            }
            float* f = fit_cells + static_cast<int64_t>(pc + cell) * CF_FIELDS;
            f[CF_LUMA] = luma;
            f[CF_CB] = cb;
            f[CF_CR] = cr;
            f[CF_WEIGHT] = weight;
        }
        root_p[t] = root_sum;
        pop_p[t] = pop_sum;
        block_p[t] = block_sum;
        low_p[t] = span_low;
        high_p[t] = span_high;
    }
    for (int half = FIT_THREADS / 2; half > 0; half /= 2)
        for (int t = 0; t < half; ++t) {
            root_p[t] = root_p[t] + root_p[t + half];
            pop_p[t] = pop_p[t] + pop_p[t + half];
            block_p[t] = block_p[t] + block_p[t + half];
            low_p[t] = std::min(low_p[t], low_p[t + half]);
            high_p[t] = std::max(high_p[t], high_p[t + half]);
        }
    float sums[3 * KNOTS + 3];
    constexpr int SUM_OFF = KNOTS, SUM_RIGHT = KNOTS + LAST_KNOT, SUM_ROOT = SUM_RIGHT + KNOTS;
    for (int knot = 0; knot < KNOTS; ++knot) {
        const int first_bin = std::max(knot, 2) - 2, last_bin = std::min(knot + 1, BRIGHTNESS_BINS);
        float diagonal = 0.0f, off = 0.0f, right = 0.0f;
        for (int i = first_bin * PER_BRIGHTNESS; i < last_bin * PER_BRIGHTNESS; ++i) {
            const uint32_t low = lows[i];
            const float fraction = fractions[i], weight = weights[i];
            const float low_share = 1.0f - fraction;
            const bool is_low = low == static_cast<uint32_t>(knot), is_high = low + 1 == static_cast<uint32_t>(knot);
            const float low_square = is_low ? low_share * low_share : 0.0f;
            const float high_square = is_high ? fraction * fraction : 0.0f;
            const float low_tent = is_low ? low_share : 0.0f;
            const float high_tent = is_high ? fraction : 0.0f;
            const float cross = is_low ? low_share * fraction : 0.0f;
            diagonal += weight * (low_square + high_square);
            off += weight * cross;
            right += weight * cell_levels[i] * (low_tent + high_tent);
        }
        sums[knot] = diagonal;
        sums[SUM_RIGHT + knot] = right;
        if (knot < LAST_KNOT) sums[SUM_OFF + knot] = off;
    }
    const float populated = pop_p[0];
    const bool has_cells = populated > 0.0f;
    const float mean_root = root_p[0] / std::max(populated, 1.0f);
    const float penalty = KNOT_PENALTY * KNOT_PENALTY * mean_root;
    (void)SUM_ROOT;
    float knots[KNOTS];
    solve_knots(sums, knots, penalty);
    for (int k = 0; k < KNOTS; ++k) {
        knots[k] = has_cells ? knots[k] : 0.0f;
        header[k] = knots[k];
    }
    const float blocks = block_p[0];
    header[P_PRIOR] = PRIOR_SHARE * blocks;
    header[P_POPULATED] = has_cells ? 1.0f : 0.0f;
    header[P_BLOCKS] = blocks;
    header[P_LUMA_LOW] = has_cells ? low_p[0] : 0.0f;
    header[P_LUMA_HIGH] = has_cells ? high_p[0] : 255.0f;
    for (int cell = 0; cell < CELLS; ++cell) {
        const uint32_t low = lows[cell];
        const float base = knots[low] + (knots[low + 1] - knots[low]) * fractions[cell];
        fit_cells[static_cast<int64_t>(pc + cell) * CF_FIELDS + CF_RESIDUAL] =
            weights[cell] > 0.0f ? cell_levels[cell] - base : 0.0f;
    }
}

// colour_fit.rs:688-796 (`noise_colour_fit_kernel`) for one plane: bases[q] for q < 2 * CELLS.
void fit_kernel(const float* fit_cells, const float* header, int plane, float* bases) {
    const int pc = plane * CELLS;
    std::vector<float> cl(CELLS), ccb(CELLS), ccr(CELLS), cw(CELLS), lift(CELLS);
    for (int c = 0; c < CELLS; ++c) {
        const float* f = fit_cells + static_cast<int64_t>(pc + c) * CF_FIELDS;
        cl[c] = f[CF_LUMA] / KERNEL_LUMA_STEP;
        ccb[c] = f[CF_CB] / KERNEL_CHROMA_STEP;
        ccr[c] = f[CF_CR] / KERNEL_CHROMA_STEP;
        cw[c] = f[CF_WEIGHT];
        lift[c] = f[CF_WEIGHT] * f[CF_RESIDUAL];
    }
    for (int q = 0; q < QUERIES; ++q) {
        const int qc = q % CELLS;
        float luma, cb, cr;
        if (q >= CELLS) {
            cell_centre(static_cast<uint32_t>(qc), &luma, &cb, &cr);
        } else {
            const float* f = fit_cells + static_cast<int64_t>(pc + qc) * CF_FIELDS;
            luma = f[CF_LUMA];
            cb = f[CF_CB];
            cr = f[CF_CR];
        }
        const float ql = luma / KERNEL_LUMA_STEP, qcb = cb / KERNEL_CHROMA_STEP, qcr = cr / KERNEL_CHROMA_STEP;
        float num[KERNEL_LANES], den[KERNEL_LANES];
        for (int lane = 0; lane < KERNEL_LANES; ++lane) {
            float n = 0.0f, d = 0.0f;
            for (int c = lane; c < CELLS; c += KERNEL_LANES) {
                if (!(cw[c] > 0.0f)) continue;
                const float lg = ql - cl[c], bg = qcb - ccb[c], rg = qcr - ccr[c];
                const float distance = lg * lg + bg * bg + rg * rg;
                const float kernel = exp_mirror(KERNEL_EXPONENT * distance);
                n += kernel * lift[c];
                d += kernel * cw[c];
            }
            num[lane] = n;
            den[lane] = d;
        }
        float qn = 0.0f, qd = 0.0f;
        for (int lane = 0; lane < KERNEL_LANES; ++lane) {
            qn += num[lane];
            qd += den[lane];
        }
        const float total = qd + header[P_PRIOR];
        const float lifted = total > 0.0f ? qn / std::max(total, 1.0e-30f) : 0.0f;
        bases[q] = brightness_base(header, luma) + lifted;
    }
}

// colour_fit.rs:798-886 (`noise_colour_fit_table`) for one plane.
void fit_table(const float* levels, const float* fit_cells, const float* bases, int plane, bool luma,
               float* table) {
    const int pc = plane * CELLS;
    const float dead_zone = luma ? LUMA_DEAD_ZONE : 0.0f;
    std::vector<float> moves(CELLS), populated(CELLS);
    for (int c = 0; c < CELLS; ++c) {
        const float weight = fit_cells[static_cast<int64_t>(pc + c) * CF_FIELDS + CF_WEIGHT];
        const float level = levels[(pc + c) * LEVEL_FIELDS + 1];
        const float pull = weight / (weight + PULL);
        const float gap = shrink(level - bases[c], dead_zone);
        moves[c] = weight > 0.0f ? pull * gap : 0.0f;
        populated[c] = weight > 0.0f ? 1.0f : 0.0f;
    }
    for (int c = 0; c < CELLS; ++c) {
        const int brightness = c / PER_BRIGHTNESS, ring = c % PER_BRIGHTNESS;
        float sum = 0.0f, count = 0.0f;
        if (brightness > 0) {
            sum += moves[c - PER_BRIGHTNESS];
            count += populated[c - PER_BRIGHTNESS];
        }
        if (brightness + 1 < BRIGHTNESS_BINS) {
            sum += moves[c + PER_BRIGHTNESS];
            count += populated[c + PER_BRIGHTNESS];
        }
        const int row = brightness * PER_BRIGHTNESS;
        if (ring == 0) {
            float ring_sum = 0.0f, ring_count = 0.0f;
            for (int s = 0; s < HUE_BINS; ++s) {
                ring_sum += moves[row + 1 + s];
                ring_count += populated[row + 1 + s];
            }
            if (ring_count > 0.0f) {
                sum += ring_sum / ring_count;
                count += 1.0f;
            }
        } else {
            const int level = (ring - 1) / HUE_BINS, sector = (ring - 1) % HUE_BINS;
            const int less = level == 0 ? row : c - HUE_BINS;
            sum += moves[less];
            count += populated[less];
            if (level + 2 < 6) {
                sum += moves[c + HUE_BINS];
                count += populated[c + HUE_BINS];
            }
            const int start = row + 1 + level * HUE_BINS;
            const int next = start + (sector + 1) % HUE_BINS, prev = start + (sector + HUE_BINS - 1) % HUE_BINS;
            sum += moves[next] + moves[prev];
            count += populated[next] + populated[prev];
        }
        const float filled = count > 0.0f ? sum / std::max(count, 1.0f) : 0.0f;
        const float cell_move = populated[c] > 0.0f ? moves[c] : filled;
        table[pc + c] = bases[CELLS + c] + cell_move;
    }
}

// colour_fit.rs:888-912 (`noise_colour_fit_ceilings`) for one plane.
void fit_ceilings(const float* window, const float* table, int plane, float* ceilings) {
    for (int c = plane * CELLS; c < (plane + 1) * CELLS; ++c) {
        const float* r = window + static_cast<int64_t>(c) * CELL_WORDS;
        const float divisor = std::max(r[W_COUNT], 1.0f);
        const float model = table_value(table + plane * CELLS, r[W_LUMA] / divisor, r[W_CB] / divisor,
                                        r[W_CR] / divisor);
        ceilings[c] = r[W_COUNT] > 0.0f ? model + LN_2F : FLT_MAX;
    }
}

struct Normaliser {
    float hist[NORM_RECORDS * HIST_BINS], cumulative[NORM_RECORDS * HIST_EDGES], shifts[NORM_RECORDS];
};

float shifted_share(const Normaliser& n, float position) {
    float share = 0.0f;
    for (int r = 0; r < NORM_RECORDS; ++r) {
        const float offset = position - n.shifts[r] - LOG_MIN;
        const float clamped = clampf(offset / LOG_STEP, 0.0f, static_cast<float>(HIST_BINS));
        const uint32_t bin = std::min(static_cast<uint32_t>(std::floor(clamped)), static_cast<uint32_t>(HIST_BINS - 1));
        const float fraction = clamped - static_cast<float>(bin);
        share += n.cumulative[r * HIST_EDGES + bin] + fraction * n.hist[r * HIST_BINS + bin];
    }
    return share;
}

// colour_fit.rs:937-1100 (`noise_colour_fit_gains`) for one plane.
void fit_gains(const float* window, const float* table, const float* header, const float* curve, bool curve_valid,
               int planes, int plane, bool luma, float* gains) {
    Normaliser n;
    for (int r = 0; r < NORM_RECORDS; ++r) {
        float shift = 0.0f;
        if (luma) {
            const float ratio = curve[r];
            const float applied = curve_valid && ratio > 0.0f ? ratio : 1.0f;
            shift = -log_mirror(applied);
        }
        n.shifts[r] = shift;
    }
    const int extra = planes * CELLS;
    for (int v = 0; v < NORM_RECORDS * HIST_BINS; ++v) {
        const int r = v / HIST_BINS, bin = v % HIST_BINS;
        float count = 0.0f;
        if (luma)
            count = window[static_cast<int64_t>(extra + r) * CELL_WORDS + W_HIST + bin];
        else if (r == 0)
            count = window[static_cast<int64_t>(extra + plane) * CELL_WORDS + W_HIST + bin];
        n.hist[v] = count;
    }
    for (int r = 0; r < NORM_RECORDS; ++r) {
        float running = 0.0f;
        n.cumulative[r * HIST_EDGES] = running;
        for (int bin = 0; bin < HIST_BINS; ++bin) {
            running += n.hist[r * HIST_BINS + bin];
            n.cumulative[r * HIST_EDGES + bin + 1] = running;
        }
    }
    float total = 0.0f;
    for (int r = 0; r < NORM_RECORDS; ++r) total += n.cumulative[r * HIST_EDGES + HIST_BINS];
    const float target = total * 0.5f;
    float below = -FLT_MAX, above = FLT_MAX;
    for (int point = 0; point < NORM_RECORDS * HIST_EDGES; ++point) {
        const int r = point / HIST_EDGES, edge = point % HIST_EDGES;
        const float position = LOG_MIN + static_cast<float>(edge) * LOG_STEP + n.shifts[r];
        if (shifted_share(n, position) < target)
            below = std::max(below, position);
        else
            above = std::min(above, position);
    }
    const float below_share = shifted_share(n, below), above_share = shifted_share(n, above);
    const float rise = std::max(above_share - below_share, 1.0e-30f);
    const float median = below + (target - below_share) / rise * (above - below);
    const bool has_median = total > 0.0f && below > -FLT_MAX && above < FLT_MAX;
    const float normaliser = has_median ? median : 0.0f;
    const bool applies = header[P_POPULATED] > 0.0f && has_median;
    const float log_min = log_mirror(CHROMA_GAIN_MIN), log_max = log_mirror(CHROMA_GAIN_MAX);
    const float blocks = header[P_BLOCKS];
    const float block_ramp = blocks / (blocks + BLOCK_RAMP);
    const float neutral_ramp = total / (total + NEUTRAL_RAMP);
    const float ramp = luma ? block_ramp * neutral_ramp : block_ramp;
    for (int c = 0; c < CELLS; ++c) {
        float log_gain = table[plane * CELLS + c] - normaliser;
        if (luma)
            log_gain += n.shifts[c / PER_BRIGHTNESS];
        else
            log_gain = clampf(log_gain, log_min, log_max);
        gains[plane * CELLS + c] = applies ? ramp * log_gain : 0.0f;
    }
}

}  // namespace

extern "C" {

int orc_colour_cells() { return CELLS; }
int orc_colour_cell_words() { return CELL_WORDS; }
int orc_colour_records(int planes, int luma) { return record_count(planes, luma != 0); }
uint32_t orc_colour_cell(float luma, float cb, float cr) { return colour_cell(luma, cb, cr); }
float orc_log_mirror(float x) { return log_mirror(x); }
float orc_atan2_mirror(float y, float x) { return atan2_mirror(y, x); }

// colour.rs:187-340: the block means of both noise grids from the three input planes (`luma` w x h,
// `cb`/`cr` at the subsampled size, each a word array of `spw` samples per word, or f32 with
// `is_float`). `luma_means` holds 3 floats per luma-grid block, `chroma_means` per chroma-grid block.
void orc_colour_means(const uint32_t* luma, const uint32_t* cb, const uint32_t* cr, int w, int h, int shift_x,
                      int shift_y, int spw, int is_float, float eight_bit_scale, float chroma_bias, float* luma_means,
                      float* chroma_means) {
    const int cw = (w + (1 << shift_x) - 1) >> shift_x, ch = (h + (1 << shift_y) - 1) >> shift_y;
    const int step_x = 1 << shift_x, step_y = 1 << shift_y;
    for (int grid = 0; grid < 2; ++grid) {
        const bool in_luma = grid == 0;
        const int own_w = in_luma ? w : cw, own_h = in_luma ? h : ch;
        const int bxn = (own_w + NB - 1) / NB, byn = (own_h + NB - 1) / NB;
        for (int by = 0; by < byn; ++by)
            for (int bx = 0; bx < bxn; ++bx) {
                const int left = bx * NB, top = by * NB;
                const int right = std::min(left + NB, own_w), bottom = std::min(top + NB, own_h);
                const int ll = in_luma ? left : left * step_x, lt = in_luma ? top : top * step_y;
                const int lr = in_luma ? right : std::min(right * step_x, w);
                const int lb = in_luma ? bottom : std::min(bottom * step_y, h);
                const int cl = in_luma ? left >> shift_x : left, ct = in_luma ? top >> shift_y : top;
                const int cr_ = in_luma ? (right + step_x - 1) >> shift_x : right;
                const int cb_ = in_luma ? (bottom + step_y - 1) >> shift_y : bottom;
                float ls[64], bs[64], rs[64];
                for (int t = 0; t < 64; ++t) {
                    auto rect = [&](const uint32_t* plane, int l, int tp, int r, int b, int stride) {
                        float sum = 0.0f;
                        for (int y = tp + t / 16; y < b; y += 4)
                            for (int x = l + t % 16; x < r; x += 16)
                                sum += read_sample(plane, static_cast<int64_t>(y) * stride + x, spw, is_float != 0);
                        return sum;
                    };
                    ls[t] = rect(luma, ll, lt, lr, lb, w);
                    bs[t] = rect(cb, cl, ct, cr_, cb_, cw);
                    rs[t] = rect(cr, cl, ct, cr_, cb_, cw);
                }
                for (int half = 32; half > 0; half /= 2)
                    for (int t = 0; t < half; ++t) {
                        ls[t] = ls[t] + ls[t + half];
                        bs[t] = bs[t] + bs[t + half];
                        rs[t] = rs[t] + rs[t + half];
                    }
                const float lp = static_cast<float>((lr - ll) * (lb - lt));
                const float cp = static_cast<float>((cr_ - cl) * (cb_ - ct));
                float* out = (in_luma ? luma_means : chroma_means) + (by * bxn + bx) * 3;
                out[0] = ls[0] / lp * eight_bit_scale;
                out[1] = (bs[0] / cp + chroma_bias) * eight_bit_scale - CHROMA_CENTRE;
                out[2] = (rs[0] / cp + chroma_bias) * eight_bit_scale - CHROMA_CENTRE;
            }
    }
}

// colour.rs:342-430: one frame's fixed-point cell sums (orc_colour_records * 69 int32 words,
// zeroed first) from its temporal records and its block means on the records' grid.
void orc_colour_accumulate(const float* records, const float* means, int w, int h, int channels, int luma,
                           float grain_scale, int32_t* cells) {
    const int bxn = (w + NB - 1) / NB, byn = (h + NB - 1) / NB, rl = 3 * channels + 26;
    std::fill(cells, cells + static_cast<int64_t>(record_count(channels, luma != 0)) * CELL_WORDS, 0);
    const float floor = luma ? LUMA_GRAIN_FLOOR : CHROMA_GRAIN_FLOOR;
    const int extra = channels * CELLS;
    for (int i = 0; i < bxn * byn; ++i) {
        const int bx = i % bxn, by = i / bxn;
        const int bw = std::min(NB, w - bx * NB), bh = std::min(NB, h - by * NB);
        const float pixels = static_cast<float>(bw * bh);
        const float* r = records + static_cast<int64_t>(i) * rl;
        const float ml = means[i * 3], mcb = means[i * 3 + 1], mcr = means[i * 3 + 2];
        const uint32_t cell = colour_cell(ml, mcb, mcr);
        const float saturation = std::sqrt(mcb * mcb + mcr * mcr);
        const bool in_range = ml > LUMA_MIN && ml < LUMA_MAX;
        const uint32_t brightness = brightness_bin(ml);
        const bool neutral = saturation < NEUTRAL_SATURATION;
        for (int c = 0; c < channels; ++c) {
            const float mean = r[c] / pixels;
            const float ms = r[channels + c] / pixels;
            const float sigma = std::sqrt(std::max(ms - mean * mean, 0.0f)) / SQRT_2F;
            const float grain = sigma * grain_scale;
            if (!(in_range && std::fabs(mean) < STATIC_GATE && grain > floor)) continue;
            const float log_grain = log_mirror(grain);
            add_block(cells, c * CELLS + static_cast<int>(cell), log_grain, ml, mcb, mcr);
            if (luma) {
                if (neutral) add_block(cells, extra + static_cast<int>(brightness), log_grain, ml, mcb, mcr);
            } else {
                add_block(cells, extra + c, log_grain, ml, mcb, mcr);
            }
        }
    }
}

// colour.rs:441-470: the window's sums of frames first..last (frame f in slot f % capacity).
void orc_colour_window(const int32_t* ring, int capacity, int first, int last, int words, float* window) {
    for (int i = 0; i < words; ++i) {
        const int word = i % CELL_WORDS;
        const float scale = word == W_LOG ? 1.0f / LOG_FIXED : (word >= W_LUMA && word < W_HIST ? 1.0f / MEAN_FIXED : 1.0f);
        float sum = 0.0f;
        for (int f = first; f <= last; ++f)
            sum += static_cast<float>(ring[static_cast<int64_t>(f % capacity) * words + i]) * scale;
        window[i] = sum;
    }
}

void orc_colour_levels(const float* window, const float* ceilings, int cells, int mean_level, float* levels) {
    levels_of(window, ceilings, 0, cells, mean_level != 0, levels);
}

// noise/colour.rs:630-680 (`ColourFit::queue`): both fits and the gains of `planes` planes from the
// window's sums. `curve` holds the 16 luma curve ratios, read when `curve_valid`. Writes each
// plane's log grain table and log gain table (CELLS floats per plane each) and its fit header
// (22 floats per plane).
void orc_colour_fit(const float* window, int planes, int luma, const float* curve, int curve_valid, float* table,
                    float* gains, float* headers) {
    const int cells = planes * CELLS;
    std::vector<float> open(cells, FLT_MAX), ceilings(cells), levels(cells * LEVEL_FIELDS),
        fit_cells(static_cast<size_t>(cells) * CF_FIELDS), bases(QUERIES);
    for (int p = 0; p < planes; ++p) {
        float* header = headers + p * PLANE_WORDS;
        levels_of(window, open.data(), p * CELLS, CELLS, luma != 0, levels.data());
        fit_base(window, levels.data(), p, fit_cells.data(), header);
        fit_kernel(fit_cells.data(), header, p, bases.data());
        fit_table(levels.data(), fit_cells.data(), bases.data(), p, luma != 0, table);
        fit_ceilings(window, table, p, ceilings.data());
        levels_of(window, ceilings.data(), p * CELLS, CELLS, luma != 0, levels.data());
        fit_base(window, levels.data(), p, fit_cells.data(), header);
        fit_kernel(fit_cells.data(), header, p, bases.data());
        fit_table(levels.data(), fit_cells.data(), bases.data(), p, luma != 0, table);
        fit_gains(window, table, header, curve, curve_valid != 0, planes, p, luma != 0, gains);
    }
}

// colour_fit.rs:196-262: the table's interpolated value at each of n colours (luma, cb, cr
// triples), and its exponential (the gain).
void orc_colour_lookup(const float* table, const float* colours, int n, float* values, float* gains) {
    for (int i = 0; i < n; ++i) {
        const float v = table_value(table, colours[3 * i], colours[3 * i + 1], colours[3 * i + 2]);
        values[i] = v;
        gains[i] = exp_mirror(v);
    }
}

}  // extern "C"
