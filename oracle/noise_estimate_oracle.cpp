// CPU ORACLE - test infrastructure only (see nlm_oracle.cpp for the rules it follows).
//
// A C++17 restatement of av-denoise's automatic noise estimate without motion compensation, in the
// arithmetic of its GPU kernels (every multiply and add separately rounded, sums in the kernels'
// order; order statistics are exact, so they come from sorting):
//
//   temporal stats  av-denoise-core/src/noise/kernels/stats.rs:141-620 (`nlm_temporal_noise_stats`):
//                   per 16x16 block the per-channel sums of d = new - prev and d^2 and the lag-1
//                   product of neighbouring channel-0 residuals, each summed over the block's 256
//                   threads in thread order; each channel's texture from 4x4 cell means
//                   (stats.rs:599-650); with the luma fields, each 8x8 quarter's residual sums, luma
//                   sum, minimum, maximum and flatness (stats.rs:466-606).
//   reading         kernels/sample.rs:143-803 (`noise_block_derive`, `noise_block_accept`,
//                   `noise_sample_finish`) with the host statement noise/temporal.rs:360-721: the
//                   static gate, the outlier ceiling from the lower quartile of the measurable
//                   candidates, the moved-texture threshold, the per-channel median and lower
//                   quartile of the kept block sigmas, the median lag-1 correlation and the static
//                   fraction; the Immerkaer words are the lower quartile of the cube sigmas. With
//                   the luma fields, the noise curve (kernels/curve.rs:37-133, sample.rs:717-803):
//                   the static quarters' median sigma and the 16 luma bins' medians, interpolated.
//   window fold     kernels/window.rs:1-498 (`noise_window_fold`) and kernels/derive.rs:1-192
//                   (`correlation_factor`, `write_derived`, `write_offset_tables`): the four chains'
//                   medians over the window, the correlation and curve medians, the stream state,
//                   the derived words and the NLM offset tables.
//
// One deliberate difference, shared with the CUDA kernel: the offset tables' exp and ln are
// evaluated in double precision and rounded to float, so this restatement and the kernel agree
// exactly (the reference evaluates them in f32, within a few ulp of these values).
//
// The reference's host tests of the reading (noise/tests/temporal.rs) and of the fold
// (noise/tests/window.rs, fold.rs) are replayed on this restatement by
// tests/test_oracle_noise_estimate.py.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr int NB = 16;                 // TEMPORAL_NOISE_BLOCK
constexpr int NOISE_CHANNELS = 2;
constexpr int IBX = 32, IBY = 8;       // Immerkaer cube
constexpr float STATIC_GATE = 1.5f / 255.0f;
constexpr float RHO_SIGMA_GATE = 0.3f / 255.0f;
constexpr float SIGMA_OUTLIER_FACTOR = 5.0f;
constexpr float STATIC_FRACTION_MIN = 0.05f;
constexpr float SIGMA_FLOOR = 0.1f / 255.0f;
constexpr float SQRT_2F = 1.41421356237309504880f;
// The noise curve (noise/curve.rs:21-50).
constexpr int CURVE_BINS = 16;
constexpr uint32_t MIN_BIN_QUARTERS = 32, MIN_POPULATED_BINS = 3;
constexpr float CLIP_LOW = 4.0f / 255.0f, CLIP_HIGH = 251.0f / 255.0f, FLAT_FACTOR = 0.5f;
constexpr float FLAT_FLOOR = (1.0f / 255.0f) * (1.0f / 255.0f);
constexpr float QUARTER_STATIC_GATE = 2.0f * STATIC_GATE;

// Reading words (noise/reading.rs:7-33).
constexpr int R_IMM_LOW = 0, R_VALID = 2, R_SIGMA = 4, R_SIGMA_LOW = 6, R_RHO = 8, R_STATIC = 9, R_ACCEPTED = 10,
              R_CURVE_VALID = 11, R_QUARTER_MEDIAN = 12, R_POPULATED = 13, R_RATIOS = 14, R_WORDS = 30;
// Fold settings words (noise/fold.rs:16-45).
constexpr int F_SIGMA_SCALE = 0, F_CURVE_APPLIES = 1, F_G_MAX = 2, F_W_FLOOR = 3, F_H2_AUTO = 4, F_H2_PIV = 5,
              F_H2_FIXED = 6, F_PILOT = 7, F_OFFSET_PV = 8, F_MAIN_OFFSET = 9, F_SAD = 10, F_CONF_SAD = 11,
              F_IMM = 12, F_SEG = 13;
// Stream state words (noise/fold.rs:47-72).
constexpr int S_MEDIAN = 0, S_LOW = 3, S_LOW_UNB = 6, S_TEMPORAL = 9, S_RHO_VALID = 12, S_RHO = 13, S_CURVE = 14,
              S_QUARTER = 15, S_RATIOS = 16;
// Derived words (noise/derived.rs:9-31).
constexpr int D_SIGMA = 0, D_WEIGHT = 2, D_CURVE = 3, D_SAD = 4, D_CONF_SAD = 5, D_H2 = 6, D_PILOT_H2 = 7,
              D_OFFSET = 8, D_INPUT_OFFSET = 9, D_RHO = 10;
// Correlation table (noise/correlation.rs:7-8).
constexpr float RHO_T[4] = {0.0f, 0.3f, 0.5f, 0.65f};
constexpr float FAC_T[4] = {1.0f, 1.05f, 1.25f, 1.45f};

int record_len(int c) { return 3 * c + 26; }
int texture_lane(int channels, int c) { return c == 0 ? 2 * channels + 1 : 2 * channels + 3 + 24 + c - 1; }

float quartile_from_pair(float low, float high, uint32_t count) {
    const uint32_t last = std::max<uint32_t>(count, 1u) - 1u;
    const float fraction = static_cast<float>(last % 4u) * 0.25f;
    return low + fraction * (high - low);
}
float median_from_pair(float low, float high) { return (low + high) * 0.5f; }

// The value and count of an order statistic over `v` (sorted ascending): an empty set gives 0.
struct Sel {
    std::vector<float> v;
    void done() { std::sort(v.begin(), v.end()); }
    uint32_t n() const { return static_cast<uint32_t>(v.size()); }
    float at(uint32_t rank) const { return rank < v.size() ? v[rank] : 0.0f; }
    float median_low() const { return n() ? at((n() - 1) / 2) : 0.0f; }
    float median_high() const { return n() ? at(n() / 2) : 0.0f; }
    float quartile_low() const { return n() ? at((n() - 1) / 4) : 0.0f; }
    float quartile_high() const { return n() ? at((n() + 2) / 4) : 0.0f; }
    float first() const { return n() ? v.front() : 0.0f; }
    float last() const { return n() ? v.back() : 0.0f; }
    float texture_share() const { return n() ? at((n() - 1) * 2 / 5) : 0.0f; }
};

// The luma quarter fields of a temporal record (noise/temporal.rs:20-62).
constexpr int QUARTERS = 4, QUARTER_SIZE = 8, QUARTER_FIELDS = 6, QUARTER_BASE = 3;
constexpr int Q_SUM_D = 0, Q_SUM_D2 = 1, Q_LUMA_SUM = 2, Q_FLATNESS = 3, Q_LUMA_MIN = 4, Q_LUMA_MAX = 5;
constexpr float UNMEASURED_FLATNESS = 3.0e38f;

// kernels/stats.rs:466-606: the four 8x8 quarters' fields of one block, from its 256 threads
// (t = ly * 16 + lx): whether the pixel is read, its new luma, the mean of its new and previous
// luma, and its channel-0 residual. Each quarter's 64 values sit at slot quarter * 64 + (ly % 8) * 8
// + lx % 8 and fold in halving rounds of stride 32, 16, ..., 1. The flatness averages the mean luma
// over 2x2 pixels into an 8x8 grid of cells; each cell adds its squared difference to its right and
// lower neighbour inside the quarter, and the quarter's 16 cell sums fold in halving rounds of 8, 4,
// 2, 1 and are divided by its 24 pairs. A quarter not wholly inside the frame reads
// UNMEASURED_FLATNESS; an unmatched block (a compensated block leaving the frame) writes zeros.
void quarter_fields(float* out, int channels, int bw, int bh, bool matched, const bool* valid, const float* new_luma,
                    const float* mean_luma, const float* d0) {
    float sum[256], lo[256], hi[256], rd[256], rq[256], cells[64], pairs[64];
    for (int t = 0; t < 256; ++t) {
        const int lx = t % NB, ly = t / NB;
        const int slot = ((ly / 8) * 2 + lx / 8) * 64 + (ly % 8) * 8 + lx % 8;
        const float d = valid[t] ? d0[t] : 0.0f;
        sum[slot] = valid[t] ? new_luma[t] : 0.0f;
        lo[slot] = valid[t] ? new_luma[t] : 1.0e30f;
        hi[slot] = valid[t] ? new_luma[t] : -1.0e30f;
        rd[slot] = d;
        rq[slot] = d * d;
    }
    for (int stride = 32; stride >= 1; stride >>= 1)
        for (int q = 0; q < QUARTERS; ++q)
            for (int p = 0; p < stride; ++p) {
                const int here = q * 64 + p, there = here + stride;
                sum[here] += sum[there];
                rd[here] += rd[there];
                rq[here] += rq[there];
                lo[here] = std::min(lo[here], lo[there]);
                hi[here] = std::max(hi[here], hi[there]);
            }
    for (int t = 0; t < 64; ++t) {
        const int cy = t / 8, cx = t % 8;
        float cell = 0.0f;
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                const int i = (2 * cy + dy) * NB + 2 * cx + dx;
                cell += valid[i] ? mean_luma[i] : 0.0f;
            }
        cells[t] = cell / 4.0f;
    }
    for (int t = 0; t < 64; ++t) {
        const int cy = t / 8, cx = t % 8;
        const float here = cells[t];
        float energy = 0.0f;
        if (cx % 4 != 3) {
            const float s = here - cells[t + 1];
            energy += s * s;
        }
        if (cy % 4 != 3) {
            const float s = here - cells[t + 8];
            energy += s * s;
        }
        pairs[((cy / 4) * 2 + cx / 4) * 16 + (cy % 4) * 4 + cx % 4] = energy;
    }
    for (int stride = 8; stride >= 1; stride >>= 1)
        for (int t = 0; t < 64; ++t)
            if (t % 16 < stride) pairs[t] += pairs[t + stride];
    for (int q = 0; q < QUARTERS; ++q) {
        float* f = out + 2 * channels + QUARTER_BASE + q * QUARTER_FIELDS;
        if (!matched) {
            std::fill(f, f + QUARTER_FIELDS, 0.0f);
            continue;
        }
        const bool full = bw >= (q % 2 + 1) * QUARTER_SIZE && bh >= (q / 2 + 1) * QUARTER_SIZE;
        f[Q_SUM_D] = rd[q * 64];
        f[Q_SUM_D2] = rq[q * 64];
        f[Q_LUMA_SUM] = sum[q * 64];
        f[Q_FLATNESS] = full ? pairs[q * 16] / 24.0f : UNMEASURED_FLATNESS;
        f[Q_LUMA_MIN] = lo[q * 64];
        f[Q_LUMA_MAX] = hi[q * 64];
    }
}

}  // namespace

extern "C" {

int orc_noise_record_len(int channels) { return record_len(channels); }

// noise/temporal.rs:83-100 (`min_static_blocks`).
uint32_t orc_min_static_blocks(uint32_t total) {
    const float t = static_cast<float>(total);
    auto reaches = [&](uint32_t a) { return static_cast<float>(a) / t >= STATIC_FRACTION_MIN; };
    uint32_t a = std::min<uint32_t>(static_cast<uint32_t>(STATIC_FRACTION_MIN * t), total);
    while (a > 0 && reaches(a - 1)) --a;
    while (a < total && !reaches(a)) ++a;
    return a;
}

// The records of `next` (its previous frame `prev`), both channel-interleaved f32 frames.
void orc_temporal_stats(const float* next, const float* prev, int channels, int w, int h, int luma_fields,
                        float* records) {
    const int bxn = (w + NB - 1) / NB, byn = (h + NB - 1) / NB, rl = record_len(channels);
    const int lanes = 2 * channels + 1;
    std::vector<float> scratch(256 * lanes), tile(256), cells(16);
    for (int by = 0; by < byn; ++by)
        for (int bx = 0; bx < bxn; ++bx) {
            const int bw = std::min(NB, w - bx * NB), bh = std::min(NB, h - by * NB);
            float* out = records + static_cast<int64_t>(by * bxn + bx) * rl;
            std::fill(out, out + rl, 0.0f);
            std::vector<float> d0(256, 0.0f);
            auto value = [&](const float* f, int x, int y, int c) {
                return f[(static_cast<int64_t>(y) * w + x) * channels + c];
            };
            for (int t = 0; t < 256; ++t) {
                const int lx = t % NB, ly = t / NB, gx = bx * NB + lx, gy = by * NB + ly;
                const bool valid = gx < w && gy < h;
                for (int c = 0; c < channels; ++c) {
                    const float r = valid ? value(next, gx, gy, c) - value(prev, gx, gy, c) : 0.0f;
                    scratch[t * lanes + c] = r;
                    scratch[t * lanes + channels + c] = r * r;
                    if (c == 0) d0[t] = r;
                }
            }
            for (int t = 0; t < 256; ++t) {
                const int lx = t % NB, gx = bx * NB + lx, gy = by * NB + t / NB;
                const bool valid = gx < w && gy < h;
                scratch[t * lanes + 2 * channels] = (valid && lx + 1 < bw) ? d0[t] * d0[t + 1] : 0.0f;
            }
            for (int lane = 0; lane < lanes; ++lane) {
                float total = 0.0f;
                for (int t = 0; t < 256; ++t) total += scratch[t * lanes + lane];
                out[lane] = total;
            }
            for (int c = 0; c < channels; ++c) {
                for (int t = 0; t < 256; ++t) {
                    const int gx = bx * NB + t % NB, gy = by * NB + t / NB;
                    tile[t] = (gx < w && gy < h) ? value(next, gx, gy, c) : 0.0f;
                }
                for (int i = 0; i < 16; ++i) {
                    const int cx = i % 4, cy = i / 4;
                    float cell = 0.0f;
                    for (int dy = 0; dy < 4; ++dy)
                        for (int dx = 0; dx < 4; ++dx) cell += tile[(4 * cy + dy) * NB + 4 * cx + dx];
                    cells[i] = cell / 16.0f;
                }
                const int cols = bw / 4, rows = bh / 4;
                float energy = 0.0f;
                uint32_t pairs = 0;
                for (int cy = 0; cy < rows; ++cy)
                    for (int cx = 0; cx < cols; ++cx) {
                        const float here = cells[cy * 4 + cx];
                        if (cx + 1 < cols) {
                            const float s = here - cells[cy * 4 + cx + 1];
                            energy += s * s;
                            ++pairs;
                        }
                        if (cy + 1 < rows) {
                            const float s = here - cells[(cy + 1) * 4 + cx];
                            energy += s * s;
                            ++pairs;
                        }
                    }
                out[texture_lane(channels, c)] = pairs ? energy / static_cast<float>(pairs) : 0.0f;
            }
            if (luma_fields) {
                bool valid[256];
                float nl[256], ml[256];
                for (int t = 0; t < 256; ++t) {
                    const int gx = bx * NB + t % NB, gy = by * NB + t / NB;
                    valid[t] = gx < w && gy < h;
                    nl[t] = valid[t] ? value(next, gx, gy, 0) : 0.0f;
                    ml[t] = valid[t] ? 0.5f * (nl[t] + value(prev, gx, gy, 0)) : 0.0f;
                }
                quarter_fields(out, channels, bw, bh, true, valid, nl, ml, d0.data());
            }
        }
}

// The records of `next` against `prev` along a motion field (kernels/stats.rs:224-330, the
// `compensated` variant): each block reads the whole-pixel vector of the motion block covering its
// origin (`mv`: (dx, dy) per block of an mv_bx x mv_by grid at `step`), follows it only when its
// channel-0 residual variance along it is at most 0.5 of the zero-vector variance (or nothing of
// it matches inside the frame), and writes an all-zero record when the followed block leaves the
// frame. The four variance sums are halving-tree reductions over the block's 256 threads.
void orc_temporal_stats_mc(const float* next, const float* prev, int channels, int w, int h, const int32_t* mv,
                           int mv_bx, int mv_by, int step, int luma_fields, float* records) {
    const int bxn = (w + NB - 1) / NB, byn = (h + NB - 1) / NB, rl = record_len(channels);
    const int lanes = 2 * channels + 1;
    auto value = [&](const float* f, int x, int y, int c) { return f[(static_cast<int64_t>(y) * w + x) * channels + c]; };
    std::vector<float> runs(4 * 256), scratch(256 * lanes), tile(256), cells(16), d0(256);
    for (int by = 0; by < byn; ++by)
        for (int bx = 0; bx < bxn; ++bx) {
            const int x0 = bx * NB, y0 = by * NB;
            const int bw = std::min(NB, w - x0), bh = std::min(NB, h - y0);
            float* out = records + static_cast<int64_t>(by * bxn + bx) * rl;
            const int col = std::min(x0 / step, mv_bx - 1), row = std::min(y0 / step, mv_by - 1);
            const int vx = mv[(row * mv_bx + col) * 2], vy = mv[(row * mv_bx + col) * 2 + 1];
            for (int t = 0; t < 256; ++t) {
                const int gx = x0 + t % NB, gy = y0 + t / NB;
                float zr = 0.0f, vr = 0.0f;
                if (gx < w && gy < h) {
                    const float nl = value(next, gx, gy, 0);
                    zr = nl - value(prev, gx, gy, 0);
                    const int mx = gx + vx, my = gy + vy;
                    if (mx >= 0 && mx < w && my >= 0 && my < h) vr = nl - value(prev, mx, my, 0);
                }
                runs[t] = zr;
                runs[256 + t] = zr * zr;
                runs[512 + t] = vr;
                runs[768 + t] = vr * vr;
            }
            for (int stride = 128; stride >= 1; stride >>= 1)
                for (int t = 0; t < stride; ++t)
                    for (int r = 0; r < 4; ++r) runs[r * 256 + t] += runs[r * 256 + t + stride];
            const int left = x0 + vx, top = y0 + vy, right = left + bw, bottom = top + bh;
            const int ow = std::max(std::min(right, w) - std::max(left, 0), 0);
            const int oh = std::max(std::min(bottom, h) - std::max(top, 0), 0);
            const float matched_pixels = static_cast<float>(ow * oh), block_pixels = static_cast<float>(bw * bh);
            const float zero_mean = runs[0] / block_pixels;
            const float zero_var = runs[256] / block_pixels - zero_mean * zero_mean;
            const float safe = std::max(matched_pixels, 1.0f);
            const float vec_mean = runs[512] / safe;
            const float vec_var = runs[768] / safe - vec_mean * vec_mean;
            const bool has_vector = vx != 0 || vy != 0;
            const bool follows = has_vector && (matched_pixels == 0.0f || vec_var <= 0.5f * zero_var);
            int sx = 0, sy = 0;
            bool matched = true;
            if (follows) {
                sx = vx;
                sy = vy;
                matched = left >= 0 && right <= w && top >= 0 && bottom <= h;
            }
            std::fill(out, out + rl, 0.0f);
            for (int t = 0; t < 256; ++t) {
                const int lx = t % NB, gx = x0 + lx, gy = y0 + t / NB;
                const bool valid = gx < w && gy < h && matched;
                for (int c = 0; c < channels; ++c) {
                    const float r = valid ? value(next, gx, gy, c) - value(prev, gx + sx, gy + sy, c) : 0.0f;
                    scratch[t * lanes + c] = r;
                    scratch[t * lanes + channels + c] = r * r;
                    if (c == 0) d0[t] = r;
                }
            }
            for (int t = 0; t < 256; ++t) {
                const int lx = t % NB, gx = x0 + lx, gy = y0 + t / NB;
                const bool valid = gx < w && gy < h && matched;
                scratch[t * lanes + 2 * channels] = (valid && lx + 1 < bw) ? d0[t] * d0[t + 1] : 0.0f;
            }
            for (int lane = 0; lane < lanes; ++lane) {
                float total = 0.0f;
                for (int t = 0; t < 256; ++t) total += scratch[t * lanes + lane];
                out[lane] = total;
            }
            for (int c = 0; c < channels; ++c) {
                for (int t = 0; t < 256; ++t) {
                    const int gx = x0 + t % NB, gy = y0 + t / NB;
                    tile[t] = (gx < w && gy < h && matched) ? value(next, gx, gy, c) : 0.0f;
                }
                for (int i = 0; i < 16; ++i) {
                    const int cx = i % 4, cy = i / 4;
                    float cell = 0.0f;
                    for (int dy = 0; dy < 4; ++dy)
                        for (int dx = 0; dx < 4; ++dx) cell += tile[(4 * cy + dy) * NB + 4 * cx + dx];
                    cells[i] = cell / 16.0f;
                }
                const int cols = bw / 4, rows = bh / 4;
                float energy = 0.0f;
                uint32_t pairs = 0;
                for (int cy = 0; cy < rows; ++cy)
                    for (int cx = 0; cx < cols; ++cx) {
                        const float here = cells[cy * 4 + cx];
                        if (cx + 1 < cols) {
                            const float s = here - cells[cy * 4 + cx + 1];
                            energy += s * s;
                            ++pairs;
                        }
                        if (cy + 1 < rows) {
                            const float s = here - cells[(cy + 1) * 4 + cx];
                            energy += s * s;
                            ++pairs;
                        }
                    }
                out[texture_lane(channels, c)] = pairs ? energy / static_cast<float>(pairs) : 0.0f;
            }
            out[2 * channels + 2] = (follows && matched) ? 1.0f : 0.0f;
            if (luma_fields) {
                bool valid[256];
                float nl[256], ml[256];
                for (int t = 0; t < 256; ++t) {
                    const int gx = x0 + t % NB, gy = y0 + t / NB;
                    valid[t] = gx < w && gy < h && matched;
                    nl[t] = valid[t] ? value(next, gx, gy, 0) : 0.0f;
                    ml[t] = valid[t] ? 0.5f * (nl[t] + value(prev, gx + sx, gy + sy, 0)) : 0.0f;
                }
                quarter_fields(out, channels, bw, bh, matched, valid, nl, ml, d0.data());
            }
        }
}

// One slot's reading (READING_WORDS floats). `records` may be null without temporal stats;
// `imm_low` holds the two Immerkaer lower quartiles (the quartile of the cube sigmas).
void orc_noise_reading(const float* records, const float* imm_low, int channels, int w, int h, int temporal,
                       int curve, float* reading) {
    std::fill(reading, reading + R_WORDS, 0.0f);
    reading[R_IMM_LOW] = imm_low[0];
    reading[R_IMM_LOW + 1] = imm_low[1];
    if (!temporal || !records) return;
    const int bxn = (w + NB - 1) / NB, byn = (h + NB - 1) / NB, nblocks = bxn * byn, rl = record_len(channels);
    struct Block {
        float sigma[NOISE_CHANNELS] = {0, 0}, mean[NOISE_CHANNELS] = {0, 0}, texture[NOISE_CHANNELS] = {0, 0};
        float var0 = 0, mean_lag = 0, pairs = 0;
        bool candidate[NOISE_CHANNELS] = {false, false};
        bool moved = false;
    };
    std::vector<Block> blocks(nblocks);
    Sel ref[NOISE_CHANNELS], moved_tex[NOISE_CHANNELS];
    uint32_t excluded[NOISE_CHANNELS] = {0, 0};
    for (int i = 0; i < nblocks; ++i) {
        const int bx = i % bxn, by = i / bxn;
        const int bw = std::min(NB, w - bx * NB), bh = std::min(NB, h - by * NB);
        const float pixels = static_cast<float>(bw * bh), pairs = static_cast<float>(bh * (bw - 1));
        const float* r = records + static_cast<int64_t>(i) * rl;
        Block& b = blocks[i];
        b.moved = r[2 * channels + 2] != 0.0f;
        for (int c = 0; c < channels; ++c) {
            const float mean = r[c] / pixels;
            const float ms = r[channels + c] / pixels;
            const float var = std::max(ms - mean * mean, 0.0f);
            const float sigma = std::sqrt(var) / SQRT_2F;
            b.sigma[c] = sigma;
            b.mean[c] = mean;
            b.texture[c] = r[texture_lane(channels, c)];
            b.candidate[c] = std::fabs(mean) < STATIC_GATE;
            const bool measurable = sigma > RHO_SIGMA_GATE;
            if (b.candidate[c]) {
                if (measurable)
                    ref[c].v.push_back(sigma);
                else
                    excluded[c] += 1;
                if (measurable && b.moved) moved_tex[c].v.push_back(b.texture[c]);
            }
            if (c == 0) b.var0 = var;
        }
        b.pairs = pairs;
        b.mean_lag = pairs > 0.0f ? r[2 * channels] / pairs : 0.0f;
    }
    float ceiling[NOISE_CHANNELS] = {0, 0}, threshold[NOISE_CHANNELS] = {0, 0};
    bool trusted[NOISE_CHANNELS] = {false, false};
    for (int c = 0; c < channels; ++c) {
        ref[c].done();
        moved_tex[c].done();
        const float q = quartile_from_pair(ref[c].quartile_low(), ref[c].quartile_high(), ref[c].n());
        ceiling[c] = ref[c].n() ? q * SIGMA_OUTLIER_FACTOR : 0.0f;
        const bool spread = ref[c].n() > 0 && ref[c].last() > ref[c].first();
        trusted[c] = excluded[c] == 0 || spread;
        threshold[c] = moved_tex[c].texture_share();
    }
    Sel kept[NOISE_CHANNELS], rho;
    uint32_t accepted[NOISE_CHANNELS] = {0, 0};
    std::vector<bool> block_accepted(nblocks, false);
    for (int i = 0; i < nblocks; ++i) {
        const Block& b = blocks[i];
        bool accepted0 = false;
        for (int c = 0; c < channels; ++c) {
            const float s = b.sigma[c];
            const bool acc = trusted[c] && b.candidate[c] && s <= ceiling[c] && s > RHO_SIGMA_GATE;
            const bool textured = b.moved && moved_tex[c].n() > 0 && b.texture[c] > threshold[c];
            if (acc && !textured) kept[c].v.push_back(s);
            if (acc) accepted[c] += 1;
            if (c == 0) accepted0 = acc;
        }
        block_accepted[i] = accepted0;
        const bool has_rho = accepted0 && b.pairs > 0.0f;
        const float variance = has_rho ? b.var0 : 1.0f;
        const float r = (b.mean_lag - b.mean[0] * b.mean[0]) / variance;
        if (has_rho) rho.v.push_back(std::min(std::max(r, 0.0f), 1.0f));
    }
    for (auto& k : kept) k.done();
    rho.done();
    const uint32_t min_acc = orc_min_static_blocks(static_cast<uint32_t>(nblocks));
    auto channel_valid = [&](int c) { return c < channels && accepted[c] >= min_acc && kept[c].n() > 0; };
    const bool valid0 = rho.n() > 0 && channel_valid(0);
    const float static_fraction = static_cast<float>(accepted[0]) / static_cast<float>(nblocks);
    for (int c = 0; c < NOISE_CHANNELS; ++c) {
        const bool k = c == 0 ? valid0 : channel_valid(c);
        const float sigma = median_from_pair(kept[c].median_low(), kept[c].median_high());
        const float low = quartile_from_pair(kept[c].quartile_low(), kept[c].quartile_high(), kept[c].n());
        reading[R_VALID + c] = k ? 1.0f : 0.0f;
        reading[R_SIGMA + c] = k ? sigma : 0.0f;
        reading[R_SIGMA_LOW + c] = k ? low : 0.0f;
    }
    reading[R_RHO] = valid0 ? median_from_pair(rho.median_low(), rho.median_high()) : 0.0f;
    reading[R_STATIC] = valid0 ? static_fraction : 0.0f;
    reading[R_ACCEPTED] = static_cast<float>(accepted[0]);
    if (!curve) return;

    // The noise curve (kernels/sample.rs:95-104, 482-510, 717-803; kernels/curve.rs:37-133). The
    // flat gate scales with channel 0's kept sigma median.
    const float sigma_median = median_from_pair(kept[0].median_low(), kept[0].median_high());
    const float flat_limit = std::max(FLAT_FACTOR * sigma_median * sigma_median, FLAT_FLOOR);
    Sel quarters, bins[CURVE_BINS];
    for (int i = 0; i < nblocks; ++i) {
        if (!block_accepted[i]) continue;
        const int bx = i % bxn, by = i / bxn;
        const int bw = std::min(NB, w - bx * NB), bh = std::min(NB, h - by * NB);
        const float* r = records + static_cast<int64_t>(i) * rl;
        for (int q = 0; q < QUARTERS; ++q) {
            const int qw = std::min(std::max(bw - (q % 2) * QUARTER_SIZE, 0), QUARTER_SIZE);
            const int qh = std::min(std::max(bh - (q / 2) * QUARTER_SIZE, 0), QUARTER_SIZE);
            const float pixels = static_cast<float>(qw * qh);
            const float* f = r + 2 * channels + QUARTER_BASE + q * QUARTER_FIELDS;
            const float divisor = pixels > 0.0f ? pixels : 1.0f;
            const float mean = f[Q_SUM_D] / divisor;
            const float ms = f[Q_SUM_D2] / divisor;
            const float sigma = std::sqrt(std::max(ms - mean * mean, 0.0f)) / SQRT_2F;
            const bool passes = pixels > 0.0f && std::fabs(mean) < QUARTER_STATIC_GATE && sigma > RHO_SIGMA_GATE;
            if (!passes) continue;
            quarters.v.push_back(sigma);
            const float mean_luma = f[Q_LUMA_SUM] / divisor;
            const float scaled = std::max(mean_luma * static_cast<float>(CURVE_BINS), 0.0f);
            const int bin = static_cast<int>(std::min(scaled, static_cast<float>(CURVE_BINS - 1)));
            const bool textured = f[Q_FLATNESS] > flat_limit;
            const bool clipped = f[Q_LUMA_MIN] < CLIP_LOW || f[Q_LUMA_MAX] > CLIP_HIGH;
            if (!textured && !clipped) bins[bin].v.push_back(sigma);
        }
    }
    quarters.done();
    for (auto& b : bins) b.done();
    const float quarter_median = median_from_pair(quarters.median_low(), quarters.median_high());
    // curve_bin_sigma: flat before the first and after the last populated bin, linear between the
    // nearest populated bin below and the nearest at or above.
    uint32_t populated = 0;
    int first_index = 0, last_index = 0;
    float first_sigma = 0.0f, last_sigma = 0.0f, medians[CURVE_BINS];
    for (int b = 0; b < CURVE_BINS; ++b) {
        medians[b] = median_from_pair(bins[b].median_low(), bins[b].median_high());
        if (bins[b].n() < MIN_BIN_QUARTERS) continue;
        if (populated == 0) {
            first_index = b;
            first_sigma = medians[b];
        }
        last_index = b;
        last_sigma = medians[b];
        ++populated;
    }
    const bool curve_valid = valid0 && quarters.n() > 0 && quarter_median > 0.0f && populated >= MIN_POPULATED_BINS;
    const float divisor = curve_valid ? quarter_median : 1.0f;
    for (int bin = 0; bin < CURVE_BINS; ++bin) {
        int low_index = 0, high_index = 0;
        float low_sigma = 0.0f, high_sigma = 0.0f;
        bool has_high = false;
        for (int b = 0; b < CURVE_BINS; ++b) {
            if (bins[b].n() < MIN_BIN_QUARTERS) continue;
            if (b < bin) {
                low_index = b;
                low_sigma = medians[b];
            }
            if (b >= bin && !has_high) {
                high_index = b;
                high_sigma = medians[b];
                has_high = true;
            }
        }
        const int span_bins = high_index > low_index ? high_index - low_index : 1;
        const int offset_bins = bin - std::min(low_index, bin);
        const float fraction = static_cast<float>(offset_bins) / static_cast<float>(span_bins);
        const float between = low_sigma + (high_sigma - low_sigma) * fraction;
        const float sigma = bin <= first_index ? first_sigma : (bin >= last_index ? last_sigma : between);
        reading[R_RATIOS + bin] = curve_valid ? sigma / divisor : 0.0f;
    }
    reading[R_CURVE_VALID] = curve_valid ? 1.0f : 0.0f;
    reading[R_QUARTER_MEDIAN] = curve_valid ? quarter_median : 0.0f;
    reading[R_POPULATED] = static_cast<float>(populated);
}

// kernels/derive.rs:46-64 (`correlation_factor`) with the host's segment reciprocals.
float orc_correlation_factor(float rho, const float* settings) {
    const float x = std::min(std::max(rho, RHO_T[0]), RHO_T[3]);
    const float f0 = (x - RHO_T[0]) * settings[F_SEG];
    const float f1 = (x - RHO_T[1]) * settings[F_SEG + 1];
    const float f2 = (x - RHO_T[2]) * settings[F_SEG + 2];
    const float first = FAC_T[0] + f0 * (FAC_T[1] - FAC_T[0]);
    const float second = FAC_T[1] + f1 * (FAC_T[2] - FAC_T[1]);
    const float third = FAC_T[2] + f2 * (FAC_T[3] - FAC_T[2]);
    const float later = x <= RHO_T[2] ? second : third;
    return x <= RHO_T[1] ? first : later;
}

// kernels/derive.rs:66-82 (`spatial_offset_factor`), exp and ln in double precision.
float orc_spatial_offset_factor(int dx, int dy, float rho) {
    const int sq = dx * dx + dy * dy;
    if (sq == 0) return 0.0f;
    if (rho <= 0.0f) return 1.0f;
    const float distance = std::sqrt(static_cast<float>(sq));
    const float log_rho = static_cast<float>(std::log(static_cast<double>(rho)));
    const float shared = static_cast<float>(std::exp(static_cast<double>(distance * log_rho)));
    return 1.0f - shared;
}

// noise/fold.rs:118-146 (`fold_words`): the fold settings for a plane of w x h.
void orc_fold_words(int w, int h, float sigma_scale, int curve_applies, float g_max, float weight_floor, int h2_auto,
                    float h2_per_inverse_variance, float h2_fixed, float pilot_h2_factor, float offset_per_variance,
                    int main_offset, float sad_per_sigma, float confidence_sad_per_sigma, float immerkaer_scale,
                    float* words) {
    std::fill(words, words + 16, 0.0f);
    const float interior = static_cast<float>(w - 2) * static_cast<float>(h - 2);
    const float divisor = 6.0f * interior;
    words[F_SIGMA_SCALE] = sigma_scale;
    words[F_CURVE_APPLIES] = curve_applies ? 1.0f : 0.0f;
    words[F_G_MAX] = g_max;
    words[F_W_FLOOR] = weight_floor;
    words[F_H2_AUTO] = h2_auto ? 1.0f : 0.0f;
    words[F_H2_PIV] = h2_auto ? h2_per_inverse_variance : 0.0f;
    words[F_H2_FIXED] = h2_fixed;
    words[F_PILOT] = pilot_h2_factor;
    words[F_OFFSET_PV] = offset_per_variance;
    words[F_MAIN_OFFSET] = main_offset ? 1.0f : 0.0f;
    words[F_SAD] = sad_per_sigma;
    words[F_CONF_SAD] = confidence_sad_per_sigma;
    words[F_IMM] = immerkaer_scale / divisor;
    for (int i = 0; i < 3; ++i) words[F_SEG + i] = 1.0f / (RHO_T[i + 1] - RHO_T[i]);
}

// kernels/window.rs:414-498 (`noise_window_fold`) over history frames first..=last.
void orc_noise_fold(const float* records, const float* results, int capacity, int first, int last,
                    const float* settings, int channels, int table_radius, float* state, float* derived,
                    float* spatial_table, float* pilot_table) {
    auto rec = [&](int frame) { return records + static_cast<int64_t>(frame % capacity) * R_WORDS; };
    auto has_sample = [&](int frame, int c) { return rec(frame)[R_VALID + c] != 0.0f; };
    auto has_curve = [&](int frame) { return rec(frame)[R_CURVE_VALID] != 0.0f; };
    auto sorted_median = [](std::vector<float>& v) {
        // Insertion sort, as the kernel's (window.rs:103-135).
        for (size_t i = 1; i < v.size(); ++i) {
            const float key = v[i];
            size_t p = i;
            while (p > 0 && v[p - 1] > key) {
                v[p] = v[p - 1];
                --p;
            }
            v[p] = key;
        }
        if (v.empty()) return 0.0f;
        const size_t n = v.size();
        return (v[(n - 1) / 2] + v[n / 2]) * 0.5f;
    };
    uint32_t sampled = 0, curved = 0;
    for (int f = first; f <= last; ++f) {
        sampled += has_sample(f, 0) ? 1 : 0;
        curved += (has_sample(f, 0) && has_curve(f)) ? 1 : 0;
    }
    const bool curve_present = sampled > 0 && 2 * curved >= sampled;
    const float sigma_scale = settings[F_SIGMA_SCALE], imm_factor = settings[F_IMM];
    auto chain_reading = [&](int frame, int chain, int c) {
        const float* r = rec(frame);
        const bool has = r[R_VALID + c] != 0.0f;
        const float factor = orc_correlation_factor(r[R_RHO], settings);
        const float abs_sum = results[static_cast<int64_t>(frame % capacity) * 2 + c];
        const float immerkaer = imm_factor * abs_sum;
        const float imm_low = r[R_IMM_LOW + c], sigma = r[R_SIGMA + c], sigma_low = r[R_SIGMA_LOW + c];
        const float boosted = std::max(immerkaer, sigma * factor);
        const float boosted_low = std::max(imm_low, sigma_low * factor);
        const float unboosted_low = std::max(imm_low, sigma_low);
        const float raw = (has ? boosted : immerkaer) * sigma_scale;
        const float raw_low = (has ? boosted_low : imm_low) * sigma_scale;
        const float raw_unboosted = (has ? unboosted_low : imm_low) * sigma_scale;
        const float raw_temporal = sigma * sigma_scale;
        switch (chain) {
            case 0: return raw;
            case 1: return raw_low;
            case 2: return raw_unboosted;
            default: return raw_temporal;
        }
    };
    float medians[4][NOISE_CHANNELS] = {};
    for (int chain = 0; chain < 4; ++chain)
        for (int c = 0; c < NOISE_CHANNELS; ++c) {
            if (c >= channels) continue;
            std::vector<float> v;
            for (int f = first; f <= last; ++f)
                if (chain != 3 || has_sample(f, c)) v.push_back(chain_reading(f, chain, c));
            const float m = sorted_median(v);
            medians[chain][c] = v.empty() ? 0.0f : std::max(m, SIGMA_FLOOR);
        }
    auto gated = [&](int word, bool curve_gate) {
        std::vector<float> v;
        for (int f = first; f <= last; ++f)
            if (has_sample(f, 0) && (!curve_gate || has_curve(f))) v.push_back(rec(f)[word]);
        return sorted_median(v);
    };
    const float rho_median = gated(R_RHO, false);
    const float quarter_median = gated(R_QUARTER_MEDIAN, true);
    float ratio_median[16];
    for (int b = 0; b < 16; ++b) ratio_median[b] = gated(R_RATIOS + b, true);
    uint32_t mask = sampled > 0 ? 1u : 0u;
    for (int c = 1; c < channels; ++c) {
        bool any = false;
        for (int f = first; f <= last; ++f) any = any || has_sample(f, c);
        if (any) mask |= 1u << c;
    }
    const bool rho_valid = (mask & 1u) != 0, any_sampled = mask != 0;
    for (int c = 0; c < NOISE_CHANNELS; ++c) {
        const bool sampled_c = (mask & (1u << c)) != 0;
        const float fallback = any_sampled ? medians[2][c] : 0.0f;
        state[S_MEDIAN + 1 + c] = medians[0][c];
        state[S_LOW + 1 + c] = medians[1][c];
        state[S_LOW_UNB + 1 + c] = medians[2][c];
        state[S_TEMPORAL + 1 + c] = sampled_c ? medians[3][c] : fallback;
        derived[D_SIGMA + c] = sampled_c ? medians[3][c] : medians[2][c];
    }
    float median_sum = 0.0f, low_sum = 0.0f;
    for (int c = 0; c < channels; ++c) {
        median_sum += medians[0][c] * medians[0][c];
        low_sum += medians[1][c] * medians[1][c];
    }
    const float rho = rho_valid ? rho_median : 0.0f;
    state[S_MEDIAN] = 1.0f;
    state[S_LOW] = 1.0f;
    state[S_LOW_UNB] = 1.0f;
    state[S_TEMPORAL] = any_sampled ? 1.0f : 0.0f;
    state[S_RHO_VALID] = rho_valid ? 1.0f : 0.0f;
    state[S_RHO] = rho;
    state[S_CURVE] = curve_present ? 1.0f : 0.0f;
    state[S_QUARTER] = curve_present ? quarter_median : 0.0f;
    const bool curve_valid = curve_present && settings[F_CURVE_APPLIES] != 0.0f;
    for (int b = 0; b < 16; ++b) state[S_RATIOS + b] = curve_present ? ratio_median[b] : 0.0f;
    // kernels/derive.rs:143-192 (`write_derived`).
    const float sigma0 = derived[D_SIGMA];
    const float g_max = settings[F_G_MAX], floor = settings[F_W_FLOOR];
    const float norm = sigma0 * sigma0 * g_max * g_max;
    const bool usable = std::isfinite(norm) && norm > floor;
    const float h2_measured = settings[F_H2_PIV] * static_cast<float>(channels) / median_sum;
    const float h2 = settings[F_H2_AUTO] != 0.0f ? h2_measured : settings[F_H2_FIXED];
    const float input_offset = settings[F_OFFSET_PV] * low_sum;
    const float noise_offset = settings[F_MAIN_OFFSET] != 0.0f ? input_offset : 0.0f;
    derived[D_WEIGHT] = usable ? norm : floor;
    derived[D_CURVE] = curve_valid ? 1.0f : 0.0f;
    derived[D_SAD] = settings[F_SAD] * medians[0][0];
    derived[D_CONF_SAD] = settings[F_CONF_SAD] * medians[0][0];
    derived[D_H2] = h2;
    derived[D_PILOT_H2] = h2 * settings[F_PILOT];
    derived[D_OFFSET] = noise_offset;
    derived[D_INPUT_OFFSET] = input_offset;
    derived[D_RHO] = rho;
    if (table_radius > 0) {
        const int side = 2 * table_radius + 1;
        for (int i = 0; i < side * side; ++i) {
            const int dx = i % side - table_radius, dy = i / side - table_radius;
            spatial_table[i] = noise_offset * orc_spatial_offset_factor(dx, dy, rho);
            pilot_table[i] = input_offset * orc_spatial_offset_factor(dx, dy, 0.0f);
        }
    }
}

}  // extern "C"
