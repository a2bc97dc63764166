// CPU ORACLE - test infrastructure only (see nlm_oracle.cpp for the rules it follows).
//
// A C++17 restatement of av-denoise's block-matching motion search with its camera-model candidate
// (a second window around each neighbour's prediction, motion/kernels/candidates.rs), and of the
// truemotion stage that can end it:
//   pyramid: av-denoise-core/src/motion/kernels/pyramid.rs:10-61 (lane-0 extract, 2x2 average,
//            odd edge repeated) and motion/pyramid.rs:82-107 (levels built one after another);
//   coarse:  motion/kernels/block_match.rs:117-215 and motion/analyse.rs:100-150 (the smallest
//            level, blksize max(b/2^l, 2), step max(s/2^l, 1), winner x 2^l seeds the fine blocks
//            of its region, the last coarse block reaching the fine grid's edge);
//   fine:    block_match.rs:274-351 and 490-521 (seeded window, confidence); with `seeded` the field
//            already holds the seeds and the coarse pass is skipped (analyse.rs:273-316, the
//            refine of chained seeds);
//   window:  block_match.rs:656-849 (clamped staging, SAD summed row by row left to right, lowest
//            SAD with the first row-major index, the window's centre winning a tie, SADs at or
//            above 1e30 never chosen);
//   truemotion: motion/truemotion/kernels/truemotion/{mod.rs,candidates.rs,score.rs} and
//            truemotion/stage.rs (one pass: candidates own, 3x3 lower median, left/right/up/down,
//            zero, the block's coarse seed and its four diagonal seeds; SAD + lambda per pixel of
//            L1 distance from the median, a surcharge off the median, the early settle, the refine
//            ring around a new best; each candidate's SAD summed per row left to right, then the
//            rows top to bottom).
// Every f32 operation is one rounded operation in the reference's order (the build turns off
// contraction), so the vectors and confidences are expected to match the CUDA path bit for bit.
//
// The pyramid layout is the CUDA path's (level after level, `frame_count` slots per level, each
// slot padded to a multiple of 8 floats), so one buffer describes both.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <cstdint>
#include <cstdint>
#include <vector>

namespace {

int64_t slot_pixels(int w, int h, int level) {
    for (int l = 0; l < level; ++l) {
        w = w / 2 > 1 ? w / 2 : 1;
        h = h / 2 > 1 ? h / 2 : 1;
    }
    return (static_cast<int64_t>(w) * h + 7) / 8 * 8;
}

void level_dims(int w, int h, int level, int* lw, int* lh) {
    for (int l = 0; l < level; ++l) {
        w = w / 2 > 1 ? w / 2 : 1;
        h = h / 2 > 1 ? h / 2 : 1;
    }
    *lw = w;
    *lh = h;
}

int64_t level_base(int w, int h, int frames, int level) {
    int64_t b = 0;
    for (int l = 0; l < level; ++l) b += static_cast<int64_t>(frames) * slot_pixels(w, h, l);
    return b;
}

int clamp_to(int v, int limit) { return v < 0 ? 0 : (v >= limit ? limit - 1 : v); }

struct Level {
    const float* base;  // first value of the level
    int64_t slot;
    int width, height, blksize, step, blocks_x, blocks_y;
};

struct Best {
    int dx, dy;
    float sad;
    float mean;      // the window's mean SAD (block_match.rs:744-751)
    float edge_bar;  // the lowest SAD off the outer ring when the winner sits on it, else 0
    int centre_dx, centre_dy;
};

// block_match.rs:674-760 and 787-849 for one centre: every candidate's SAD summed row-major, the
// lowest SAD with the first row-major index, the centre winning a tie, SADs at or above 1e30 never
// chosen; the mean sums every SAD in row-major order.
Best search_window(const Level& L, int centre_slot, int nbr_slot, int ox, int oy, int cdx, int cdy, int R) {
    const int b = L.blksize, side = 2 * R + 1;
    const float* cf = L.base + centre_slot * L.slot;
    const float* nf = L.base + nbr_slot * L.slot;
    std::vector<float> centre(b * b), sads(side * side);
    for (int py = 0; py < b; ++py)
        for (int px = 0; px < b; ++px)
            centre[py * b + px] =
                cf[static_cast<int64_t>(clamp_to(oy + py, L.height)) * L.width + clamp_to(ox + px, L.width)];
    for (int dy = 0; dy < side; ++dy)
        for (int dx = 0; dx < side; ++dx) {
            float sad = 0.0f;
            for (int iy = 0; iy < b; ++iy)
                for (int ix = 0; ix < b; ++ix) {
                    const int sx = clamp_to(ox + cdx - R + dx + ix, L.width);
                    const int sy = clamp_to(oy + cdy - R + dy + iy, L.height);
                    const float diff = centre[iy * b + ix] - nf[static_cast<int64_t>(sy) * L.width + sx];
                    sad += std::fabs(diff);
                }
            sads[dy * side + dx] = sad;
        }
    Best best{cdx, cdy, 1.0e30f, 0.0f, 0.0f, cdx, cdy};
    for (int i = 0; i < side * side; ++i)
        if (sads[i] < best.sad) {
            best.sad = sads[i];
            best.dx = cdx + i % side - R;
            best.dy = cdy + i / side - R;
        }
    const float centre_sad = sads[R * side + R];
    if (centre_sad <= best.sad) {
        best.sad = centre_sad;
        best.dx = cdx;
        best.dy = cdy;
    }
    float total = 0.0f;
    for (int i = 0; i < side * side; ++i) total += sads[i];
    best.mean = total * (1.0f / static_cast<float>(side * side));
    if (std::abs(best.dx - cdx) == R || std::abs(best.dy - cdy) == R) {
        float bar = 1.0e30f;
        for (int y = 1; y < side - 1; ++y)
            for (int x = 1; x < side - 1; ++x) bar = std::min(bar, sads[y * side + x]);
        best.edge_bar = bar;
    }
    return best;
}

// candidates.rs:71-121 (`model_displacement`): the motion neighbour n's camera model predicts at a
// block's centre on a level `scale` times smaller, capped to the level and rounded half up.
void model_displacement(const float* predictions, int n, int ox, int oy, int blksize, int scale, int lw, int lh,
                        int* dx, int* dy) {
    const float* p = predictions + n * 6;
    const float s = static_cast<float>(scale);
    const int half = blksize / 2;
    const float cx = static_cast<float>(ox + half) * s, cy = static_cast<float>(oy + half) * s;
    const float mx = p[0] * cx + p[1] * cy + p[4];
    const float my = p[2] * cx + p[3] * cy + p[5];
    float ldx = (mx - cx) / s, ldy = (my - cy) / s;
    const float limx = static_cast<float>(lw), limy = static_cast<float>(lh);
    ldx = ldx < -limx ? -limx : (ldx > limx ? limx : ldx);
    ldy = ldy < -limy ? -limy : (ldy > limy ? limy : ldy);
    const float rx = std::floor(ldx + 0.5f), ry = std::floor(ldy + 0.5f);
    *dx = std::isnan(rx) ? 0 : static_cast<int>(rx);
    *dy = std::isnan(ry) ? 0 : static_cast<int>(ry);
}

// candidates.rs:123-134 (`predicts_motion`).
bool predicts_motion(const float* predictions, int n) {
    const float* p = predictions + n * 6;
    return p[0] != 1.0f || p[3] != 1.0f || p[1] != 0.0f || p[2] != 0.0f || p[4] != 0.0f || p[5] != 0.0f;
}

// block_match.rs:213-265 and 384-470 with candidates.rs:136-166: the window around `seed`, then,
// when the model moves anything and its point lies outside that window, the window around the
// model's point, which wins only when its SAD plus `bias` is below the incumbent's.
Best search_with_model(const Level& L, int cs, int ns, int ox, int oy, int sdx, int sdy, int R,
                       const float* predictions, int n, int scale, float bias) {
    Best best = search_window(L, cs, ns, ox, oy, sdx, sdy, R);
    if (!predictions) return best;
    int mdx, mdy;
    model_displacement(predictions, n, ox, oy, L.blksize, scale, L.width, L.height, &mdx, &mdy);
    const bool outside = std::abs(mdx - sdx) > R || std::abs(mdy - sdy) > R;
    if (!(predicts_motion(predictions, n) && outside)) return best;
    const Best ch = search_window(L, cs, ns, ox, oy, mdx, mdy, R);
    if (ch.sad + bias < best.sad) best = ch;
    return best;
}

// analyse.rs:150-157 (`coarse_floor_scale`).
float coarse_floor_scale(int coarse_blksize, int blksize, int scale) {
    const float coarse_area = static_cast<float>(coarse_blksize * coarse_blksize);
    const float fine_area = static_cast<float>(blksize * blksize);
    return coarse_area / fine_area / static_cast<float>(scale);
}

constexpr float kModelCandidateBias = 0.125f;  // candidates.rs:6-11

float match_confidence(float sad, float floor, float thsad) {
    float excess = sad - floor;
    if (excess < 0.0f) excess = 0.0f;
    const float t2 = thsad * thsad, e2 = excess * excess;
    const float c = (t2 - e2) / (t2 + e2);
    return c < 0.0f ? 0.0f : c;
}

// motion/kernels/escalate.rs:14-67: the constants of the escalation stage.
constexpr float kEscalateBelowConfidence = 0.5f;
constexpr int kNeighbourDisagreement = 4;
constexpr float kEscalateSadMargin = 0.125f;
constexpr uint32_t kFloorSamples = 4096, kFloorRankDivisor = 4, kFloorBinShift = 16, kInfinityBin = 0x7F80;
constexpr float kExactMatchSad = 1.0e-6f, kFlatShare = 0.25f;

uint32_t float_bits(float v) {
    uint32_t u;
    std::memcpy(&u, &v, 4);
    return u;
}

float bits_float(uint32_t u) {
    float v;
    std::memcpy(&v, &u, 4);
    return v;
}

// escalate.rs:259-297 (`ranked_bin`): the lowest bin b >= lower with divisor * |{lower <= key <= b}|
// >= |{key >= lower}|, found by the same bisection over [lower, infinity's bin].
uint32_t ranked_bin(const std::vector<uint32_t>& keys, uint32_t lower, uint32_t divisor) {
    auto count = [&](uint32_t lo, uint32_t hi) {
        uint32_t c = 0;
        for (uint32_t k : keys) c += (k >= lo && k <= hi) ? 1u : 0u;
        return c;
    };
    const uint32_t valid = count(lower, 0xFFFFFFFFu);
    uint32_t low = lower, high = kInfinityBin;
    while (low < high) {
        const uint32_t middle = low + (high - low) / 2;
        if (divisor * count(lower, middle) >= valid)
            high = middle;
        else
            low = middle + 1;
    }
    return low;
}

// escalate.rs:168-257 (`mc_measure_floor`) over the kept SADs `kept` (neighbour n's block b at
// n * blocks + b).
float measure_floor(const std::vector<float>& kept, int neighbours, int blocks) {
    const uint32_t total = static_cast<uint32_t>(neighbours) * static_cast<uint32_t>(blocks);
    const uint32_t sample_step = (total + kFloorSamples - 1) / kFloorSamples;
    const uint32_t sample_count = (total + sample_step - 1) / sample_step;
    std::vector<uint32_t> keys(kFloorSamples);
    for (uint32_t s = 0; s < kFloorSamples; ++s) {
        const uint32_t flat = std::min(s, sample_count - 1) * sample_step;
        const float k = kept[flat];
        const bool counted = s < sample_count && k > kExactMatchSad;
        keys[s] = counted ? float_bits(k) >> kFloorBinShift : 0u;
    }
    uint32_t valid = 0;
    for (uint32_t k : keys) valid += k >= 1 ? 1u : 0u;
    const uint32_t median_bin = ranked_bin(keys, 1, 2);
    const float median = bits_float(median_bin << kFloorBinShift);
    const float flat_limit = median * kFlatShare;
    const uint32_t grainy = std::max(float_bits(flat_limit) >> kFloorBinShift, 1u);
    const uint32_t floor_bin = ranked_bin(keys, grainy, kFloorRankDivisor);
    return valid == 0 ? 0.0f : bits_float(floor_bin << kFloorBinShift);
}

}  // namespace

extern "C" {

struct OrcMotionArgs {
    const float* pyramid;
    const uint32_t* neighbour_slots;
    int32_t* mv_field;
    float* confidence;  // null: not written
    const float* noise;
    uint32_t width, height, frame_count, centre_slot, neighbours;
    uint32_t blksize, overlap, search_radius, levels;
    uint32_t mv_stride, conf_stride, sad_floor_word;
    float thsad;
    uint32_t seeded;  // 1: mv_field holds the seeds; no coarse pass (motion/analyse.rs:273-316)
    int32_t* keep_seeds;  // non-null: the field after the coarse pass is copied here (analyse.rs:268-277)
    // motion/escalate.rs:19-57: with ceiling > search_radius the blocks that fail the first pass
    // search again `ceiling` either side of their first window's centre; `esc_reads_floor` takes the
    // floor from the noise word when it is positive; `widen_coarse` searches the coarse level again.
    uint32_t ceiling, esc_reads_floor, widen_coarse;
    // motion/analyse.rs:41-60: with `predictions` (6 words per neighbour) every block also searches
    // around its neighbour's camera-model prediction; with `sad_out` the fine pass writes each
    // block's winning SAD, then `neighbours * conf_stride` values on, its window's mean SAD.
    const float* predictions;
    float* sad_out;
    // motion/context.rs:30-45: the coarse pass's radius and how many times wider its blocks are than
    // the content a fine block covers.
    uint32_t coarse_radius, coarse_block_factor;
};

int64_t orc_motion_pyramid_floats(int w, int h, int frames, int levels) { return level_base(w, h, frames, levels); }

void orc_motion_pyramid_build(const float* ring, int channels, int w, int h, int frames, int ring_slot, int levels,
                              float* pyramid, int pyramid_slot) {
    const int64_t pixels = static_cast<int64_t>(w) * h;
    float* l0 = pyramid + pyramid_slot * slot_pixels(w, h, 0);
    for (int64_t p = 0; p < pixels; ++p) l0[p] = ring[(ring_slot * pixels + p) * channels];
    for (int l = 1; l < levels; ++l) {
        int sw, sh, dw, dh;
        level_dims(w, h, l - 1, &sw, &sh);
        level_dims(w, h, l, &dw, &dh);
        const float* src = pyramid + level_base(w, h, frames, l - 1) + pyramid_slot * slot_pixels(w, h, l - 1);
        float* dst = pyramid + level_base(w, h, frames, l) + pyramid_slot * slot_pixels(w, h, l);
        for (int y = 0; y < dh; ++y)
            for (int x = 0; x < dw; ++x) {
                const int sx = 2 * x, sy = 2 * y;
                const int sx1 = sx + 1 < sw ? sx + 1 : sx, sy1 = sy + 1 < sh ? sy + 1 : sy;
                const float sum = src[sy * sw + sx] + src[sy * sw + sx1] + src[sy1 * sw + sx] + src[sy1 * sw + sx1];
                dst[y * dw + x] = sum * 0.25f;
            }
    }
}

void orc_motion_search(const OrcMotionArgs* a) {
    const int w = static_cast<int>(a->width), h = static_cast<int>(a->height), frames = static_cast<int>(a->frame_count);
    const int step = static_cast<int>(a->blksize - a->overlap);
    const int bx_n = (w + step - 1) / step > 1 ? (w + step - 1) / step : 1;
    const int by_n = (h + step - 1) / step > 1 ? (h + step - 1) / step : 1;
    const int R = static_cast<int>(a->search_radius);
    const int Rc = static_cast<int>(a->coarse_radius);
    const int factor = a->coarse_block_factor > 0 ? static_cast<int>(a->coarse_block_factor) : 1;
    const bool coarse = a->levels > 1 && !a->seeded;
    const bool seeded = coarse || a->seeded;
    const float* noise_floor = a->noise ? a->noise + a->sad_floor_word : nullptr;
    const float model_floor = a->predictions && noise_floor ? *noise_floor : 0.0f;
    // analyse.rs:118-148 (`coarse_level`): the smallest level, its blocks `factor` times the content a
    // fine block covers there.
    Level Lc{};
    int scale = 1;
    float floor_scale = 1.0f;
    if (a->levels > 1) {
        const int level = static_cast<int>(a->levels) - 1;
        scale = 1 << level;
        level_dims(w, h, level, &Lc.width, &Lc.height);
        Lc.base = a->pyramid + level_base(w, h, frames, level);
        Lc.slot = slot_pixels(w, h, level);
        Lc.blksize = (static_cast<int>(a->blksize) / scale > 2 ? static_cast<int>(a->blksize) / scale : 2) * factor;
        Lc.step = step / scale > 1 ? step / scale : 1;
        Lc.blocks_x = (Lc.width + Lc.step - 1) / Lc.step > 1 ? (Lc.width + Lc.step - 1) / Lc.step : 1;
        Lc.blocks_y = (Lc.height + Lc.step - 1) / Lc.step > 1 ? (Lc.height + Lc.step - 1) / Lc.step : 1;
        floor_scale = coarse_floor_scale(Lc.blksize, static_cast<int>(a->blksize), scale);
    }
    if (coarse) {
        const int s = Lc.step * scale;
        const float bias = kModelCandidateBias * model_floor * floor_scale;
#pragma omp parallel for collapse(2) schedule(dynamic)
        for (int n = 0; n < static_cast<int>(a->neighbours); ++n)
            for (int by = 0; by < Lc.blocks_y; ++by)
                for (int bx = 0; bx < Lc.blocks_x; ++bx) {
                    const Best b = search_with_model(Lc, static_cast<int>(a->centre_slot),
                                                     static_cast<int>(a->neighbour_slots[n]), bx * Lc.step,
                                                     by * Lc.step, 0, 0, Rc, a->predictions, n, scale, bias);
                    const int c0 = std::min(bx * s / step, bx_n);
                    const int c1 = bx == Lc.blocks_x - 1 ? bx_n : std::min((bx + 1) * s / step, bx_n);
                    const int r0 = std::min(by * s / step, by_n);
                    const int r1 = by == Lc.blocks_y - 1 ? by_n : std::min((by + 1) * s / step, by_n);
                    int32_t* mv = a->mv_field + static_cast<int64_t>(n) * a->mv_stride;
                    for (int r = r0; r < r1; ++r)
                        for (int c = c0; c < c1; ++c) {
                            mv[(r * bx_n + c) * 2] = b.dx * scale;
                            mv[(r * bx_n + c) * 2 + 1] = b.dy * scale;
                        }
                }
        if (a->keep_seeds)
            std::copy(a->mv_field, a->mv_field + static_cast<int64_t>(a->neighbours) * a->mv_stride, a->keep_seeds);
    }
    Level L{a->pyramid, slot_pixels(w, h, 0), w, h, static_cast<int>(a->blksize), step, bx_n, by_n};
    const int neighbours = static_cast<int>(a->neighbours), blocks = bx_n * by_n;
    const int C = static_cast<int>(a->ceiling);
    const bool escalates = C > R;
    const int64_t means_base = static_cast<int64_t>(neighbours) * a->conf_stride;
    // escalate.rs:60-67: the kept SAD, the edge bar, and the winning window's centre of every block.
    std::vector<float> kept, edge;
    std::vector<int> centre_x, centre_y;
    if (escalates) {
        kept.assign(static_cast<size_t>(neighbours) * blocks, 0.0f);
        edge = kept;
        centre_x.assign(kept.size(), 0);
        centre_y.assign(kept.size(), 0);
    }
    const float fine_bias = kModelCandidateBias * model_floor;
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int n = 0; n < neighbours; ++n)
        for (int by = 0; by < by_n; ++by)
            for (int bx = 0; bx < bx_n; ++bx) {
                int32_t* mv = a->mv_field + static_cast<int64_t>(n) * a->mv_stride + (by * bx_n + bx) * 2;
                const int sdx = seeded ? mv[0] : 0, sdy = seeded ? mv[1] : 0;
                const Best b = search_with_model(L, static_cast<int>(a->centre_slot),
                                                 static_cast<int>(a->neighbour_slots[n]), bx * step, by * step, sdx,
                                                 sdy, R, a->predictions, n, 1, fine_bias);
                const int64_t slot = static_cast<int64_t>(n) * a->conf_stride + by * bx_n + bx;
                if (escalates) {
                    const size_t i = static_cast<size_t>(n) * blocks + by * bx_n + bx;
                    kept[i] = b.sad;
                    centre_x[i] = b.centre_dx;
                    centre_y[i] = b.centre_dy;
                    edge[i] = b.edge_bar;
                }
                mv[0] = b.dx;
                mv[1] = b.dy;
                if (a->sad_out) {
                    a->sad_out[slot] = b.sad;
                    a->sad_out[means_base + slot] = b.mean;
                }
                if (a->confidence) a->confidence[slot] = match_confidence(b.sad, a->noise[a->sad_floor_word], a->thsad);
            }
    if (!escalates) return;
    // escalate.rs:168-257: the floor the flags and margins score against.
    const float reading = a->noise ? a->noise[a->sad_floor_word] : 0.0f;
    const float floor = a->esc_reads_floor && reading > 0.0f ? reading : measure_floor(kept, neighbours, blocks);
    const float margin = kEscalateSadMargin * floor;
    // escalate.rs:335-395 (`mc_flag_failures`), on the field the fine pass left.
    std::vector<char> failed(kept.size(), 0);
    for (int n = 0; n < neighbours; ++n)
        for (int by = 0; by < by_n; ++by)
            for (int bx = 0; bx < bx_n; ++bx) {
                const size_t i = static_cast<size_t>(n) * blocks + by * bx_n + bx;
                const int32_t* f = a->mv_field + static_cast<int64_t>(n) * a->mv_stride;
                const int own = (by * bx_n + bx) * 2;
                int closest = INT32_MAX;
                auto gap = [&](int slot) {
                    closest = std::min(closest, std::max(std::abs(f[slot] - f[own]), std::abs(f[slot + 1] - f[own + 1])));
                };
                if (bx > 0) gap(own - 2);
                if (bx + 1 < bx_n) gap(own + 2);
                if (by > 0) gap(own - 2 * bx_n);
                if (by + 1 < by_n) gap(own + 2 * bx_n);
                if (closest == INT32_MAX) closest = 0;
                const bool low = match_confidence(kept[i], floor, a->thsad) < kEscalateBelowConfidence;
                const bool on_edge = kept[i] + margin < edge[i];
                failed[i] = low || on_edge || closest > kNeighbourDisagreement;
            }
    // escalate.rs:400-559 (`mc_escalate_search`). escalate.rs:203-205 (`reaches_further`): only a
    // ceiling past the coarse pass's radius searches the coarse level again, around no motion and the
    // camera model's prediction, the model's window winning by more than 1/8 of the floor scaled to
    // the coarse block.
    const bool widen = a->widen_coarse && a->levels > 1 && !a->seeded && C > Rc;
    const float coarse_bias = kModelCandidateBias * floor * floor_scale;
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int n = 0; n < neighbours; ++n)
        for (int by = 0; by < by_n; ++by)
            for (int bx = 0; bx < bx_n; ++bx) {
                const size_t i = static_cast<size_t>(n) * blocks + by * bx_n + bx;
                if (!failed[i]) continue;
                const int cs = static_cast<int>(a->centre_slot), ns = static_cast<int>(a->neighbour_slots[n]);
                Best best = search_window(L, cs, ns, bx * step, by * step, centre_x[i], centre_y[i], C);
                if (widen) {
                    const Best cb = search_with_model(Lc, cs, ns, bx * step / scale, by * step / scale, 0, 0, C,
                                                      a->predictions, n, scale, coarse_bias);
                    const int cx = cb.dx * scale, cy = cb.dy * scale;
                    if (cx != centre_x[i] || cy != centre_y[i]) {
                        const Best ch = search_window(L, cs, ns, bx * step, by * step, cx, cy, C);
                        if (ch.sad + margin < best.sad) best = ch;
                    }
                }
                if (best.sad + margin < kept[i]) {
                    const int64_t slot = static_cast<int64_t>(n) * a->conf_stride + by * bx_n + bx;
                    int32_t* mv = a->mv_field + static_cast<int64_t>(n) * a->mv_stride + (by * bx_n + bx) * 2;
                    mv[0] = best.dx;
                    mv[1] = best.dy;
                    if (a->sad_out) a->sad_out[slot] = best.sad;
                    if (a->confidence) a->confidence[slot] = match_confidence(best.sad, a->noise[a->sad_floor_word], a->thsad);
                }
            }
}

// One truemotion pass (motion/truemotion/kernels/truemotion/mod.rs:560-763, `mc_truemotion` with
// the serial scoring of score.rs:7-61) over level 0 of `pyramid`: every block of every neighbour
// picks its vector from `mv_in` (and `seeds` and the camera model's prediction, when given) into
// `mv_out`, with its confidence when `confidence` is given.
struct OrcTruemotionArgs {
    const float* pyramid;
    const uint32_t* neighbour_slots;
    const int32_t* mv_in;
    const int32_t* seeds;  // null: no seed candidates
    int32_t* mv_out;
    float* confidence;  // null: not written
    const float* noise;
    uint32_t width, height, frame_count, centre_slot, neighbours, blksize, overlap, mv_stride, conf_stride;
    uint32_t sad_field, reads_floor, refine_radius;
    float lambda_base, lambda_noise, surcharge, fade_level, thsad;
    // truemotion/kernels/truemotion/mod.rs:483-520, 560-575, 656-680: with `changes_in`, a block
    // whose 3x3 neighbourhood (itself included) changed nothing in the pass before copies its own
    // vector and keeps its confidence; `changes_out` flags each block whose pick left its own vector.
    const uint32_t* changes_in;
    uint32_t* changes_out;
    // mod.rs:878-900: with `predictions`, the camera model's prediction is a candidate; with
    // `sad_out`, every rescored block writes its winning SAD there (conf layout).
    const float* predictions;
    float* sad_out;
};

namespace {

struct Vec2 {
    int dx, dy;
};

bool on_grid(int c, int r, int bx, int by) { return c >= 0 && r >= 0 && c < bx && r < by; }

// candidates.rs:83-108 (`push_unique`).
void push_unique(std::vector<Vec2>& list, Vec2 v) {
    for (const Vec2& e : list)
        if (e.dx == v.dx && e.dy == v.dy) return;
    list.push_back(v);
}

// truemotion/kernels/truemotion/mod.rs:230-248 (`penalised_cost`).
float penalised_cost(float sad, Vec2 v, Vec2 median, float lambda, float surcharge) {
    const int deviation = std::abs(v.dx - median.dx) + std::abs(v.dy - median.dy);
    float cost = sad + lambda * static_cast<float>(deviation);
    if (deviation != 0 && surcharge > 0.0f) cost += surcharge * sad;
    return cost;
}

// mod.rs:448-463 (`pass_confidence`).
float pass_confidence(float sad, float floor, float thsad) {
    float excess = sad - floor;
    if (excess < 0.0f) excess = 0.0f;
    const float t2 = thsad * thsad, e2 = excess * excess;
    float c = (t2 - e2) / (t2 + e2);
    if (c < 0.0f) c = 0.0f;
    return c;
}

}  // namespace

void orc_truemotion_pass(const OrcTruemotionArgs* a) {
    const int w = static_cast<int>(a->width), h = static_cast<int>(a->height);
    const int b = static_cast<int>(a->blksize), step = static_cast<int>(a->blksize - a->overlap);
    const int bx_n = (w + step - 1) / step > 1 ? (w + step - 1) / step : 1;
    const int by_n = (h + step - 1) / step > 1 ? (h + step - 1) / step : 1;
    const int64_t slot = slot_pixels(w, h, 0);
#pragma omp parallel for collapse(2) schedule(dynamic, 16)
    for (int n = 0; n < static_cast<int>(a->neighbours); ++n)
        for (int blk = 0; blk < bx_n * by_n; ++blk) {
            const int col = blk % bx_n, row = blk / bx_n;
            const int ox = col * step, oy = row * step;
            const int64_t mv_base = static_cast<int64_t>(n) * a->mv_stride;
            const float* cf = a->pyramid + a->centre_slot * slot;
            const float* nf = a->pyramid + a->neighbour_slots[n] * slot;
            auto field = [&](const int32_t* f, int c, int r) -> Vec2 {
                if (!f || !on_grid(c, r, bx_n, by_n)) return Vec2{0, 0};
                const int32_t* v = f + mv_base + (static_cast<int64_t>(r) * bx_n + c) * 2;
                return Vec2{v[0], v[1]};
            };
            const Vec2 own = field(a->mv_in, col, row);
            if (a->changes_in) {
                bool changed = false;
                for (int pos = 0; pos < 9; ++pos) {
                    const int c = col + pos % 3 - 1, r = row + pos / 3 - 1;
                    if (on_grid(c, r, bx_n, by_n) && a->changes_in[static_cast<int64_t>(n) * a->conf_stride + r * bx_n + c])
                        changed = true;
                }
                if (!changed) {
                    int32_t* out = a->mv_out + mv_base + static_cast<int64_t>(blk) * 2;
                    out[0] = own.dx;
                    out[1] = own.dy;
                    if (a->changes_out) a->changes_out[static_cast<int64_t>(n) * a->conf_stride + blk] = 0;
                    continue;
                }
            }
            // candidates.rs:124-176 (`neighbourhood_median`): the component-wise lower median of the
            // on-grid blocks of the 3x3 neighbourhood, the block's own vector without any.
            std::vector<int> xs, ys;
            for (int pos = 0; pos < 9; ++pos) {
                if (pos == 4) continue;
                const int c = col + pos % 3 - 1, r = row + pos / 3 - 1;
                if (!on_grid(c, r, bx_n, by_n)) continue;
                const Vec2 v = field(a->mv_in, c, r);
                xs.push_back(v.dx);
                ys.push_back(v.dy);
            }
            Vec2 median = own;
            if (!xs.empty()) {
                std::sort(xs.begin(), xs.end());
                std::sort(ys.begin(), ys.end());
                median = Vec2{xs[(xs.size() - 1) / 2], ys[(ys.size() - 1) / 2]};
            }
            // candidates.rs:178-306 (`gather_candidates`).
            std::vector<Vec2> list;
            push_unique(list, own);
            push_unique(list, median);
            const int side_dx[4] = {-1, 1, 0, 0}, side_dy[4] = {0, 0, -1, 1};
            for (int sd = 0; sd < 4; ++sd)
                if (on_grid(col + side_dx[sd], row + side_dy[sd], bx_n, by_n))
                    push_unique(list, field(a->mv_in, col + side_dx[sd], row + side_dy[sd]));
            push_unique(list, Vec2{0, 0});
            if (a->predictions && predicts_motion(a->predictions, n)) {
                Vec2 m;
                model_displacement(a->predictions, n, ox, oy, b, 1, w, h, &m.dx, &m.dy);
                push_unique(list, m);
            }
            if (a->seeds) {
                push_unique(list, field(a->seeds, col, row));
                for (int corner = 0; corner < 4; ++corner) {
                    const int cc = col + (corner % 2) * 2 - 1, rr = row + (corner / 2) * 2 - 1;
                    if (on_grid(cc, rr, bx_n, by_n)) push_unique(list, field(a->seeds, cc, rr));
                }
            }
            int median_entry = 0;
            for (int e = static_cast<int>(list.size()) - 1; e >= 0; --e)
                if (list[e].dx == median.dx && list[e].dy == median.dy) median_entry = e;
            // score.rs:7-61: each row summed left to right, then the rows top to bottom.
            std::vector<float> centre(static_cast<size_t>(b) * b);
            for (int py = 0; py < b; ++py)
                for (int px = 0; px < b; ++px)
                    centre[py * b + px] = cf[static_cast<int64_t>(clamp_to(oy + py, h)) * w + clamp_to(ox + px, w)];
            auto sad_of = [&](Vec2 v) {
                float sad = 0.0f;
                for (int iy = 0; iy < b; ++iy) {
                    const int ny = clamp_to(oy + iy + v.dy, h);
                    float row_sum = 0.0f;
                    for (int ix = 0; ix < b; ++ix) {
                        const float diff = centre[iy * b + ix] - nf[static_cast<int64_t>(ny) * w + clamp_to(ox + ix + v.dx, w)];
                        row_sum += diff < 0.0f ? -diff : diff;
                    }
                    sad += row_sum;
                }
                return sad;
            };
            std::vector<float> sads(list.size());
            for (size_t e = 0; e < list.size(); ++e) sads[e] = sad_of(list[e]);
            // mod.rs:250-276 (`block_lambda`).
            const float median_sad = sads[median_entry];
            float floor = 0.0f;
            if (a->reads_floor) {
                const float reading = a->noise[a->sad_field];
                if (reading > 0.0f) floor = reading;
            }
            float lambda = a->lambda_base + a->lambda_noise * floor;
            if (a->fade_level > 0.0f) {
                const float excess = std::max(median_sad - floor, 0.0f);
                const float level_sq = a->fade_level * a->fade_level;
                const float fade = level_sq / (level_sq + excess * excess);
                lambda *= fade;
            }
            // mod.rs:292-345 (`settle_early`).
            const float own_cost = penalised_cost(sads[0], list[0], median, lambda, a->surcharge);
            const float median_cost = penalised_cost(median_sad, median, median, lambda, a->surcharge);
            int outcome = 0;  // 0 unsettled, 1 own wins, 2 median wins
            if (list.size() == 1 || (median_entry == 0 && own_cost <= lambda)) {
                outcome = 1;
            } else if (median_entry == 1) {
                if (own_cost <= median_cost && own_cost <= lambda) outcome = 1;
                else if (median_cost < own_cost && median_cost <= lambda) outcome = 2;
            }
            Vec2 best = list[0];
            float best_cost = own_cost, best_sad = sads[0];
            if (outcome == 2) {
                best = list[1];
                best_cost = median_cost;
                best_sad = sads[1];
            }
            if (outcome == 0) {
                // mod.rs:347-387 (`pick_listed`): the lowest cost, a tie keeping the earlier entry.
                size_t bi = 0;
                for (size_t e = 1; e < list.size(); ++e) {
                    const float cost = penalised_cost(sads[e], list[e], median, lambda, a->surcharge);
                    if (cost < best_cost) {
                        best_cost = cost;
                        bi = e;
                    }
                }
                best = list[bi];
                best_sad = sads[bi];
            }
            const bool kept = best.dx == own.dx && best.dy == own.dy;
            if (outcome != 1 && a->refine_radius > 0 && !kept) {
                // mod.rs:389-441: the ring around the best, each replacing it only when cheaper.
                const int reach = static_cast<int>(a->refine_radius);
                const Vec2 centre_vec = best;
                for (int ry = -reach; ry <= reach; ++ry)
                    for (int rx = -reach; rx <= reach; ++rx) {
                        if (rx == 0 && ry == 0) continue;
                        const Vec2 v{centre_vec.dx + rx, centre_vec.dy + ry};
                        const float sad = sad_of(v);
                        const float cost = penalised_cost(sad, v, median, lambda, a->surcharge);
                        if (cost < best_cost) {
                            best_cost = cost;
                            best_sad = sad;
                            best = v;
                        }
                    }
            }
            int32_t* out = a->mv_out + mv_base + static_cast<int64_t>(blk) * 2;
            out[0] = best.dx;
            out[1] = best.dy;
            if (a->confidence)
                a->confidence[static_cast<int64_t>(n) * a->conf_stride + blk] =
                    pass_confidence(best_sad, a->noise[a->sad_field], a->thsad);
            if (a->sad_out) a->sad_out[static_cast<int64_t>(n) * a->conf_stride + blk] = best_sad;
            if (a->changes_out)
                a->changes_out[static_cast<int64_t>(n) * a->conf_stride + blk] =
                    (best.dx == own.dx && best.dy == own.dy) ? 0u : 1u;
        }
}

}  // extern "C"
