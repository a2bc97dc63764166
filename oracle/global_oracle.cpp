// CPU ORACLE - test infrastructure only (see nlm_oracle.cpp for the rules it follows).
//
// A C++17 restatement of av-denoise's camera model: one similarity (a, b, tx, ty, valid) per
// adjacent frame pair, fitted to a block-match field and composed into per-neighbour predictions
// that the motion searches add as a second search centre.
//   compose:    motion/kernels/global.rs:18-119 (`mc_compose_models`), global/compose.rs:18-64
//               (`compose_gaps`, restated in oracle.py);
//   block means: global.rs:121-155 (`mc_block_means`);
//   high-pass:  motion/kernels/pyramid.rs:66-132 (`mc_box_rows`, `mc_high_pass_cols`);
//   fit:        global.rs:286-975 (`mc_fit_bands`, `mc_fit_sums`, `mc_fit_finish`) in the stage
//               order of global/fit.rs:196-250 (bands; weigh; gate with a prior; solve at 16, 8, 4,
//               2; polish; score), every workgroup of 256 blocks reducing its 8 lane sums by the
//               same halving tree and the finish adding the partials thread by thread before its
//               own halving tree;
//   prediction: motion/kernels/candidates.rs:71-166 (`model_displacement`, `predicts_motion`,
//               `model_centre`, `beats_incumbent`).
// Every f32 operation is one rounded operation in the reference's order (the build turns off
// contraction), so the models are expected to match the CUDA path bit for bit.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr int kModelWords = 5;
constexpr int kAffineWords = 6;
constexpr uint32_t kNoPair = 0xFFFFFFFFu;
constexpr int kFitThreads = 256;
constexpr int kFitLanes = 8;

// global.rs:208-283 and global/fit.rs:8-60: the fit's constants.
constexpr float kUnlimitedScale = 1.0e30f;
constexpr float kContrastHalfWeight = 0.25f;
constexpr float kContrastMinSad = 1e-6f;
constexpr float kBarMaxContrast = kContrastHalfWeight;
constexpr float kBarMaxLuma = 32.0f / 255.0f;
constexpr float kZeroVectorWeight = 0.2f;
constexpr float kNeighbourPrior = 0.5f;
constexpr uint32_t kBandEdgeEighths = 7;
constexpr uint32_t kBandPairSlack = 2;
constexpr float kMinFitWeight = 1e-3f;
constexpr float kMinFitSpread = 64.0f;
constexpr float kAcceptMargin = 0.7f;
constexpr float kMinMotionScore = 1e-3f;
constexpr float kMaxZoomChange = 0.15f;
constexpr float kMaxCornerShift = 400.0f;
constexpr float kFitInlierCap = 2.0f;
constexpr float kMaxRollTan = 0.2679492f;
constexpr float kFitScales[4] = {16.0f, 8.0f, 4.0f, 2.0f};

enum Stage { kWeigh = 0, kGate = 1, kSolve = 2, kPolish = 3, kScore = 4 };
enum StateWord { kSadScale = 0, kRefValid = 1, kRef = 2, kScaleLimit = 6 };
enum BandWord { kTop = 0, kBottom = 1, kLeft = 2, kRight = 3 };

struct Grid {
    int width, height, blksize, step, blocks_x, blocks_y;
};

struct FitField {
    const int32_t* field;  // one direction: (dx, dy) per block
    const float* sad;      // winning SADs, then window means and block means `means_offset` apart; or null
    bool has_contrast;
    uint32_t means_offset;
    bool older_to_newer;
};

// global.rs:752-760 (`block_contrast`) and 740-749 (`contrast_weight`).
float block_contrast(float best_sad, float mean_sad) {
    const float gap = std::fmax(mean_sad - best_sad, 0.0f);
    const float safe_best = std::fmax(best_sad, kContrastMinSad);
    return gap / safe_best;
}

float contrast_weight(float best_sad, float mean_sad) {
    const float c = block_contrast(best_sad, mean_sad);
    return c / (c + kContrastHalfWeight);
}

// global.rs:830-852 (`block_in_picture`).
uint32_t block_in_picture(const FitField& f, uint32_t block) {
    bool in_picture = f.field[block * 2] != 0 || f.field[block * 2 + 1] != 0;
    if (f.has_contrast) {
        const float best = f.sad[block], mean = f.sad[f.means_offset + block], luma = f.sad[2 * f.means_offset + block];
        in_picture = in_picture || block_contrast(best, mean) > kBarMaxContrast || luma > kBarMaxLuma;
    }
    return in_picture ? 1u : 0u;
}

uint32_t band_line(uint32_t start, uint32_t steps, bool upward) { return upward ? start + steps : start - steps; }

// global.rs:855-882 (`leading_band`).
uint32_t leading_band(const std::vector<uint32_t>& moving, uint32_t start, bool upward, uint32_t last, uint32_t width) {
    uint32_t steps = 0;
    for (;;) {
        const uint32_t line = band_line(start, steps, upward);
        const bool still = steps < last && moving[line] == 0u;
        if (!still) break;
        ++steps;
    }
    const uint32_t edge_moving = moving[band_line(start, steps, upward)];
    const bool is_short = steps * 3 <= last;
    const bool edge_ok = steps < last && edge_moving * 8 >= kBandEdgeEighths * width;
    return steps > 0 && is_short && edge_ok ? steps : 0u;
}

bool bands_pair(uint32_t a, uint32_t b) {
    const uint32_t longer = a > b ? a : b, shorter = a < b ? a : b;
    return shorter > 0 && longer - shorter <= kBandPairSlack;
}

// global.rs:286-392 (`mc_fit_bands`).
void fit_bands(const Grid& g, const FitField& f, uint32_t* bands) {
    const uint32_t bx = static_cast<uint32_t>(g.blocks_x), by = static_cast<uint32_t>(g.blocks_y);
    const uint32_t w = static_cast<uint32_t>(g.width), h = static_cast<uint32_t>(g.height);
    const uint32_t b = static_cast<uint32_t>(g.blksize), s = static_cast<uint32_t>(g.step);
    const uint32_t inside_rows = (h > b ? h - b : 0) / s, inside_cols = (w > b ? w - b : 0) / s;
    const uint32_t interior_rows = by > 2 ? by - 2 : 0, interior_cols = bx > 2 ? bx - 2 : 0;
    const uint32_t last_row = inside_rows < interior_rows ? inside_rows : interior_rows;
    const uint32_t last_col = inside_cols < interior_cols ? inside_cols : interior_cols;
    const bool counted = last_row >= 1 && last_col >= 1;
    std::vector<uint32_t> row_moving(by, 0), col_moving(bx, 0);
    for (uint32_t row = 0; row < by; ++row)
        if (row >= 1 && row <= last_row)
            for (uint32_t col = 1; col <= last_col; ++col) row_moving[row] += block_in_picture(f, row * bx + col);
    for (uint32_t col = 0; col < bx; ++col)
        if (col >= 1 && col <= last_col)
            for (uint32_t row = 1; row <= last_row; ++row) col_moving[col] += block_in_picture(f, row * bx + col);
    uint32_t top = 0, bottom = 0, left = 0, right = 0;
    if (counted) {
        top = leading_band(row_moving, 1, true, last_row, last_col);
        bottom = leading_band(row_moving, last_row, false, last_row, last_col);
        left = leading_band(col_moving, 1, true, last_col, last_row);
        right = leading_band(col_moving, last_col, false, last_col, last_row);
    }
    const bool rows_paired = bands_pair(top, bottom), cols_paired = bands_pair(left, right);
    bands[kTop] = rows_paired ? 1 + top : 0u;
    bands[kBottom] = rows_paired ? last_row + 1 - bottom : by;
    bands[kLeft] = cols_paired ? 1 + left : 0u;
    bands[kRight] = cols_paired ? last_col + 1 - right : bx;
}

uint32_t neighbour_agrees(const int32_t* field, uint32_t nb, int mvx, int mvy, int tolerance) {
    const int gx = field[nb * 2] - mvx, gy = field[nb * 2 + 1] - mvy;
    return (std::abs(gx) <= tolerance && std::abs(gy) <= tolerance) ? 1u : 0u;
}

// global.rs:762-816 (`block_base_weight`).
float block_base_weight(const Grid& g, const int32_t* field, const uint32_t* bands, uint32_t col, uint32_t row, int mvx,
                        int mvy) {
    const int tolerance = 1 + (3 * g.step) / 10;
    const int ox = static_cast<int>(col) * g.step, oy = static_cast<int>(row) * g.step, size = g.blksize;
    const uint32_t bx = static_cast<uint32_t>(g.blocks_x), by = static_cast<uint32_t>(g.blocks_y);
    const bool interior = col >= 1 && row >= 1 && col + 1 < bx && row + 1 < by;
    const bool inside = ox + size <= g.width && oy + size <= g.height;
    const int tx = ox + mvx, ty = oy + mvy;
    const bool lands = tx >= 0 && tx + size <= g.width && ty >= 0 && ty + size <= g.height;
    const bool in_rows = row >= bands[kTop] && row < bands[kBottom];
    const bool in_cols = col >= bands[kLeft] && col < bands[kRight];
    if (!(interior && inside && lands && in_rows && in_cols)) return 0.0f;
    const uint32_t block = row * bx + col;
    const uint32_t agreeing = neighbour_agrees(field, block - 1, mvx, mvy, tolerance) +
                              neighbour_agrees(field, block + 1, mvx, mvy, tolerance) +
                              neighbour_agrees(field, block - bx, mvx, mvy, tolerance) +
                              neighbour_agrees(field, block + bx, mvx, mvy, tolerance);
    return (static_cast<float>(agreeing) + kNeighbourPrior) / (4.0f + kNeighbourPrior);
}

// global.rs:951-962 (`residual_sq`).
float residual_sq(float a, float b, float tx, float ty, float x, float y, float mx, float my) {
    const float px = (a - 1.0f) * x - b * y + tx;
    const float py = b * x + (a - 1.0f) * y + ty;
    const float rx = mx - px, ry = my - py;
    return rx * rx + ry * ry;
}

float corner_shift_sq(float a, float b, float tx, float ty, float x, float y) {
    const float sx = a * x - b * y + tx - x;
    const float sy = b * x + a * y + ty - y;
    return sx * sx + sy * sy;
}

bool beats_still(float model_score, float still_score, float weight) {
    const bool moving = weight > 0.0f && still_score > kMinMotionScore * weight;
    return moving && model_score <= kAcceptMargin * still_score;
}

// global.rs:918-939 (`reduce_lanes`): the halving tree over one workgroup's 256 slots of each lane.
void reduce_lanes(std::vector<float>& scratch) {
    for (int stride = kFitThreads / 2; stride >= 1; stride >>= 1)
        for (int t = 0; t < stride; ++t)
            for (int lane = 0; lane < kFitLanes; ++lane) scratch[lane * kFitThreads + t] += scratch[lane * kFitThreads + t + stride];
}

// global.rs:394-577 (`mc_fit_sums`): one stage's partial sums, kFitLanes per workgroup.
void fit_sums(const Grid& g, const FitField& f, const uint32_t* bands, std::vector<float>& weights, const float* state,
              const float* models, uint32_t prior_slot, int stage, float scale, std::vector<float>& partials) {
    const int blocks = g.blocks_x * g.blocks_y;
    const int groups = (blocks + kFitThreads - 1) / kFitThreads;
    partials.assign(static_cast<size_t>(groups) * kFitLanes, 0.0f);
    const bool has_sad = f.sad != nullptr;
    const bool solve = stage == kSolve || stage == kPolish;
    std::vector<float> scratch(kFitLanes * kFitThreads);
    for (int grp = 0; grp < groups; ++grp) {
        std::fill(scratch.begin(), scratch.end(), 0.0f);
        for (int t = 0; t < kFitThreads; ++t) {
            const int block = grp * kFitThreads + t;
            if (block >= blocks) continue;
            auto set = [&](int lane, float v) { scratch[lane * kFitThreads + t] = v; };
            const uint32_t col = static_cast<uint32_t>(block % g.blocks_x), row = static_cast<uint32_t>(block / g.blocks_x);
            const int mvx = f.field[block * 2], mvy = f.field[block * 2 + 1];
            const float block_sad = has_sad ? f.sad[block] : 0.0f;
            const float half = static_cast<float>(g.blksize) * 0.5f;
            const float centre_x = static_cast<float>(g.width) * 0.5f, centre_y = static_cast<float>(g.height) * 0.5f;
            const float block_x = static_cast<float>(col * g.step) + half - centre_x;
            const float block_y = static_cast<float>(row * g.step) + half - centre_y;
            const float shift_x = static_cast<float>(mvx), shift_y = static_cast<float>(mvy);
            float px = block_x, py = block_y, mx = shift_x, my = shift_y;
            if (!f.older_to_newer) {
                px = block_x + shift_x;
                py = block_y + shift_y;
                mx = -shift_x;
                my = -shift_y;
            }
            const float scale_sq = scale * scale;
            if (stage == kWeigh) {
                float base = block_base_weight(g, f.field, bands, col, row, mvx, mvy);
                if (f.has_contrast) base *= contrast_weight(block_sad, f.sad[f.means_offset + block]);
                weights[block] = base;
                set(0, base);
                set(1, base * block_sad);
                continue;
            }
            float matched = weights[block];
            if (has_sad) {
                const float sad_scale = state[kSadScale];
                const float safe = std::fmax(sad_scale, 1e-12f);
                const float ratio = block_sad / safe;
                const float ratio_sq = ratio * ratio;
                const float sad_weight = 1.0f / (1.0f + ratio_sq * ratio_sq);
                matched *= sad_scale > 0.0f ? sad_weight : 1.0f;
            }
            const bool ref_valid = state[kRefValid] != 0.0f;
            const float ref_sq = residual_sq(state[kRef], state[kRef + 1], state[kRef + 2], state[kRef + 3], px, py, mx, my);
            if (solve) {
                const float limited = std::fmin(scale, state[kScaleLimit]);
                const float limited_sq = limited * limited;
                const float damping = 1.0f / (1.0f + ref_sq / limited_sq);
                float residual_weight = damping * damping;
                if (stage == kPolish) residual_weight = ref_sq <= limited_sq ? 1.0f : 0.0f;
                const bool still = mvx == 0 && mvy == 0;
                const float zero_weight = still ? kZeroVectorWeight : 1.0f;
                const float fit_weight = ref_valid ? residual_weight : 1.0f;
                const float weight = matched * zero_weight * fit_weight;
                const float dot = px * mx + py * my;
                const float cross = px * my - py * mx;
                const float spread = px * px + py * py;
                set(0, weight);
                set(1, weight * px);
                set(2, weight * py);
                set(3, weight * mx);
                set(4, weight * my);
                set(5, weight * dot);
                set(6, weight * cross);
                set(7, weight * spread);
            } else {
                float model_sq = ref_sq;
                if (stage == kGate) {
                    const float* p = models + prior_slot * kModelWords;
                    model_sq = residual_sq(p[0], p[1], p[2], p[3], px + centre_x, py + centre_y, mx, my);
                }
                const float motion_sq = mx * mx + my * my;
                set(0, matched * std::fmin(model_sq, scale_sq));
                set(1, matched * std::fmin(motion_sq, scale_sq));
                set(2, matched);
            }
        }
        reduce_lanes(scratch);
        for (int lane = 0; lane < kFitLanes; ++lane) partials[static_cast<size_t>(grp) * kFitLanes + lane] = scratch[lane * kFitThreads];
    }
}

void write_reference(float* state, float valid, float a, float b, float tx, float ty) {
    state[kRefValid] = valid;
    state[kRef] = a;
    state[kRef + 1] = b;
    state[kRef + 2] = tx;
    state[kRef + 3] = ty;
}

// global.rs:579-738 (`mc_fit_finish`).
void fit_finish(const Grid& g, const std::vector<float>& partials, float* state, float* models, uint32_t prior_slot,
                uint32_t slot, int stage) {
    const int groups = static_cast<int>(partials.size() / kFitLanes);
    std::vector<float> scratch(kFitLanes * kFitThreads, 0.0f);
    for (int lane = 0; lane < kFitLanes; ++lane)
        for (int t = 0; t < kFitThreads; ++t) {
            float sum = 0.0f;
            for (int i = t; i < groups; i += kFitThreads) sum += partials[static_cast<size_t>(i) * kFitLanes + lane];
            scratch[lane * kFitThreads + t] = sum;
        }
    reduce_lanes(scratch);
    auto total = [&](int lane) { return scratch[lane * kFitThreads]; };
    const float centre_x = static_cast<float>(g.width) * 0.5f, centre_y = static_cast<float>(g.height) * 0.5f;
    if (stage == kWeigh) {
        const float base = total(0), base_sad = total(1);
        const float safe_base = std::fmax(base, 1e-12f);
        state[kSadScale] = base > 0.0f ? base_sad / safe_base : 0.0f;
        state[kScaleLimit] = kUnlimitedScale;
        write_reference(state, 0.0f, 1.0f, 0.0f, 0.0f, 0.0f);
    } else if (stage == kGate) {
        const float* p = models + prior_slot * kModelWords;
        if (p[4] != 0.0f && beats_still(total(0), total(1), total(2))) {
            const float ctx = p[2] + p[0] * centre_x - p[1] * centre_y - centre_x;
            const float cty = p[3] + p[1] * centre_x + p[0] * centre_y - centre_y;
            state[kScaleLimit] = kFitInlierCap;
            write_reference(state, 1.0f, p[0], p[1], ctx, cty);
        }
    } else if (stage == kSolve || stage == kPolish) {
        const float weight = total(0);
        const float inverse_weight = 1.0f / std::fmax(weight, kMinFitWeight);
        const float mean_px = total(1) * inverse_weight, mean_py = total(2) * inverse_weight;
        const float mean_dx = total(3) * inverse_weight, mean_dy = total(4) * inverse_weight;
        const float spread = total(7) - weight * (mean_px * mean_px + mean_py * mean_py);
        const float dot = total(5) - weight * (mean_px * mean_dx + mean_py * mean_dy);
        const float cross = total(6) - weight * (mean_px * mean_dy - mean_py * mean_dx);
        float valid = 0.0f, a = 1.0f, b = 0.0f, tx = 0.0f, ty = 0.0f;
        if (weight >= kMinFitWeight && spread > kMinFitSpread * weight) {
            const float inverse_spread = 1.0f / spread;
            valid = 1.0f;
            a = 1.0f + dot * inverse_spread;
            b = cross * inverse_spread;
            tx = mean_px + mean_dx - (a * mean_px - b * mean_py);
            ty = mean_py + mean_dy - (b * mean_px + a * mean_py);
        }
        write_reference(state, valid, a, b, tx, ty);
    } else {
        const bool ref_valid = state[kRefValid] != 0.0f;
        const float a = state[kRef], b = state[kRef + 1];
        const float tx = state[kRef + 2] + centre_x - (a * centre_x - b * centre_y);
        const float ty = state[kRef + 3] + centre_y - (b * centre_x + a * centre_y);
        const bool passes = beats_still(total(0), total(1), total(2));
        const float zoom = std::sqrt(a * a + b * b);
        const bool zoom_ok = std::fabs(zoom - 1.0f) <= kMaxZoomChange;
        const bool roll_ok = a > 0.0f && std::fabs(b) <= kMaxRollTan * a;
        const float fx = static_cast<float>(g.width), fy = static_cast<float>(g.height);
        const float limit = kMaxCornerShift * kMaxCornerShift;
        const bool top_ok = corner_shift_sq(a, b, tx, ty, 0.0f, 0.0f) <= limit && corner_shift_sq(a, b, tx, ty, fx, 0.0f) <= limit;
        const bool bottom_ok = corner_shift_sq(a, b, tx, ty, 0.0f, fy) <= limit && corner_shift_sq(a, b, tx, ty, fx, fy) <= limit;
        const bool accepted = ref_valid && passes && zoom_ok && roll_ok && top_ok && bottom_ok;
        float* m = models + slot * kModelWords;
        m[0] = accepted ? a : 1.0f;
        m[1] = accepted ? b : 0.0f;
        m[2] = accepted ? tx : 0.0f;
        m[3] = accepted ? ty : 0.0f;
        m[4] = accepted ? 1.0f : 0.0f;
    }
}

int clamp_to(int v, int limit) { return v < 0 ? 0 : (v >= limit ? limit - 1 : v); }

}  // namespace

extern "C" {

// global.rs:18-119 (`mc_compose_models`): one prediction per neighbour, AFFINE_WORDS each.
void orc_compose_models(const float* models, const uint32_t* gaps, float* out, uint32_t neighbours, uint32_t max_steps,
                        uint32_t past_neighbours) {
    for (uint32_t n = 0; n < neighbours; ++n) {
        const bool past = n < past_neighbours;
        float acc_a = 1.0f, acc_b = 0.0f, acc_tx = 0.0f, acc_ty = 0.0f;
        for (uint32_t step = 0; step < max_steps; ++step) {
            const uint32_t gap = gaps[n * max_steps + step];
            float pa = 1.0f, pb = 0.0f, ptx = 0.0f, pty = 0.0f;
            if (gap != kNoPair) {
                const float* m = models + gap * kModelWords;
                if (m[4] != 0.0f) {
                    pa = m[0];
                    pb = m[1];
                    ptx = m[2];
                    pty = m[3];
                }
            }
            float oa = pa, ob = pb, otx = ptx, oty = pty, ia = acc_a, ib = acc_b, itx = acc_tx, ity = acc_ty;
            if (past) {
                oa = acc_a;
                ob = acc_b;
                otx = acc_tx;
                oty = acc_ty;
                ia = pa;
                ib = pb;
                itx = ptx;
                ity = pty;
            }
            acc_a = oa * ia - ob * ib;
            acc_b = oa * ib + ob * ia;
            acc_tx = oa * itx - ob * ity + otx;
            acc_ty = ob * itx + oa * ity + oty;
        }
        if (past) {
            const float norm = acc_a * acc_a + acc_b * acc_b;
            float ia = 1.0f, ib = 0.0f, itx = 0.0f, ity = 0.0f;
            if (norm > 0.0f) {
                const float r = 1.0f / norm;
                ia = acc_a * r;
                ib = -acc_b * r;
                itx = -(ia * acc_tx - ib * acc_ty);
                ity = -(ib * acc_tx + ia * acc_ty);
            }
            acc_a = ia;
            acc_b = ib;
            acc_tx = itx;
            acc_ty = ity;
        }
        float* o = out + n * kAffineWords;
        o[0] = acc_a;
        o[1] = -acc_b;
        o[2] = acc_b;
        o[3] = acc_a;
        o[4] = acc_tx;
        o[5] = acc_ty;
    }
}

// global.rs:121-155 (`mc_block_means`): each block's mean sample, row-major, clamped to the frame.
void orc_block_means(const float* plane, float* out, int width, int height, int blksize, int step, int blocks_x,
                     int blocks_y) {
    const float inverse = 1.0f / static_cast<float>(blksize * blksize);
    for (int block = 0; block < blocks_x * blocks_y; ++block) {
        const int ox = (block % blocks_x) * step, oy = (block / blocks_x) * step;
        float total = 0.0f;
        for (int y = 0; y < blksize; ++y) {
            const int sy = oy + y < height - 1 ? oy + y : height - 1;
            for (int x = 0; x < blksize; ++x) {
                const int sx = ox + x < width - 1 ? ox + x : width - 1;
                total += plane[static_cast<int64_t>(sy) * width + sx];
            }
        }
        out[block] = total * inverse;
    }
}

// pyramid.rs:66-132: `rows` takes the row box mean, `out` the plane minus the box mean of `rows`.
void orc_high_pass(const float* src, float* rows, float* out, int width, int height, int radius) {
    const int taps = 2 * radius + 1;
    const float inverse = 1.0f / static_cast<float>(taps);
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            float total = 0.0f;
            for (int t = 0; t < taps; ++t) total += src[static_cast<int64_t>(y) * width + clamp_to(x + t - radius, width)];
            rows[static_cast<int64_t>(y) * width + x] = total * inverse;
        }
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            float total = 0.0f;
            for (int t = 0; t < taps; ++t) total += rows[static_cast<int64_t>(clamp_to(y + t - radius, height)) * width + x];
            const int64_t i = static_cast<int64_t>(y) * width + x;
            out[i] = src[i] - total * inverse;
        }
}

// global/fit.rs:196-250 (`run_model_fit`): fits one direction of a pair field into ring slot `slot`,
// from ring slot `prior` when it is at least 0. `sad` (or null) holds the winning SADs, then, with
// `has_contrast`, the window means and the block means, `means_offset` values apart. `state` (8
// floats) receives the fit's final state.
void orc_model_fit(const int32_t* field, const float* sad, int has_contrast, uint32_t means_offset, int older_to_newer,
                   int width, int height, int blksize, int step, int blocks_x, int blocks_y, int prior, float* models,
                   uint32_t slot, float* state) {
    const Grid g{width, height, blksize, step, blocks_x, blocks_y};
    const FitField f{field, sad, sad != nullptr && has_contrast != 0, means_offset, older_to_newer != 0};
    uint32_t bands[4];
    fit_bands(g, f, bands);
    std::vector<float> weights(static_cast<size_t>(blocks_x) * blocks_y, 0.0f), partials;
    const uint32_t prior_slot = prior >= 0 ? static_cast<uint32_t>(prior) : 0u;
    auto stage = [&](int st, float scale) {
        fit_sums(g, f, bands, weights, state, models, prior_slot, st, scale, partials);
        fit_finish(g, partials, state, models, prior_slot, slot, st);
    };
    stage(kWeigh, kFitInlierCap);
    if (prior >= 0) stage(kGate, kFitInlierCap);
    for (float scale : kFitScales) stage(kSolve, scale);
    stage(kPolish, kFitInlierCap);
    stage(kScore, kFitInlierCap);
}

// global.rs:157-172 (`mc_model_identity`).
void orc_model_identity(float* models, uint32_t slot) {
    float* m = models + slot * kModelWords;
    m[0] = 1.0f;
    m[1] = m[2] = m[3] = m[4] = 0.0f;
}

// global/fit.rs band bounds alone, for the tests of the bars.
void orc_fit_bands(const int32_t* field, const float* sad, int has_contrast, uint32_t means_offset, int width,
                   int height, int blksize, int step, int blocks_x, int blocks_y, uint32_t* bands) {
    const Grid g{width, height, blksize, step, blocks_x, blocks_y};
    const FitField f{field, sad, sad != nullptr && has_contrast != 0, means_offset, true};
    fit_bands(g, f, bands);
}

}  // extern "C"
