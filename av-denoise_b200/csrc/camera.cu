// The camera model on sm_100a: one similarity per adjacent frame pair fitted to a block-match field,
// composed into each neighbour's prediction, and the high-passed luma and block means the pair
// model's search and fit read.
//
// Reference behaviour (av-denoise-core/src/motion):
//   kernels/global.rs:18-119     `mc_compose_models`: a future neighbour applies its pairs from the
//                                centre outward, a past one multiplies them into the motion from the
//                                neighbour to the centre and takes the inverse; a missing or invalid
//                                pair is no motion; output m00 m01 m10 m11 tx ty = a -b b a tx ty.
//   kernels/global.rs:121-172    `mc_block_means` (row-major, clamped), `mc_model_identity`.
//   kernels/pyramid.rs:66-132    `mc_box_rows`, `mc_high_pass_cols`: the plane minus its 17x17 box
//                                mean, taps summed left to right, then top to bottom, clamped.
//   kernels/global.rs:286-975 with global/fit.rs:196-250  the fit: letterbox bars; the weigh stage
//                                (neighbour agreement, contrast, mean SAD); the gate on a prior; four
//                                Geman-McClure solves at residual scales 16, 8, 4, 2; an inlier
//                                polish; the score against no motion and the plausibility bounds.
//
// Layout and design: a model is 5 f32 words (a, b, tx, ty, valid) in a ring of slots; a fit keeps 8
// state words, 4 band words, a launch count, the bars' line counts, one weight per block and 8 partial
// sums per 256 blocks in its scratch. The bars take one launch of one CTA per block row (integer
// counts); each fit stage one launch of 256-thread CTAs (one block per thread) that reduce their 8
// lane sums by a fixed halving tree, the last CTA to finish then adding the partials thread by
// thread and halving again before it updates the state, so the sums, and the model, are the same
// bits on every run and match the CPU restatement. The file is built with -fmad=false: every
// multiply and add rounds on its own.

#include <cuda_runtime.h>

#include <cstdint>

#include "camera_model.cuh"
#include "kernels.h"

namespace avd {

namespace {

constexpr int kFitThreads = 256;
constexpr int kFitLanes = 8;
constexpr uint32_t kNoPair = 0xFFFFFFFFu;

// global.rs:208-283 and global/fit.rs:8-60.
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

enum Stage { kWeigh = 0, kGate = 1, kSolve = 2, kPolish = 3, kScore = 4 };
enum StateWord { kSadScale = 0, kRefValid = 1, kRef = 2, kScaleLimit = 6 };
enum BandWord { kTop = 0, kBottom = 1, kLeft = 2, kRight = 3 };

__device__ __forceinline__ int clamp_to(int v, int limit) { return v < 0 ? 0 : (v >= limit ? limit - 1 : v); }

__device__ __forceinline__ void compose_one(const float* __restrict__ models, const uint32_t* __restrict__ gaps,
                                            float* __restrict__ out, int neighbours, int max_steps,
                                            int past_neighbours) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= neighbours) return;
    const bool past = n < past_neighbours;
    float acc_a = 1.0f, acc_b = 0.0f, acc_tx = 0.0f, acc_ty = 0.0f;
    for (int step = 0; step < max_steps; ++step) {
        const uint32_t gap = gaps[n * max_steps + step];
        float pa = 1.0f, pb = 0.0f, ptx = 0.0f, pty = 0.0f;
        if (gap != kNoPair) {
            const float* m = models + static_cast<int64_t>(gap) * kModelWords;
            if (m[4] != 0.0f) {
                pa = m[0];
                pb = m[1];
                ptx = m[2];
                pty = m[3];
            }
        }
        // Future steps apply after the motion so far, past steps before it.
        const float oa = past ? acc_a : pa, ob = past ? acc_b : pb, otx = past ? acc_tx : ptx, oty = past ? acc_ty : pty;
        const float ia = past ? pa : acc_a, ib = past ? pb : acc_b, itx = past ? ptx : acc_tx, ity = past ? pty : acc_ty;
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

__global__ void __launch_bounds__(32) compose_kernel(const float* __restrict__ models, const uint32_t* __restrict__ gaps,
                                                     float* __restrict__ out, int neighbours, int max_steps,
                                                     int past_neighbours) {
    compose_one(models, gaps, out, neighbours, max_steps, past_neighbours);
}

// The same composition with the gap table passed by value, for tables the host builds per window.
struct InlineGaps {
    uint32_t g[kMaxInlineGaps];
};

__global__ void __launch_bounds__(32) compose_inline_kernel(const float* __restrict__ models, InlineGaps gaps,
                                                            float* __restrict__ out, int neighbours, int max_steps,
                                                            int past_neighbours) {
    compose_one(models, gaps.g, out, neighbours, max_steps, past_neighbours);
}

__global__ void __launch_bounds__(256) block_means_kernel(const float* __restrict__ plane, float* __restrict__ out,
                                                          int width, int height, int blksize, int step, int blocks_x,
                                                          int blocks) {
    const int block = blockIdx.x * blockDim.x + threadIdx.x;
    if (block >= blocks) return;
    const float inverse = 1.0f / static_cast<float>(blksize * blksize);
    const int ox = (block % blocks_x) * step, oy = (block / blocks_x) * step;
    float total = 0.0f;
    for (int y = 0; y < blksize; ++y) {
        const float* row = plane + static_cast<int64_t>(min(oy + y, height - 1)) * width;
        for (int x = 0; x < blksize; ++x) total += __ldg(row + min(ox + x, width - 1));
    }
    out[block] = total * inverse;
}

__global__ void model_identity_kernel(float* models, int slot) {
    float* m = models + static_cast<int64_t>(slot) * kModelWords;
    m[0] = 1.0f;
    m[1] = 0.0f;
    m[2] = 0.0f;
    m[3] = 0.0f;
    m[4] = 0.0f;
}

// pyramid.rs:66-98 (`mc_box_rows`).
__global__ void __launch_bounds__(256) box_rows_kernel(const float* __restrict__ src, float* __restrict__ rows, int width,
                                                       int height, int radius) {
    const int x = blockIdx.x * 16 + threadIdx.x % 16, y = blockIdx.y * 16 + threadIdx.x / 16;
    if (x >= width || y >= height) return;
    const int taps = 2 * radius + 1;
    const float inverse = 1.0f / static_cast<float>(taps);
    const float* row = src + static_cast<int64_t>(y) * width;
    float total = 0.0f;
    for (int t = 0; t < taps; ++t) total += __ldg(row + clamp_to(x + t - radius, width));
    rows[static_cast<int64_t>(y) * width + x] = total * inverse;
}

// pyramid.rs:100-132 (`mc_high_pass_cols`).
__global__ void __launch_bounds__(256) high_pass_cols_kernel(const float* __restrict__ src,
                                                             const float* __restrict__ rows, float* __restrict__ out,
                                                             int width, int height, int radius) {
    const int x = blockIdx.x * 16 + threadIdx.x % 16, y = blockIdx.y * 16 + threadIdx.x / 16;
    if (x >= width || y >= height) return;
    const int taps = 2 * radius + 1;
    const float inverse = 1.0f / static_cast<float>(taps);
    float total = 0.0f;
    for (int t = 0; t < taps; ++t) total += __ldg(rows + static_cast<int64_t>(clamp_to(y + t - radius, height)) * width + x);
    const int64_t i = static_cast<int64_t>(y) * width + x;
    out[i] = __ldg(src + i) - total * inverse;
}

// ---- the fit ----------------------------------------------------------------------------------

struct FitArgs {
    const int32_t* field;  // one direction of a pair field: (dx, dy) per block
    const float* sad;      // winning SADs, then window means and block means `means_offset` apart; or null
    int has_contrast;
    int means_offset;
    int older_to_newer;
    int width, height, blksize, step, blocks_x, blocks_y;
    uint32_t* bands;
    unsigned* done;         // CTAs finished in the current launch (the last one finishes the stage)
    uint32_t* row_moving;   // blocks_y, then blocks_x line counts of the bars
    float* weights;
    float* state;
    float* partials;
    float* models;
    int prior_slot, slot;
};

// global.rs:740-760 (`contrast_weight`, `block_contrast`).
__device__ __forceinline__ float block_contrast(float best_sad, float mean_sad) {
    const float gap = fmaxf(mean_sad - best_sad, 0.0f);
    const float safe_best = fmaxf(best_sad, kContrastMinSad);
    return gap / safe_best;
}

__device__ __forceinline__ float contrast_weight(float best_sad, float mean_sad) {
    const float c = block_contrast(best_sad, mean_sad);
    return c / (c + kContrastHalfWeight);
}

// global.rs:830-852 (`block_in_picture`).
__device__ __forceinline__ uint32_t block_in_picture(const FitArgs& f, int block) {
    bool in_picture = f.field[block * 2] != 0 || f.field[block * 2 + 1] != 0;
    if (f.has_contrast) {
        const float best = f.sad[block], mean = f.sad[f.means_offset + block], luma = f.sad[2 * f.means_offset + block];
        in_picture = in_picture || block_contrast(best, mean) > kBarMaxContrast || luma > kBarMaxLuma;
    }
    return in_picture ? 1u : 0u;
}

__device__ __forceinline__ uint32_t band_line(uint32_t start, uint32_t steps, bool upward) {
    return upward ? start + steps : start - steps;
}

// global.rs:855-882 (`leading_band`).
__device__ uint32_t leading_band(const uint32_t* moving, uint32_t start, bool upward, uint32_t last, uint32_t width) {
    // The counts come from every CTA of the launch: read past L1.
    uint32_t steps = 0;
    while (steps < last && __ldcg(moving + band_line(start, steps, upward)) == 0u) ++steps;
    const uint32_t edge_moving = __ldcg(moving + band_line(start, steps, upward));
    const bool is_short = steps * 3 <= last;
    const bool edge_ok = steps < last && edge_moving * 8 >= kBandEdgeEighths * width;
    return steps > 0 && is_short && edge_ok ? steps : 0u;
}

__device__ __forceinline__ bool bands_pair(uint32_t a, uint32_t b) {
    const uint32_t longer = max(a, b), shorter = min(a, b);
    return shorter > 0 && longer - shorter <= kBandPairSlack;
}

// The last CTA of a launch: every CTA's writes are fenced before its count, so the CTA that counts
// last sees them all. It resets the count for the next launch. Uniform across the CTA.
__device__ __forceinline__ bool last_cta(unsigned* done) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned before = atomicAdd(done, 1u);
        last = before == gridDim.x - 1;
        if (last) *done = 0u;
    }
    __syncthreads();
    if (last) __threadfence();
    return last;
}

// global.rs:286-392 (`mc_fit_bands`): one CTA per block row counts the row's blocks that belong to
// the picture and adds each to its column's count (integer sums: the order does not matter); the
// last CTA walks the bars.
__global__ void __launch_bounds__(kFitThreads) fit_bands_kernel(FitArgs f) {
    __shared__ uint32_t row_count;
    const uint32_t bx = static_cast<uint32_t>(f.blocks_x), by = static_cast<uint32_t>(f.blocks_y);
    uint32_t* row_moving = f.row_moving;
    uint32_t* col_moving = f.row_moving + by;
    const uint32_t w = static_cast<uint32_t>(f.width), h = static_cast<uint32_t>(f.height);
    const uint32_t b = static_cast<uint32_t>(f.blksize), s = static_cast<uint32_t>(f.step);
    const uint32_t inside_rows = (h > b ? h - b : 0) / s, inside_cols = (w > b ? w - b : 0) / s;
    const uint32_t interior_rows = by > 2 ? by - 2 : 0, interior_cols = bx > 2 ? bx - 2 : 0;
    const uint32_t last_row = min(inside_rows, interior_rows), last_col = min(inside_cols, interior_cols);
    const uint32_t row = blockIdx.x;
    if (threadIdx.x == 0) row_count = 0;
    __syncthreads();
    uint32_t count = 0;
    if (row >= 1 && row <= last_row)
        for (uint32_t col = 1 + threadIdx.x; col <= last_col; col += kFitThreads) {
            const uint32_t moving = block_in_picture(f, static_cast<int>(row * bx + col));
            count += moving;
            if (moving) atomicAdd(col_moving + col, 1u);
        }
    count = __reduce_add_sync(0xffffffffu, count);
    if ((threadIdx.x & 31) == 0 && count) atomicAdd(&row_count, count);
    __syncthreads();
    if (threadIdx.x == 0) row_moving[row] = row_count;
    if (!last_cta(f.done) || threadIdx.x != 0) return;
    uint32_t top = 0, bottom = 0, left = 0, right = 0;
    if (last_row >= 1 && last_col >= 1) {
        top = leading_band(row_moving, 1, true, last_row, last_col);
        bottom = leading_band(row_moving, last_row, false, last_row, last_col);
        left = leading_band(col_moving, 1, true, last_col, last_row);
        right = leading_band(col_moving, last_col, false, last_col, last_row);
    }
    const bool rows_paired = bands_pair(top, bottom), cols_paired = bands_pair(left, right);
    f.bands[kTop] = rows_paired ? 1 + top : 0u;
    f.bands[kBottom] = rows_paired ? last_row + 1 - bottom : by;
    f.bands[kLeft] = cols_paired ? 1 + left : 0u;
    f.bands[kRight] = cols_paired ? last_col + 1 - right : bx;
}

__device__ __forceinline__ uint32_t neighbour_agrees(const int32_t* field, int nb, int mvx, int mvy, int tolerance) {
    const int gx = field[nb * 2] - mvx, gy = field[nb * 2 + 1] - mvy;
    return (abs(gx) <= tolerance && abs(gy) <= tolerance) ? 1u : 0u;
}

// global.rs:762-816 (`block_base_weight`).
__device__ float block_base_weight(const FitArgs& f, int col, int row, int mvx, int mvy) {
    const int tolerance = 1 + (3 * f.step) / 10;
    const int ox = col * f.step, oy = row * f.step, size = f.blksize;
    const bool interior = col >= 1 && row >= 1 && col + 1 < f.blocks_x && row + 1 < f.blocks_y;
    const bool inside = ox + size <= f.width && oy + size <= f.height;
    const int tx = ox + mvx, ty = oy + mvy;
    const bool lands = tx >= 0 && tx + size <= f.width && ty >= 0 && ty + size <= f.height;
    const uint32_t r = static_cast<uint32_t>(row), c = static_cast<uint32_t>(col);
    const bool in_rows = r >= f.bands[kTop] && r < f.bands[kBottom];
    const bool in_cols = c >= f.bands[kLeft] && c < f.bands[kRight];
    if (!(interior && inside && lands && in_rows && in_cols)) return 0.0f;
    const int block = row * f.blocks_x + col;
    const uint32_t agreeing = neighbour_agrees(f.field, block - 1, mvx, mvy, tolerance) +
                              neighbour_agrees(f.field, block + 1, mvx, mvy, tolerance) +
                              neighbour_agrees(f.field, block - f.blocks_x, mvx, mvy, tolerance) +
                              neighbour_agrees(f.field, block + f.blocks_x, mvx, mvy, tolerance);
    return (static_cast<float>(agreeing) + kNeighbourPrior) / (4.0f + kNeighbourPrior);
}

// global.rs:951-962 (`residual_sq`).
__device__ __forceinline__ float residual_sq(float a, float b, float tx, float ty, float x, float y, float mx, float my) {
    const float px = (a - 1.0f) * x - b * y + tx;
    const float py = b * x + (a - 1.0f) * y + ty;
    const float rx = mx - px, ry = my - py;
    return rx * rx + ry * ry;
}

__device__ __forceinline__ float corner_shift_sq(float a, float b, float tx, float ty, float x, float y) {
    const float sx = a * x - b * y + tx - x;
    const float sy = b * x + a * y + ty - y;
    return sx * sx + sy * sy;
}

__device__ __forceinline__ bool beats_still(float model_score, float still_score, float weight) {
    const bool moving = weight > 0.0f && still_score > kMinMotionScore * weight;
    return moving && model_score <= kAcceptMargin * still_score;
}

// global.rs:918-939 (`reduce_lanes`): the fixed halving tree over a CTA's 256 slots of each lane.
__device__ __forceinline__ void reduce_lanes(float (*scratch)[kFitThreads]) {
#pragma unroll 1
    for (int stride = kFitThreads / 2; stride >= 1; stride >>= 1) {
        if (static_cast<int>(threadIdx.x) < stride)
#pragma unroll
            for (int lane = 0; lane < kFitLanes; ++lane) scratch[lane][threadIdx.x] += scratch[lane][threadIdx.x + stride];
        __syncthreads();
    }
}

__device__ __forceinline__ void write_reference(float* state, float valid, float a, float b, float tx, float ty) {
    state[kRefValid] = valid;
    state[kRef] = a;
    state[kRef + 1] = b;
    state[kRef + 2] = tx;
    state[kRef + 3] = ty;
}

// global.rs:579-738 (`mc_fit_finish`), run by the last CTA of the stage's launch: every thread adds
// its share of the partials in order, the halving tree adds the threads' sums.
template <int STAGE>
__device__ void finish_stage(const FitArgs& f, int groups, float (*scratch)[kFitThreads]) {
    __syncthreads();
#pragma unroll
    for (int lane = 0; lane < kFitLanes; ++lane) {
        float sum = 0.0f;
        for (int i = threadIdx.x; i < groups; i += kFitThreads) sum += __ldcg(f.partials + i * kFitLanes + lane);
        scratch[lane][threadIdx.x] = sum;
    }
    __syncthreads();
    reduce_lanes(scratch);
    if (threadIdx.x != 0) return;
    float* state = f.state;
    const float centre_x = static_cast<float>(f.width) * 0.5f, centre_y = static_cast<float>(f.height) * 0.5f;
    if (STAGE == kWeigh) {
        const float base = scratch[0][0], base_sad = scratch[1][0];
        const float safe_base = fmaxf(base, 1e-12f);
        state[kSadScale] = base > 0.0f ? base_sad / safe_base : 0.0f;
        state[kScaleLimit] = kUnlimitedScale;
        write_reference(state, 0.0f, 1.0f, 0.0f, 0.0f, 0.0f);
    } else if (STAGE == kGate) {
        const float* p = f.models + static_cast<int64_t>(f.prior_slot) * kModelWords;
        if (p[4] != 0.0f && beats_still(scratch[0][0], scratch[1][0], scratch[2][0])) {
            const float ctx = p[2] + p[0] * centre_x - p[1] * centre_y - centre_x;
            const float cty = p[3] + p[1] * centre_x + p[0] * centre_y - centre_y;
            state[kScaleLimit] = kFitInlierCap;
            write_reference(state, 1.0f, p[0], p[1], ctx, cty);
        }
    } else if (STAGE == kSolve || STAGE == kPolish) {
        const float weight = scratch[0][0];
        const float inverse_weight = 1.0f / fmaxf(weight, kMinFitWeight);
        const float mean_px = scratch[1][0] * inverse_weight, mean_py = scratch[2][0] * inverse_weight;
        const float mean_dx = scratch[3][0] * inverse_weight, mean_dy = scratch[4][0] * inverse_weight;
        const float spread = scratch[7][0] - weight * (mean_px * mean_px + mean_py * mean_py);
        const float dot = scratch[5][0] - weight * (mean_px * mean_dx + mean_py * mean_dy);
        const float cross = scratch[6][0] - weight * (mean_px * mean_dy - mean_py * mean_dx);
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
        const bool passes = beats_still(scratch[0][0], scratch[1][0], scratch[2][0]);
        const float zoom = sqrtf(a * a + b * b);
        const bool zoom_ok = fabsf(zoom - 1.0f) <= kMaxZoomChange;
        const bool roll_ok = a > 0.0f && fabsf(b) <= kMaxRollTan * a;
        const float fx = static_cast<float>(f.width), fy = static_cast<float>(f.height);
        const float limit = kMaxCornerShift * kMaxCornerShift;
        const bool top_ok = corner_shift_sq(a, b, tx, ty, 0.0f, 0.0f) <= limit && corner_shift_sq(a, b, tx, ty, fx, 0.0f) <= limit;
        const bool bottom_ok = corner_shift_sq(a, b, tx, ty, 0.0f, fy) <= limit && corner_shift_sq(a, b, tx, ty, fx, fy) <= limit;
        const bool accepted = ref_valid && passes && zoom_ok && roll_ok && top_ok && bottom_ok;
        float* m = f.models + static_cast<int64_t>(f.slot) * kModelWords;
        m[0] = accepted ? a : 1.0f;
        m[1] = accepted ? b : 0.0f;
        m[2] = accepted ? tx : 0.0f;
        m[3] = accepted ? ty : 0.0f;
        m[4] = accepted ? 1.0f : 0.0f;
    }
}

// global.rs:394-577 (`mc_fit_sums`): one stage's lane sums, one block per thread.
template <int STAGE>
__global__ void __launch_bounds__(kFitThreads) fit_sums_kernel(FitArgs f, float scale) {
    __shared__ float scratch[kFitLanes][kFitThreads];
#pragma unroll
    for (int lane = 0; lane < kFitLanes; ++lane) scratch[lane][threadIdx.x] = 0.0f;
    const int blocks = f.blocks_x * f.blocks_y;
    const int block = blockIdx.x * kFitThreads + threadIdx.x;
    if (block < blocks) {
        float* lanes[kFitLanes];
#pragma unroll
        for (int lane = 0; lane < kFitLanes; ++lane) lanes[lane] = &scratch[lane][threadIdx.x];
        const int col = block % f.blocks_x, row = block / f.blocks_x;
        const int mvx = f.field[block * 2], mvy = f.field[block * 2 + 1];
        const bool has_sad = f.sad != nullptr;
        const float block_sad = has_sad ? f.sad[block] : 0.0f;
        const float half = static_cast<float>(f.blksize) * 0.5f;
        const float centre_x = static_cast<float>(f.width) * 0.5f, centre_y = static_cast<float>(f.height) * 0.5f;
        const float block_x = static_cast<float>(col * f.step) + half - centre_x;
        const float block_y = static_cast<float>(row * f.step) + half - centre_y;
        const float shift_x = static_cast<float>(mvx), shift_y = static_cast<float>(mvy);
        float px = block_x, py = block_y, mx = shift_x, my = shift_y;
        if (!f.older_to_newer) {
            px = block_x + shift_x;
            py = block_y + shift_y;
            mx = -shift_x;
            my = -shift_y;
        }
        const float scale_sq = scale * scale;
        if (STAGE == kWeigh) {
            float base = block_base_weight(f, col, row, mvx, mvy);
            if (f.has_contrast) base *= contrast_weight(block_sad, f.sad[f.means_offset + block]);
            f.weights[block] = base;
            *lanes[0] = base;
            *lanes[1] = base * block_sad;
        } else {
            float matched = f.weights[block];
            if (has_sad) {
                const float sad_scale = f.state[kSadScale];
                const float safe = fmaxf(sad_scale, 1e-12f);
                const float ratio = block_sad / safe;
                const float ratio_sq = ratio * ratio;
                const float sad_weight = 1.0f / (1.0f + ratio_sq * ratio_sq);
                matched *= sad_scale > 0.0f ? sad_weight : 1.0f;
            }
            const bool ref_valid = f.state[kRefValid] != 0.0f;
            const float ref_sq =
                residual_sq(f.state[kRef], f.state[kRef + 1], f.state[kRef + 2], f.state[kRef + 3], px, py, mx, my);
            if (STAGE == kSolve || STAGE == kPolish) {
                const float limited = fminf(scale, f.state[kScaleLimit]);
                const float limited_sq = limited * limited;
                const float damping = 1.0f / (1.0f + ref_sq / limited_sq);
                float residual_weight = damping * damping;
                if (STAGE == kPolish) residual_weight = ref_sq <= limited_sq ? 1.0f : 0.0f;
                const bool still = mvx == 0 && mvy == 0;
                const float zero_weight = still ? kZeroVectorWeight : 1.0f;
                const float fit_weight = ref_valid ? residual_weight : 1.0f;
                const float weight = matched * zero_weight * fit_weight;
                const float dot = px * mx + py * my;
                const float cross = px * my - py * mx;
                const float spread = px * px + py * py;
                *lanes[0] = weight;
                *lanes[1] = weight * px;
                *lanes[2] = weight * py;
                *lanes[3] = weight * mx;
                *lanes[4] = weight * my;
                *lanes[5] = weight * dot;
                *lanes[6] = weight * cross;
                *lanes[7] = weight * spread;
            } else {
                float model_sq = ref_sq;
                if (STAGE == kGate) {
                    const float* p = f.models + static_cast<int64_t>(f.prior_slot) * kModelWords;
                    model_sq = residual_sq(p[0], p[1], p[2], p[3], px + centre_x, py + centre_y, mx, my);
                }
                const float motion_sq = mx * mx + my * my;
                *lanes[0] = matched * fminf(model_sq, scale_sq);
                *lanes[1] = matched * fminf(motion_sq, scale_sq);
                *lanes[2] = matched;
            }
        }
    }
    __syncthreads();
    reduce_lanes(scratch);
    if (threadIdx.x < kFitLanes) f.partials[blockIdx.x * kFitLanes + threadIdx.x] = scratch[threadIdx.x][0];
    if (last_cta(f.done)) finish_stage<STAGE>(f, static_cast<int>(gridDim.x), scratch);
}


template <int STAGE>
void fit_stage(const FitArgs& f, int groups, float scale, cudaStream_t s) {
    fit_sums_kernel<STAGE><<<groups, kFitThreads, 0, s>>>(f, scale);
}

}  // namespace

// The scratch: 8 state words, 4 band words, the launch count (and 3 spare), blocks + 2 line counts
// (blocks_x + blocks_y never exceeds blocks + 1), one weight per block, 8 partials per 256 blocks.
size_t model_fit_scratch_floats(int blocks) {
    const size_t groups = (static_cast<size_t>(blocks) + kFitThreads - 1) / kFitThreads;
    return 8 + 4 + 4 + (static_cast<size_t>(blocks) + 2) + static_cast<size_t>(blocks) + groups * kFitLanes;
}

cudaError_t launch_compose_models(const float* models, const uint32_t* gaps, float* out, int neighbours, int max_steps,
                                  int past_neighbours, cudaStream_t s) {
    if (!models || !gaps || !out || neighbours < 1 || max_steps < 0) return cudaErrorInvalidValue;
    compose_kernel<<<(neighbours + 31) / 32, 32, 0, s>>>(models, gaps, out, neighbours, max_steps, past_neighbours);
    return cudaGetLastError();
}

cudaError_t launch_compose_inline(const float* models, const uint32_t* host_gaps, float* out, int neighbours,
                                  int max_steps, int past_neighbours, cudaStream_t s) {
    if (!models || !out || neighbours < 1 || max_steps < 0 || neighbours * max_steps > kMaxInlineGaps)
        return cudaErrorInvalidValue;
    InlineGaps gaps{};
    for (int i = 0; i < neighbours * max_steps; ++i) gaps.g[i] = host_gaps[i];
    compose_inline_kernel<<<(neighbours + 31) / 32, 32, 0, s>>>(models, gaps, out, neighbours, max_steps,
                                                                past_neighbours);
    return cudaGetLastError();
}

cudaError_t launch_block_means(const float* plane, float* out, int width, int height, int blksize, int step,
                               cudaStream_t s) {
    if (!plane || !out || width < 1 || height < 1 || blksize < 1 || step < 1) return cudaErrorInvalidValue;
    const int bx = (width + step - 1) / step > 1 ? (width + step - 1) / step : 1;
    const int by = (height + step - 1) / step > 1 ? (height + step - 1) / step : 1;
    block_means_kernel<<<(bx * by + 255) / 256, 256, 0, s>>>(plane, out, width, height, blksize, step, bx, bx * by);
    return cudaGetLastError();
}

cudaError_t launch_high_pass(const float* plane, float* rows, float* out, int width, int height, int radius,
                             cudaStream_t s) {
    if (!plane || !rows || !out || width < 1 || height < 1 || radius < 0) return cudaErrorInvalidValue;
    const dim3 grid((width + 15) / 16, (height + 15) / 16);
    box_rows_kernel<<<grid, 256, 0, s>>>(plane, rows, width, height, radius);
    high_pass_cols_kernel<<<grid, 256, 0, s>>>(plane, rows, out, width, height, radius);
    return cudaGetLastError();
}

cudaError_t launch_model_identity(float* models, int slot, cudaStream_t s) {
    if (!models || slot < 0) return cudaErrorInvalidValue;
    model_identity_kernel<<<1, 1, 0, s>>>(models, slot);
    return cudaGetLastError();
}

cudaError_t launch_model_fit(const ModelFitLaunch& l, cudaStream_t s) {
    if (!l.field || !l.models || !l.scratch || l.width < 1 || l.height < 1 || l.blksize < 1 || l.step < 1 ||
        l.slot < 0 || (l.has_contrast && !l.sad))
        return cudaErrorInvalidValue;
    FitArgs f{};
    f.field = l.field;
    f.sad = l.sad;
    f.has_contrast = l.sad && l.has_contrast ? 1 : 0;
    f.means_offset = l.means_offset;
    f.older_to_newer = l.older_to_newer ? 1 : 0;
    f.width = l.width;
    f.height = l.height;
    f.blksize = l.blksize;
    f.step = l.step;
    f.blocks_x = (l.width + l.step - 1) / l.step > 1 ? (l.width + l.step - 1) / l.step : 1;
    f.blocks_y = (l.height + l.step - 1) / l.step > 1 ? (l.height + l.step - 1) / l.step : 1;
    const int blocks = f.blocks_x * f.blocks_y;
    const int groups = (blocks + kFitThreads - 1) / kFitThreads;
    f.state = l.scratch;
    f.bands = reinterpret_cast<uint32_t*>(l.scratch + 8);
    f.done = reinterpret_cast<unsigned*>(l.scratch + 12);
    f.row_moving = reinterpret_cast<uint32_t*>(l.scratch + 16);
    f.weights = l.scratch + 16 + (blocks + 2);
    f.partials = f.weights + blocks;
    f.models = l.models;
    f.prior_slot = l.prior >= 0 ? l.prior : 0;
    f.slot = l.slot;
    // global/fit.rs:212-234: bars; weigh; the gate on a prior; solves at 16, 8, 4, 2; polish; score.
    // The launch count and the line counts start at zero; each launch's last CTA leaves the count at 0.
    cudaError_t e = cudaMemsetAsync(f.done, 0, (4 + static_cast<size_t>(blocks) + 2) * sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    fit_bands_kernel<<<f.blocks_y, kFitThreads, 0, s>>>(f);
    fit_stage<kWeigh>(f, groups, kFitInlierCap, s);
    if (l.prior >= 0) fit_stage<kGate>(f, groups, kFitInlierCap, s);
    for (float scale : {16.0f, 8.0f, 4.0f, 2.0f}) fit_stage<kSolve>(f, groups, scale, s);
    fit_stage<kPolish>(f, groups, kFitInlierCap, s);
    fit_stage<kScore>(f, groups, kFitInlierCap, s);
    return cudaGetLastError();
}

}  // namespace avd
