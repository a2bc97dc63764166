// The colour grain gains on sm_100a: the block means of a frame, each reading's cell sums, the
// window's sums and the two-pass fit of the grain model into per-cell log gains, which the NL4D
// filter reads at each reference patch's colour.
//
// Reference behaviour (av-denoise-core/src/noise):
//   kernels/colour.rs:187-340     `noise_colour_means`: each 16x16 block's mean luma, Cb and Cr on
//                                 the 8-bit scale, on the luma and the chroma noise grids.
//   kernels/colour.rs:342-470     `noise_colour_accumulate`, `noise_colour_window`: fixed-point cell
//                                 sums per frame, decoded and added oldest first over the window.
//   kernels/colour.rs:472-559     `noise_colour_levels`: each cell's kept blocks and level.
//   kernels/colour_fit.rs:341-1125 the brightness base, the wide-kernel lift, the cell table, the
//                                 ceilings and the gains; noise/colour.rs:630-680 runs them twice.
//
// Design. The reference runs the fit as ten launches; here it is five per fold: levels + base (one
// CTA per plane), the Gaussian-kernel lift (61 CTAs per plane, 8 lanes per query), table + ceilings
// + second levels + second base (one CTA per plane), the lift again, and table + gains. Every sum
// keeps the reference kernels' order (per-thread strided partials folded in halving rounds, lanes
// added in order), every operation rounds on its own (this file is built with -fmad=false), and the
// transcendental functions are the mirrors, so the results equal the oracle's bit for bit.

#include <cfloat>
#include <cstdint>

#include "colour_lookup.cuh"
#include "kernels.h"

namespace avd {
namespace {

using namespace colour;

constexpr int kNB = 16;
constexpr int kMeanThreads = 64;
constexpr int kFitThreads = 256;
constexpr int kLanes = 8;
constexpr int kQueries = 2 * kCells;
constexpr int kWords = 69;
constexpr int W_COUNT = 0, W_LOG = 1, W_LUMA = 2, W_CB = 3, W_CR = 4, W_HIST = 5;
constexpr int kHistBins = 64;
constexpr float kLogMin = -3.5f, kLogStep = 0.125f;
constexpr float kLogMax = kLogMin + static_cast<float>(kHistBins) * kLogStep;
constexpr float kLogFixed = 2048.0f, kMeanFixed = 16.0f;
constexpr float kStaticGate = 1.5f / 255.0f;
constexpr float kSqrt2 = 1.41421356237309504880f;
constexpr float kLn2 = 0.693147180559945309f;
constexpr int kKnots = 17, kLastKnot = 16;
constexpr float kKnotStep = 255.0f / static_cast<float>(kLastKnot);
constexpr float kRidge = 1.0e-5f;
constexpr int CF_LUMA = 0, CF_CB = 1, CF_CR = 2, CF_WEIGHT = 3, CF_RESIDUAL = 4, kCellFields = 5;
constexpr int P_PRIOR = kKnots, P_POPULATED = kKnots + 1, P_BLOCKS = kKnots + 2, P_LUMA_LOW = kKnots + 3,
              P_LUMA_HIGH = kKnots + 4;
constexpr int kNormRecords = kBrightnessBins, kHistEdges = kHistBins + 1;

// cos and sin of each hue sector's centre angle, -pi + (s + 0.5) pi / 6, correctly rounded.
constexpr float kC15 = 0.965925826289068287f, kS15 = 0.258819045102520762f, kH45 = 0.707106781186547524f;
__constant__ float kSectorCos[12] = {-kC15, -kH45, -kS15, kS15, kH45, kC15, kC15, kH45, kS15, -kS15, -kH45, -kC15};
__constant__ float kSectorSin[12] = {-kS15, -kH45, -kC15, -kC15, -kH45, -kS15, kS15, kH45, kC15, kC15, kH45, kS15};
__constant__ float kSatCentres[6] = {3.0f, 9.0f, 16.0f, 25.0f, 37.0f, 51.0f};

// ---- block means (colour.rs:187-340) ------------------------------------------------------------

template <int SPW, bool FLOAT>
__device__ __forceinline__ float read_sample(const uint32_t* plane, int64_t index) {
    const uint32_t word = __ldg(plane + index / SPW);
    if (FLOAT) return __uint_as_float(word);
    constexpr int kBits = 32 / SPW;
    constexpr uint32_t kMask = SPW == 1 ? 0xFFFFFFFFu : ((1u << kBits) - 1u);
    return static_cast<float>((word >> ((index % SPW) * kBits)) & kMask);
}

template <int SPW, bool FLOAT>
__device__ float rectangle_sum(const uint32_t* plane, int left, int top, int right, int bottom, int stride) {
    float sum = 0.0f;
    for (int y = top + static_cast<int>(threadIdx.x) / 16; y < bottom; y += 4)
        for (int x = left + static_cast<int>(threadIdx.x) % 16; x < right; x += 16)
            sum = __fadd_rn(sum, read_sample<SPW, FLOAT>(plane, static_cast<int64_t>(y) * stride + x));
    return sum;
}

template <int SPW, bool FLOAT>
__global__ void __launch_bounds__(kMeanThreads) colour_means_kernel(ColourMeansLaunch a) {
    __shared__ float ls[kMeanThreads], bs[kMeanThreads], rs[kMeanThreads];
    const int cw = (a.width + (1 << a.shift_x) - 1) >> a.shift_x, ch = (a.height + (1 << a.shift_y) - 1) >> a.shift_y;
    const int lbx = (a.width + kNB - 1) / kNB, lby = (a.height + kNB - 1) / kNB;
    const int cbx = (cw + kNB - 1) / kNB, cby = (ch + kNB - 1) / kNB;
    const bool in_luma = static_cast<int>(blockIdx.y) < lby;
    const int bx = blockIdx.x, by = in_luma ? blockIdx.y : blockIdx.y - lby;
    const int bxn = in_luma ? lbx : cbx, byn = in_luma ? lby : cby;
    const bool active = bx < bxn && by < byn;
    const int sx = 1 << a.shift_x, sy = 1 << a.shift_y;
    const int left = bx * kNB, top = by * kNB;
    const int right = min(left + kNB, in_luma ? a.width : cw), bottom = min(top + kNB, in_luma ? a.height : ch);
    // A luma block's chroma area rounds outwards, and a chroma block's luma area clips to the plane.
    const int ll = in_luma ? left : left * sx, lt = in_luma ? top : top * sy;
    const int lr = in_luma ? right : min(right * sx, a.width), lb = in_luma ? bottom : min(bottom * sy, a.height);
    const int cl = in_luma ? left >> a.shift_x : left, ct = in_luma ? top >> a.shift_y : top;
    const int cr = in_luma ? (right + sx - 1) >> a.shift_x : right, cb = in_luma ? (bottom + sy - 1) >> a.shift_y : bottom;
    const int t = threadIdx.x;
    ls[t] = bs[t] = rs[t] = 0.0f;
    if (active) {
        ls[t] = rectangle_sum<SPW, FLOAT>(a.luma, ll, lt, lr, lb, a.width);
        bs[t] = rectangle_sum<SPW, FLOAT>(a.cb, cl, ct, cr, cb, cw);
        rs[t] = rectangle_sum<SPW, FLOAT>(a.cr, cl, ct, cr, cb, cw);
    }
    __syncthreads();
#pragma unroll
    for (int half = kMeanThreads / 2; half > 0; half /= 2) {
        if (t < half) {
            ls[t] = __fadd_rn(ls[t], ls[t + half]);
            bs[t] = __fadd_rn(bs[t], bs[t + half]);
            rs[t] = __fadd_rn(rs[t], rs[t + half]);
        }
        __syncthreads();
    }
    if (active && t == 0) {
        const float lp = static_cast<float>((lr - ll) * (lb - lt)), cp = static_cast<float>((cr - cl) * (cb - ct));
        float* out = (in_luma ? a.luma_means : a.chroma_means) + (by * bxn + bx) * kMeanFields;
        out[0] = __fmul_rn(__fdiv_rn(ls[0], lp), a.eight_bit_scale);
        out[1] = __fsub_rn(__fmul_rn(__fadd_rn(__fdiv_rn(bs[0], cp), a.chroma_bias), a.eight_bit_scale), kChromaCentre);
        out[2] = __fsub_rn(__fmul_rn(__fadd_rn(__fdiv_rn(rs[0], cp), a.chroma_bias), a.eight_bit_scale), kChromaCentre);
    }
}

// ---- cell sums (colour.rs:342-470) --------------------------------------------------------------

__device__ __forceinline__ uint32_t histogram_bin(float log_grain) {
    const float position = floorf(__fdiv_rn(__fsub_rn(log_grain, kLogMin), kLogStep));
    return static_cast<uint32_t>(clampf(position, 0.0f, static_cast<float>(kHistBins - 1)));
}

__device__ __forceinline__ void add_block(int32_t* cells, int record, float log_grain, float luma, float cb,
                                          float cr) {
    int32_t* r = cells + static_cast<int64_t>(record) * kWords;
    const float clamped = clampf(log_grain, kLogMin, kLogMax);
    atomicAdd(r + W_COUNT, 1);
    atomicAdd(r + W_LOG, static_cast<int32_t>(roundf(__fmul_rn(clamped, kLogFixed))));
    atomicAdd(r + W_LUMA, static_cast<int32_t>(roundf(__fmul_rn(luma, kMeanFixed))));
    atomicAdd(r + W_CB, static_cast<int32_t>(roundf(__fmul_rn(cb, kMeanFixed))));
    atomicAdd(r + W_CR, static_cast<int32_t>(roundf(__fmul_rn(cr, kMeanFixed))));
    atomicAdd(r + W_HIST + histogram_bin(log_grain), 1);
}

template <int C, bool LUMA>
__global__ void __launch_bounds__(256) colour_accumulate_kernel(const float* __restrict__ records,
                                                                const float* __restrict__ means, int width,
                                                                int height, float grain_scale, int32_t* cells) {
    const int bxn = (width + kNB - 1) / kNB, byn = (height + kNB - 1) / kNB;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= bxn * byn) return;
    const int bw = min(kNB, width - (i % bxn) * kNB), bh = min(kNB, height - (i / bxn) * kNB);
    const float pixels = static_cast<float>(bw * bh);
    const float* r = records + static_cast<int64_t>(i) * (3 * C + 26);
    const float ml = __ldg(means + i * 3), mcb = __ldg(means + i * 3 + 1), mcr = __ldg(means + i * 3 + 2);
    const uint32_t cell = colour_cell(ml, mcb, mcr);
    const bool in_range = ml > 20.0f && ml < 240.0f;
    const uint32_t brightness = brightness_bin(ml);
    const bool neutral = saturation_of(mcb, mcr) < 8.0f;
    constexpr float kFloor = LUMA ? 0.05f : 0.03f;
#pragma unroll
    for (int c = 0; c < C; ++c) {
        const float mean = __fdiv_rn(r[c], pixels);
        const float ms = __fdiv_rn(r[C + c], pixels);
        const float var = fmaxf(__fsub_rn(ms, __fmul_rn(mean, mean)), 0.0f);
        const float grain = __fmul_rn(__fdiv_rn(__fsqrt_rn(var), kSqrt2), grain_scale);
        if (!(in_range && fabsf(mean) < kStaticGate && grain > kFloor)) continue;
        const float log_grain = log_mirror(grain);
        add_block(cells, c * kCells + static_cast<int>(cell), log_grain, ml, mcb, mcr);
        if (LUMA) {
            if (neutral) add_block(cells, C * kCells + static_cast<int>(brightness), log_grain, ml, mcb, mcr);
        } else {
            add_block(cells, C * kCells + c, log_grain, ml, mcb, mcr);
        }
    }
}

__global__ void colour_window_kernel(const int32_t* __restrict__ ring, int capacity, int first, int last, int words,
                                     float* __restrict__ window) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= words) return;
    const int word = i % kWords;
    const float scale =
        word == W_LOG ? 1.0f / kLogFixed : ((word >= W_LUMA && word < W_HIST) ? 1.0f / kMeanFixed : 1.0f);
    float sum = 0.0f;
    for (int f = first; f <= last; ++f)
        sum = __fadd_rn(sum, __fmul_rn(static_cast<float>(ring[static_cast<int64_t>(f % capacity) * words + i]), scale));
    window[i] = sum;
}

// ---- the fit (colour_fit.rs) ---------------------------------------------------------------------

__device__ __forceinline__ float knot_position(float luma) {
    return clampf(__fdiv_rn(luma, kKnotStep), 0.0f, static_cast<float>(kLastKnot));
}
__device__ __forceinline__ uint32_t knot_low(float position) {
    return min(static_cast<uint32_t>(floorf(position)), static_cast<uint32_t>(kLastKnot - 1));
}

// colour.rs:505-559 for one cell: its kept blocks under `ceiling` and its level.
__device__ void cell_level(const float* r, float ceiling, bool mean_level, float* kept_out, float* level_out) {
    float dropped = 0.0f, dropped_log = 0.0f;
    for (int bin = 0; bin < kHistBins; ++bin) {
        const float n = r[W_HIST + bin];
        const float low = __fadd_rn(kLogMin, __fmul_rn(static_cast<float>(bin), kLogStep));
        const float high = __fadd_rn(low, kLogStep);
        const float above = clampf(__fdiv_rn(__fsub_rn(high, ceiling), kLogStep), 0.0f, 1.0f);
        const float cut = fmaxf(low, ceiling);
        dropped = __fadd_rn(dropped, __fmul_rn(n, above));
        dropped_log = __fadd_rn(dropped_log, __fmul_rn(__fmul_rn(__fmul_rn(n, above), __fadd_rn(cut, high)), 0.5f));
    }
    const float kept = fmaxf(__fsub_rn(r[W_COUNT], dropped), 0.0f);
    float level = 0.0f;
    if (mean_level) {
        level = __fdiv_rn(__fsub_rn(r[W_LOG], dropped_log), fmaxf(kept, 1.0f));
    } else {
        const float target = __fmul_rn(kept, 0.5f);
        float below = 0.0f;
        bool found = false;
        for (int bin = 0; bin < kHistBins; ++bin) {
            const float n = r[W_HIST + bin];
            const float low = __fadd_rn(kLogMin, __fmul_rn(static_cast<float>(bin), kLogStep));
            const float high = __fadd_rn(low, kLogStep);
            const float above = clampf(__fdiv_rn(__fsub_rn(high, ceiling), kLogStep), 0.0f, 1.0f);
            const float share = __fsub_rn(1.0f, above);
            const float kept_count = __fmul_rn(n, share);
            if (!found && __fadd_rn(below, kept_count) >= target && kept_count > 0.0f) {
                level = __fadd_rn(
                    low, __fmul_rn(__fmul_rn(__fdiv_rn(__fsub_rn(target, below), kept_count), share), kLogStep));
                found = true;
            }
            below = __fadd_rn(below, kept_count);
        }
    }
    *kept_out = kept;
    *level_out = kept > 0.0f ? level : 0.0f;
}

// colour_fit.rs:534-686 (`solve_knots`), one thread.
__device__ void solve_knots(const float* sums, float* knots, float penalty) {
    constexpr int SUM_OFF = kKnots, SUM_RIGHT = kKnots + kLastKnot;
    float diag[kKnots], first[kKnots], second[kKnots], right[kKnots];
#pragma unroll
    for (int k = 0; k < kKnots; ++k) {
        diag[k] = sums[k];
        right[k] = sums[SUM_RIGHT + k];
        first[k] = k < kLastKnot ? sums[SUM_OFF + k] : 0.0f;
        second[k] = 0.0f;
    }
#pragma unroll
    for (int row = 0; row < kKnots - 2; ++row) {
        diag[row] = __fadd_rn(diag[row], penalty);
        diag[row + 1] = __fadd_rn(diag[row + 1], __fmul_rn(4.0f, penalty));
        diag[row + 2] = __fadd_rn(diag[row + 2], penalty);
        first[row] = __fsub_rn(first[row], __fmul_rn(2.0f, penalty));
        first[row + 1] = __fsub_rn(first[row + 1], __fmul_rn(2.0f, penalty));
        second[row] = __fadd_rn(second[row], penalty);
    }
    float scale[kKnots], ld[kKnots], l1[kKnots], l2[kKnots];
#pragma unroll
    for (int k = 0; k < kKnots; ++k) scale[k] = __fdiv_rn(1.0f, __fsqrt_rn(fmaxf(diag[k], 1.0e-30f)));
#pragma unroll
    for (int k = 0; k < kKnots; ++k) {
        float pivot = 1.0f + kRidge;
        if (k >= 1) pivot = __fsub_rn(pivot, __fmul_rn(l1[k - 1], l1[k - 1]));
        if (k >= 2) pivot = __fsub_rn(pivot, __fmul_rn(l2[k - 2], l2[k - 2]));
        const float root = __fsqrt_rn(fmaxf(pivot, 1.0e-12f));
        ld[k] = root;
        l1[k] = 0.0f;
        l2[k] = 0.0f;
        if (k + 1 < kKnots) {
            float below = __fmul_rn(__fmul_rn(first[k], scale[k]), scale[k + 1]);
            if (k >= 1) below = __fsub_rn(below, __fmul_rn(l2[k - 1], l1[k - 1]));
            l1[k] = __fdiv_rn(below, root);
        }
        if (k + 2 < kKnots) l2[k] = __fdiv_rn(__fmul_rn(__fmul_rn(second[k], scale[k]), scale[k + 2]), root);
    }
    float solution[kKnots], residual[kKnots];
#pragma unroll
    for (int k = 0; k < kKnots; ++k) {
        solution[k] = 0.0f;
        residual[k] = right[k];
    }
#pragma unroll
    for (int pass = 0; pass < 2; ++pass) {
        float fwd[kKnots], bwd[kKnots];
#pragma unroll
        for (int k = 0; k < kKnots; ++k) {
            float v = __fmul_rn(residual[k], scale[k]);
            if (k >= 1) v = __fsub_rn(v, __fmul_rn(l1[k - 1], fwd[k - 1]));
            if (k >= 2) v = __fsub_rn(v, __fmul_rn(l2[k - 2], fwd[k - 2]));
            fwd[k] = __fdiv_rn(v, ld[k]);
        }
#pragma unroll
        for (int k = kLastKnot; k >= 0; --k) {
            float v = fwd[k];
            if (k + 1 < kKnots) v = __fsub_rn(v, __fmul_rn(l1[k], bwd[k + 1]));
            if (k + 2 < kKnots) v = __fsub_rn(v, __fmul_rn(l2[k], bwd[k + 2]));
            bwd[k] = __fdiv_rn(v, ld[k]);
        }
#pragma unroll
        for (int k = 0; k < kKnots; ++k) solution[k] = __fadd_rn(solution[k], __fmul_rn(bwd[k], scale[k]));
#pragma unroll
        for (int k = 0; k < kKnots; ++k) {
            const float ridge = __fmul_rn(kRidge, diag[k]);
            float product = __fmul_rn(__fadd_rn(diag[k], ridge), solution[k]);
            if (k >= 1) product = __fadd_rn(product, __fmul_rn(first[k - 1], solution[k - 1]));
            if (k >= 2) product = __fadd_rn(product, __fmul_rn(second[k - 2], solution[k - 2]));
            if (k + 1 < kKnots) product = __fadd_rn(product, __fmul_rn(first[k], solution[k + 1]));
            if (k + 2 < kKnots) product = __fadd_rn(product, __fmul_rn(second[k], solution[k + 2]));
            residual[k] = __fsub_rn(right[k], product);
        }
    }
#pragma unroll
    for (int k = 0; k < kKnots; ++k) knots[k] = solution[k];
}

struct BaseShared {
    uint32_t lows[kCells];
    float fractions[kCells], weights[kCells], cell_levels[kCells];
    float root_p[kFitThreads], pop_p[kFitThreads], block_p[kFitThreads], low_p[kFitThreads], high_p[kFitThreads];
    float sums[3 * kKnots];
    float knots[kKnots];
};

// colour.rs:505-559 then colour_fit.rs:341-532 for plane blockIdx.x: the cells' levels under
// `ceilings` (null: every block kept) into `levels`, the brightness base into the plane header and
// each cell's fit record.
__device__ void levels_and_base(const float* window, const float* ceilings, bool mean_level, int plane, float* levels,
                                float* fit_cells, float* header, BaseShared& sh) {
    const int t = threadIdx.x, pc = plane * kCells;
    float root_sum = 0.0f, pop_sum = 0.0f, block_sum = 0.0f, span_low = FLT_MAX, span_high = -FLT_MAX;
    for (int cell = t; cell < kCells; cell += kFitThreads) {
        const float* r = window + static_cast<int64_t>(pc + cell) * kWords;
        float kept, level;
        cell_level(r, ceilings ? ceilings[pc + cell] : FLT_MAX, mean_level, &kept, &level);
        levels[(pc + cell) * 2] = kept;
        levels[(pc + cell) * 2 + 1] = level;
        const float divisor = fmaxf(r[W_COUNT], 1.0f);
        const float luma = __fdiv_rn(r[W_LUMA], divisor), cb = __fdiv_rn(r[W_CB], divisor),
                    cr = __fdiv_rn(r[W_CR], divisor);
        const bool populated = kept >= 8.0f;
        const float position = knot_position(luma);
        const uint32_t low = knot_low(position);
        const float weight = populated ? kept : 0.0f;
        sh.lows[cell] = low;
        sh.fractions[cell] = __fsub_rn(position, static_cast<float>(low));
        sh.weights[cell] = weight;
        sh.cell_levels[cell] = level;
        root_sum = __fadd_rn(root_sum, __fsqrt_rn(weight));
        pop_sum = __fadd_rn(pop_sum, populated ? 1.0f : 0.0f);
        block_sum = __fadd_rn(block_sum, kept);
        if (populated) {
            span_low = fminf(span_low, luma);
            span_high = fmaxf(span_high, luma);
        }
        float* f = fit_cells + static_cast<int64_t>(pc + cell) * kCellFields;
        f[CF_LUMA] = luma;
        f[CF_CB] = cb;
        f[CF_CR] = cr;
        f[CF_WEIGHT] = weight;
    }
    sh.root_p[t] = root_sum;
    sh.pop_p[t] = pop_sum;
    sh.block_p[t] = block_sum;
    sh.low_p[t] = span_low;
    sh.high_p[t] = span_high;
    __syncthreads();
    for (int half = kFitThreads / 2; half > 0; half /= 2) {
        if (t < half) {
            sh.root_p[t] = __fadd_rn(sh.root_p[t], sh.root_p[t + half]);
            sh.pop_p[t] = __fadd_rn(sh.pop_p[t], sh.pop_p[t + half]);
            sh.block_p[t] = __fadd_rn(sh.block_p[t], sh.block_p[t + half]);
            sh.low_p[t] = fminf(sh.low_p[t], sh.low_p[t + half]);
            sh.high_p[t] = fmaxf(sh.high_p[t], sh.high_p[t + half]);
        }
        __syncthreads();
    }
    // A cell of brightness bin b has its lower knot at b or b + 1, so knot k gathers bins k-2..k.
    if (t < kKnots) {
        const int knot = t;
        const int first_bin = max(knot, 2) - 2, last_bin = min(knot + 1, kBrightnessBins);
        float diagonal = 0.0f, off = 0.0f, right = 0.0f;
        for (int i = first_bin * kPerBrightness; i < last_bin * kPerBrightness; ++i) {
            const uint32_t low = sh.lows[i];
            const float fraction = sh.fractions[i], weight = sh.weights[i];
            const float low_share = __fsub_rn(1.0f, fraction);
            const bool is_low = low == static_cast<uint32_t>(knot), is_high = low + 1 == static_cast<uint32_t>(knot);
            const float low_square = is_low ? __fmul_rn(low_share, low_share) : 0.0f;
            const float high_square = is_high ? __fmul_rn(fraction, fraction) : 0.0f;
            const float low_tent = is_low ? low_share : 0.0f;
            const float high_tent = is_high ? fraction : 0.0f;
            const float cross = is_low ? __fmul_rn(low_share, fraction) : 0.0f;
            diagonal = __fadd_rn(diagonal, __fmul_rn(weight, __fadd_rn(low_square, high_square)));
            off = __fadd_rn(off, __fmul_rn(weight, cross));
            right = __fadd_rn(right, __fmul_rn(__fmul_rn(weight, sh.cell_levels[i]), __fadd_rn(low_tent, high_tent)));
        }
        sh.sums[knot] = diagonal;
        sh.sums[kKnots + kLastKnot + knot] = right;
        if (knot < kLastKnot) sh.sums[kKnots + knot] = off;
    }
    __syncthreads();
    if (t == 0) {
        const float populated = sh.pop_p[0];
        const bool has_cells = populated > 0.0f;
        const float mean_root = __fdiv_rn(sh.root_p[0], fmaxf(populated, 1.0f));
        const float penalty = __fmul_rn(__fmul_rn(2.0f, 2.0f), mean_root);
        float knots[kKnots];
        solve_knots(sh.sums, knots, penalty);
        for (int k = 0; k < kKnots; ++k) {
            sh.knots[k] = has_cells ? knots[k] : 0.0f;
            header[k] = sh.knots[k];
        }
        const float blocks = sh.block_p[0];
        header[P_PRIOR] = __fmul_rn(0.002f, blocks);
        header[P_POPULATED] = has_cells ? 1.0f : 0.0f;
        header[P_BLOCKS] = blocks;
        header[P_LUMA_LOW] = has_cells ? sh.low_p[0] : 0.0f;
        header[P_LUMA_HIGH] = has_cells ? sh.high_p[0] : 255.0f;
    }
    __syncthreads();
    for (int cell = t; cell < kCells; cell += kFitThreads) {
        const uint32_t low = sh.lows[cell];
        const float base = __fadd_rn(sh.knots[low], __fmul_rn(__fsub_rn(sh.knots[low + 1], sh.knots[low]),
                                                              sh.fractions[cell]));
        fit_cells[static_cast<int64_t>(pc + cell) * kCellFields + CF_RESIDUAL] =
            sh.weights[cell] > 0.0f ? __fsub_rn(sh.cell_levels[cell], base) : 0.0f;
    }
}

__global__ void __launch_bounds__(kFitThreads) colour_fit_start_kernel(ColourFitLaunch a) {
    __shared__ BaseShared sh;
    const int plane = blockIdx.x;
    levels_and_base(a.window, nullptr, a.luma, plane, a.levels, a.fit_cells,
                    a.fit_planes + plane * kColourFitPlaneWords, sh);
}

__device__ __forceinline__ float brightness_base(const float* header, float luma) {
    const float held = clampf(luma, header[P_LUMA_LOW], header[P_LUMA_HIGH]);
    const float position = knot_position(held);
    const uint32_t low = knot_low(position);
    const float fraction = __fsub_rn(position, static_cast<float>(low));
    return __fadd_rn(header[low], __fmul_rn(__fsub_rn(header[low + 1], header[low]), fraction));
}

__device__ __forceinline__ void cell_centre(int cell, float* luma, float* cb, float* cr) {
    const int brightness = cell / kPerBrightness, ring = cell % kPerBrightness;
    *luma = __fmul_rn(__fadd_rn(static_cast<float>(brightness), 0.5f), kBrightnessStep);
    const int coloured = max(ring, 1) - 1;
    const int level = coloured / kHueBins + 1, sector = coloured % kHueBins;
    const float saturation = ring == 0 ? 0.0f : kSatCentres[level];
    *cb = __fmul_rn(saturation, kSectorCos[sector]);
    *cr = __fmul_rn(saturation, kSectorSin[sector]);
}

// colour_fit.rs:688-796 (`noise_colour_fit_kernel`): grid (queries * 8 / 256, planes); 8 lanes per
// query, lane l summing cells l, l + 8, ...; lane 0 adds the 8 partials in order.
__global__ void __launch_bounds__(kFitThreads) colour_fit_lift_kernel(ColourFitLaunch a) {
    __shared__ float cl[kCells], ccb[kCells], ccr[kCells], cw[kCells], lift[kCells];
    __shared__ float num[kFitThreads], den[kFitThreads];
    const int plane = blockIdx.y, pc = plane * kCells;
    const int t = threadIdx.x, lane = t % kLanes;
    const int query = (blockIdx.x * kFitThreads + t) / kLanes;
    const float* header = a.fit_planes + plane * kColourFitPlaneWords;
    for (int c = t; c < kCells; c += kFitThreads) {
        const float* f = a.fit_cells + static_cast<int64_t>(pc + c) * kCellFields;
        cl[c] = __fdiv_rn(f[CF_LUMA], 32.0f);
        ccb[c] = __fdiv_rn(f[CF_CB], 12.0f);
        ccr[c] = __fdiv_rn(f[CF_CR], 12.0f);
        cw[c] = f[CF_WEIGHT];
        lift[c] = __fmul_rn(f[CF_WEIGHT], f[CF_RESIDUAL]);
    }
    __syncthreads();
    const bool in_range = query < kQueries;
    const int qc = query % kCells;
    float luma = 0.0f, cb = 0.0f, cr = 0.0f;
    if (query >= kCells) {
        cell_centre(qc, &luma, &cb, &cr);
    } else {
        const float* f = a.fit_cells + static_cast<int64_t>(pc + qc) * kCellFields;
        luma = f[CF_LUMA];
        cb = f[CF_CB];
        cr = f[CF_CR];
    }
    const float ql = __fdiv_rn(luma, 32.0f), qcb = __fdiv_rn(cb, 12.0f), qcr = __fdiv_rn(cr, 12.0f);
    float n = 0.0f, d = 0.0f;
    for (int c = lane; c < kCells; c += kLanes) {
        const float w = cw[c];
        if (!(w > 0.0f)) continue;
        const float lg = __fsub_rn(ql, cl[c]), bg = __fsub_rn(qcb, ccb[c]), rg = __fsub_rn(qcr, ccr[c]);
        const float distance = __fadd_rn(__fadd_rn(__fmul_rn(lg, lg), __fmul_rn(bg, bg)), __fmul_rn(rg, rg));
        const float kernel = exp_mirror(__fmul_rn(-0.5f, distance));
        n = __fadd_rn(n, __fmul_rn(kernel, lift[c]));
        d = __fadd_rn(d, __fmul_rn(kernel, w));
    }
    num[t] = n;
    den[t] = d;
    __syncthreads();
    if (in_range && lane == 0) {
        float qn = 0.0f, qd = 0.0f;
        for (int o = 0; o < kLanes; ++o) {
            qn = __fadd_rn(qn, num[t + o]);
            qd = __fadd_rn(qd, den[t + o]);
        }
        const float total = __fadd_rn(qd, header[P_PRIOR]);
        const float lifted = total > 0.0f ? __fdiv_rn(qn, fmaxf(total, 1.0e-30f)) : 0.0f;
        a.bases[plane * kQueries + query] = __fadd_rn(brightness_base(header, luma), lifted);
    }
}

__device__ __forceinline__ float shrink(float value, float dead_zone) {
    const float size = fmaxf(__fsub_rn(fabsf(value), dead_zone), 0.0f);
    return value < 0.0f ? -size : size;
}

struct TableShared {
    float moves[kCells], populated[kCells];
};

// colour_fit.rs:798-886 (`noise_colour_fit_table`) for one plane into `table`.
__device__ void cell_table(const ColourFitLaunch& a, int plane, TableShared& sh) {
    const int t = threadIdx.x, pc = plane * kCells;
    const float dead_zone = a.luma ? 0.1f : 0.0f;
    const float* bases = a.bases + plane * kQueries;
    for (int c = t; c < kCells; c += kFitThreads) {
        const float weight = a.fit_cells[static_cast<int64_t>(pc + c) * kCellFields + CF_WEIGHT];
        const float level = a.levels[(pc + c) * 2 + 1];
        const float pull = __fdiv_rn(weight, __fadd_rn(weight, 15.0f));
        const float gap = shrink(__fsub_rn(level, bases[c]), dead_zone);
        sh.moves[c] = weight > 0.0f ? __fmul_rn(pull, gap) : 0.0f;
        sh.populated[c] = weight > 0.0f ? 1.0f : 0.0f;
    }
    __syncthreads();
    for (int c = t; c < kCells; c += kFitThreads) {
        const int brightness = c / kPerBrightness, ring = c % kPerBrightness;
        float sum = 0.0f, count = 0.0f;
        if (brightness > 0) {
            sum = __fadd_rn(sum, sh.moves[c - kPerBrightness]);
            count = __fadd_rn(count, sh.populated[c - kPerBrightness]);
        }
        if (brightness + 1 < kBrightnessBins) {
            sum = __fadd_rn(sum, sh.moves[c + kPerBrightness]);
            count = __fadd_rn(count, sh.populated[c + kPerBrightness]);
        }
        const int row = brightness * kPerBrightness;
        if (ring == 0) {
            float ring_sum = 0.0f, ring_count = 0.0f;
            for (int s = 0; s < kHueBins; ++s) {
                ring_sum = __fadd_rn(ring_sum, sh.moves[row + 1 + s]);
                ring_count = __fadd_rn(ring_count, sh.populated[row + 1 + s]);
            }
            if (ring_count > 0.0f) {
                sum = __fadd_rn(sum, __fdiv_rn(ring_sum, ring_count));
                count = __fadd_rn(count, 1.0f);
            }
        } else {
            const int level = (ring - 1) / kHueBins, sector = (ring - 1) % kHueBins;
            const int less = level == 0 ? row : c - kHueBins;
            sum = __fadd_rn(sum, sh.moves[less]);
            count = __fadd_rn(count, sh.populated[less]);
            if (level + 2 < kLevels) {
                sum = __fadd_rn(sum, sh.moves[c + kHueBins]);
                count = __fadd_rn(count, sh.populated[c + kHueBins]);
            }
            const int start = row + 1 + level * kHueBins;
            const int next = start + (sector + 1) % kHueBins, prev = start + (sector + kHueBins - 1) % kHueBins;
            sum = __fadd_rn(sum, __fadd_rn(sh.moves[next], sh.moves[prev]));
            count = __fadd_rn(count, __fadd_rn(sh.populated[next], sh.populated[prev]));
        }
        const float filled = count > 0.0f ? __fdiv_rn(sum, fmaxf(count, 1.0f)) : 0.0f;
        const float cell_move = sh.populated[c] > 0.0f ? sh.moves[c] : filled;
        a.table[pc + c] = __fadd_rn(bases[kCells + c], cell_move);
    }
}

// The first fit's table, each cell's ceiling (colour_fit.rs:888-912: the table at the cell's mean
// colour plus ln 2), then the second fit's levels and base.
__global__ void __launch_bounds__(kFitThreads) colour_fit_refit_kernel(ColourFitLaunch a) {
    __shared__ union {
        TableShared table;
        BaseShared base;
    } sh;
    const int plane = blockIdx.x, pc = plane * kCells;
    cell_table(a, plane, sh.table);
    __syncthreads();
    for (int c = threadIdx.x; c < kCells; c += kFitThreads) {
        const float* r = a.window + static_cast<int64_t>(pc + c) * kWords;
        const float divisor = fmaxf(r[W_COUNT], 1.0f);
        const float model = table_value(a.table + pc, __fdiv_rn(r[W_LUMA], divisor), __fdiv_rn(r[W_CB], divisor),
                                        __fdiv_rn(r[W_CR], divisor));
        a.ceilings[pc + c] = r[W_COUNT] > 0.0f ? __fadd_rn(model, kLn2) : FLT_MAX;
    }
    __syncthreads();
    levels_and_base(a.window, a.ceilings, a.luma, plane, a.levels, a.fit_cells,
                    a.fit_planes + plane * kColourFitPlaneWords, sh.base);
}

struct GainShared {
    float hist[kNormRecords * kHistBins], cumulative[kNormRecords * kHistEdges], shifts[kNormRecords];
    float below[kFitThreads], above[kFitThreads];
    float normaliser[2];
};

__device__ float shifted_share(const GainShared& g, float position) {
    float share = 0.0f;
    for (int r = 0; r < kNormRecords; ++r) {
        const float offset = __fsub_rn(__fsub_rn(position, g.shifts[r]), kLogMin);
        const float clamped = clampf(__fdiv_rn(offset, kLogStep), 0.0f, static_cast<float>(kHistBins));
        const uint32_t bin = min(static_cast<uint32_t>(floorf(clamped)), static_cast<uint32_t>(kHistBins - 1));
        const float fraction = __fsub_rn(clamped, static_cast<float>(bin));
        share = __fadd_rn(share, __fadd_rn(g.cumulative[r * kHistEdges + bin],
                                           __fmul_rn(fraction, g.hist[r * kHistBins + bin])));
    }
    return share;
}

// The second fit's table, then colour_fit.rs:937-1100 (`noise_colour_fit_gains`).
__global__ void __launch_bounds__(kFitThreads) colour_fit_finish_kernel(ColourFitLaunch a) {
    __shared__ union {
        TableShared table;
        GainShared gain;
    } sh;
    const int plane = blockIdx.x, pc = plane * kCells, t = threadIdx.x;
    cell_table(a, plane, sh.table);
    __syncthreads();
    GainShared& g = sh.gain;
    const bool curve_valid = a.derived[kColourDerivedCurveWord] != 0.0f;
    if (t < kNormRecords) {
        float shift = 0.0f;
        if (a.luma) {
            const float ratio = a.curve[t];
            shift = -log_mirror(curve_valid && ratio > 0.0f ? ratio : 1.0f);
        }
        g.shifts[t] = shift;
    }
    const int extra = a.planes * kCells;
    for (int v = t; v < kNormRecords * kHistBins; v += kFitThreads) {
        const int r = v / kHistBins, bin = v % kHistBins;
        float count = 0.0f;
        if (a.luma)
            count = a.window[static_cast<int64_t>(extra + r) * kWords + W_HIST + bin];
        else if (r == 0)
            count = a.window[static_cast<int64_t>(extra + plane) * kWords + W_HIST + bin];
        g.hist[v] = count;
    }
    __syncthreads();
    if (t < kNormRecords) {
        float running = 0.0f;
        g.cumulative[t * kHistEdges] = running;
        for (int bin = 0; bin < kHistBins; ++bin) {
            running = __fadd_rn(running, g.hist[t * kHistBins + bin]);
            g.cumulative[t * kHistEdges + bin + 1] = running;
        }
    }
    __syncthreads();
    float total = 0.0f;
    for (int r = 0; r < kNormRecords; ++r) total = __fadd_rn(total, g.cumulative[r * kHistEdges + kHistBins]);
    const float target = __fmul_rn(total, 0.5f);
    float best_below = -FLT_MAX, best_above = FLT_MAX;
    for (int point = t; point < kNormRecords * kHistEdges; point += kFitThreads) {
        const int r = point / kHistEdges, edge = point % kHistEdges;
        const float position = __fadd_rn(__fadd_rn(kLogMin, __fmul_rn(static_cast<float>(edge), kLogStep)), g.shifts[r]);
        if (shifted_share(g, position) < target)
            best_below = fmaxf(best_below, position);
        else
            best_above = fminf(best_above, position);
    }
    g.below[t] = best_below;
    g.above[t] = best_above;
    __syncthreads();
    for (int half = kFitThreads / 2; half > 0; half /= 2) {
        if (t < half) {
            g.below[t] = fmaxf(g.below[t], g.below[t + half]);
            g.above[t] = fminf(g.above[t], g.above[t + half]);
        }
        __syncthreads();
    }
    if (t == 0) {
        const float below = g.below[0], above = g.above[0];
        const float below_share = shifted_share(g, below), above_share = shifted_share(g, above);
        const float rise = fmaxf(__fsub_rn(above_share, below_share), 1.0e-30f);
        const float median =
            __fadd_rn(below, __fmul_rn(__fdiv_rn(__fsub_rn(target, below_share), rise), __fsub_rn(above, below)));
        const bool has_median = total > 0.0f && below > -FLT_MAX && above < FLT_MAX;
        g.normaliser[0] = has_median ? median : 0.0f;
        g.normaliser[1] = has_median ? 1.0f : 0.0f;
    }
    __syncthreads();
    const float* header = a.fit_planes + plane * kColourFitPlaneWords;
    const bool applies = header[P_POPULATED] > 0.0f && g.normaliser[1] > 0.0f;
    const float normaliser = g.normaliser[0];
    const float log_min = log_mirror(0.4f), log_max = log_mirror(3.0f);
    const float blocks = header[P_BLOCKS];
    const float block_ramp = __fdiv_rn(blocks, __fadd_rn(blocks, 256.0f));
    const float neutral_ramp = __fdiv_rn(total, __fadd_rn(total, 256.0f));
    const float ramp = a.luma ? __fmul_rn(block_ramp, neutral_ramp) : block_ramp;
    for (int c = t; c < kCells; c += kFitThreads) {
        float log_gain = __fsub_rn(a.table[pc + c], normaliser);
        if (a.luma)
            log_gain = __fadd_rn(log_gain, g.shifts[c / kPerBrightness]);
        else
            log_gain = clampf(log_gain, log_min, log_max);
        a.gains[pc + c] = applies ? __fmul_rn(ramp, log_gain) : 0.0f;
    }
}

__global__ void colour_lookup_kernel(const float* __restrict__ table, const float* __restrict__ colours, int n,
                                     float* __restrict__ values, float* __restrict__ gains) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = table_value(table, colours[3 * i], colours[3 * i + 1], colours[3 * i + 2]);
    values[i] = v;
    gains[i] = exp_mirror(v);
}

}  // namespace

size_t colour_records(int planes, bool luma) {
    return static_cast<size_t>(planes) * kCells + (luma ? kBrightnessBins : planes);
}

cudaError_t launch_colour_means(const ColourMeansLaunch& a, cudaStream_t s) {
    if (a.width < 1 || a.height < 1 || a.shift_x < 0 || a.shift_x > 1 || a.shift_y < 0 || a.shift_y > 1 ||
        !a.luma || !a.cb || !a.cr || !a.luma_means || !a.chroma_means)
        return cudaErrorInvalidValue;
    const int cw = (a.width + (1 << a.shift_x) - 1) >> a.shift_x, ch = (a.height + (1 << a.shift_y) - 1) >> a.shift_y;
    const int lbx = (a.width + kNB - 1) / kNB, lby = (a.height + kNB - 1) / kNB;
    const int cbx = (cw + kNB - 1) / kNB, cby = (ch + kNB - 1) / kNB;
    const dim3 grid(max(lbx, cbx), lby + cby);
    switch (a.samples_per_word * 2 + (a.is_float ? 1 : 0)) {
        case 8: colour_means_kernel<4, false><<<grid, kMeanThreads, 0, s>>>(a); break;
        case 4: colour_means_kernel<2, false><<<grid, kMeanThreads, 0, s>>>(a); break;
        case 3: colour_means_kernel<1, true><<<grid, kMeanThreads, 0, s>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_colour_accumulate(const float* records, const float* means, int width, int height, int channels,
                                     bool luma, float grain_scale, int32_t* cells, cudaStream_t s) {
    if (channels < 1 || channels > 2 || width < 1 || height < 1) return cudaErrorInvalidValue;
    const size_t words = colour_records(channels, luma) * kWords;
    cudaError_t e = cudaMemsetAsync(cells, 0, words * sizeof(int32_t), s);
    if (e != cudaSuccess) return e;
    const int blocks = ((width + kNB - 1) / kNB) * ((height + kNB - 1) / kNB);
    const int grid = (blocks + 255) / 256;
    if (channels == 1 && luma)
        colour_accumulate_kernel<1, true><<<grid, 256, 0, s>>>(records, means, width, height, grain_scale, cells);
    else if (channels == 1)
        colour_accumulate_kernel<1, false><<<grid, 256, 0, s>>>(records, means, width, height, grain_scale, cells);
    else if (luma)
        colour_accumulate_kernel<2, true><<<grid, 256, 0, s>>>(records, means, width, height, grain_scale, cells);
    else
        colour_accumulate_kernel<2, false><<<grid, 256, 0, s>>>(records, means, width, height, grain_scale, cells);
    return cudaGetLastError();
}

cudaError_t launch_colour_window(const int32_t* ring, int capacity, int first, int last, int words, float* window,
                                 cudaStream_t s) {
    if (capacity < 1 || last < first || last - first + 1 > capacity || words < 1) return cudaErrorInvalidValue;
    colour_window_kernel<<<(words + 255) / 256, 256, 0, s>>>(ring, capacity, first, last, words, window);
    return cudaGetLastError();
}

cudaError_t launch_colour_fit(const ColourFitLaunch& a, cudaStream_t s) {
    if (a.planes < 1 || a.planes > 2 || !a.window || !a.derived || (a.luma && !a.curve)) return cudaErrorInvalidValue;
    const dim3 lift_grid((kQueries * kLanes + kFitThreads - 1) / kFitThreads, a.planes);
    colour_fit_start_kernel<<<a.planes, kFitThreads, 0, s>>>(a);
    colour_fit_lift_kernel<<<lift_grid, kFitThreads, 0, s>>>(a);
    colour_fit_refit_kernel<<<a.planes, kFitThreads, 0, s>>>(a);
    colour_fit_lift_kernel<<<lift_grid, kFitThreads, 0, s>>>(a);
    colour_fit_finish_kernel<<<a.planes, kFitThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_colour_lookup(const float* table, const float* colours, int n, float* values, float* gains,
                                 cudaStream_t s) {
    if (n < 1) return cudaErrorInvalidValue;
    colour_lookup_kernel<<<(n + 127) / 128, 128, 0, s>>>(table, colours, n, values, gains);
    return cudaGetLastError();
}

}  // namespace avd
