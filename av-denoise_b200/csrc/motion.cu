// Block-matching motion search on sm_100a: the luma pyramid, the coarse pass on its smallest level
// and the seeded fine pass at full resolution that writes each block's vector and confidence.
//
// Reference behaviour (av-denoise-core/src/motion):
//   kernels/pyramid.rs:10-61     level 0 is lane 0 of a ring slot; each further level averages 2x2
//                                pixels, the odd last row/column repeating its edge pixel.
//   kernels/block_match.rs:117-215, 274-351, 656-760, 787-849
//                                one search per (block, neighbour): the block's pixels and the
//                                window the search reaches are staged clamped to the frame; every
//                                candidate's SAD sums |centre - neighbour| row by row, left to
//                                right; the lowest SAD wins with the first in row-major order on a
//                                tie, and the window's centre wins a tie with that pick.
//   kernels/block_match.rs:505-521  confidence = max(0, (T^2 - e^2) / (T^2 + e^2)),
//                                e = max(SAD - floor, 0).
//   analyse.rs:100-157           the coarse level: blksize max(b / 2^l, 2) times the coarse block
//                                factor, step max(s / 2^l, 1), its winner scaled by 2^l seeds every
//                                fine block it covers.
//   block_match.rs:213-265, 384-578 with candidates.rs  the camera model: a second window around
//                                each neighbour's prediction when it moves anything and lies outside
//                                the first window, winning only by more than 1/8 of the SAD floor
//                                (scaled to the coarse block on the coarse level); the winning
//                                window's mean SAD and edge bar go with its winner.
//
// Layout in HBM: the pyramid holds, level after level, `frame_count` slots of that level's
// pixels, each slot padded to a multiple of 8 floats (32 bytes). Vectors are (dx, dy) i32 pairs per
// block, `mv_stride` values per neighbour; confidence one f32 per block, `conf_stride` per
// neighbour.
//
// Design: one CTA per (block, neighbour); every thread owns one candidate offset and sums its SAD
// sequentially in the order above (the sum is bit-identical to the reference's for any grouping of
// candidates, because each SAD is a sequential f32 sum in a fixed order). The argmin packs
// (SAD bits, candidate index) into one 64-bit key: non-negative floats order like their bit
// patterns, so the minimum key is the lowest SAD with the lowest index, found with warp shuffles.

#include <algorithm>
#include <cstdint>

#include "camera_model.cuh"
#include "kernels.h"

namespace avd {
namespace {

constexpr int kMaxBlk = 32;
constexpr int kMaxRadius = 8;           // fine windows and escalation ceilings
constexpr int kAcquisitionRadius = 12;  // the camera model's deep coarse search (global/producer.rs:54-55)
constexpr float kNoSad = 1.0e30f;
constexpr float kModelCandidateBias = 0.125f;  // candidates.rs:6-11
constexpr int kMaxNeighbours = MotionLaunch::kMaxInlineSlots;

__device__ __forceinline__ int clamp_to(int v, int limit) { return v < 0 ? 0 : (v >= limit ? limit - 1 : v); }

__global__ void pyramid_level0_kernel(const float* __restrict__ ring, float* __restrict__ dst, int64_t pixels,
                                      int channels, int64_t src_slot_elems) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= pixels) return;
    dst[p] = ring[src_slot_elems + p * channels];
}

__global__ void pyramid_down_kernel(const float* __restrict__ src, float* __restrict__ dst, int src_w, int src_h,
                                    int dst_w, int dst_h) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= dst_w || y >= dst_h) return;
    const int sx = 2 * x, sy = 2 * y;
    const int sx1 = sx + 1 < src_w ? sx + 1 : sx;
    const int sy1 = sy + 1 < src_h ? sy + 1 : sy;
    const float tl = src[sy * src_w + sx], tr = src[sy * src_w + sx1];
    const float bl = src[sy1 * src_w + sx], br = src[sy1 * src_w + sx1];
    dst[y * dst_w + x] = __fmul_rn(__fadd_rn(__fadd_rn(__fadd_rn(tl, tr), bl), br), 0.25f);
}

struct SearchLevel {
    const float* pyramid;
    int width, height;
    int64_t level_base;  // first value of this level
    int64_t slot_pixels;
    int blksize, step, blocks_x, blocks_y;
};

// One window's result (block_match.rs:580-600, `WindowBest`): the winner, its SAD, the window's
// mean SAD (when measured), the edge bar (the lowest SAD off the outer ring when the winner sits on
// it, else 0) and the window's centre.
struct WinBest {
    int dx, dy;
    float sad, mean, bar;
    int cdx, cdy;
};

// candidates.rs:136-156 (`model_centre`): whether neighbour n's prediction adds a window of radius R
// beside the one around (sdx, sdy): the model moves anything and its point lies outside that window.
// Every thread of a CTA (or lane of a warp) reads the same words, so the answer is uniform.
__device__ __forceinline__ bool model_window(const float* predictions, int n, int ox, int oy, int blksize, int scale,
                                             int lw, int lh, int R, int sdx, int sdy, int* mdx, int* mdy) {
    if (!predictions) return false;
    const float* p = predictions + n * kAffineWords;
    model_point(p, ox, oy, blksize, scale, lw, lh, mdx, mdy);
    return predicts_motion(p) && (abs(*mdx - sdx) > R || abs(*mdy - sdy) > R);
}

// The best offset of one window, at thread 0. `sads` holds every candidate's SAD.
template <int R>
__device__ __forceinline__ void window_argmin(const float* sads, unsigned long long* warp_keys, int* best_index) {
    constexpr int kSide = 2 * R + 1;
    constexpr int kCand = kSide * kSide;
    const int t = threadIdx.x;
    unsigned long long key = ~0ull;
    for (int i = t; i < kCand; i += blockDim.x) {
        const float s = sads[i];
        // Only SADs below the 1e30 start count, and NaN never compares below it.
        if (s < kNoSad) {
            const unsigned long long k = (static_cast<unsigned long long>(__float_as_uint(s)) << 32) | static_cast<unsigned>(i);
            key = k < key ? k : key;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
        key = other < key ? other : key;
    }
    if ((t & 31) == 0) warp_keys[t >> 5] = key;
    __syncthreads();
    if (t == 0) {
        unsigned long long best = warp_keys[0];
        for (int w = 1; w < static_cast<int>(blockDim.x >> 5); ++w) best = warp_keys[w] < best ? warp_keys[w] : best;
        *best_index = best == ~0ull ? -1 : static_cast<int>(best & 0xffffffffu);
    }
}

// Stages the block (clamped) and the window around `centre` (clamped) and scores every candidate.
template <int R>
__device__ __forceinline__ void score_window(const SearchLevel& L, int64_t centre_base, int64_t nbr_base, int ox,
                                             int oy, int cdx, int cdy, float* centre_tile, float* window,
                                             float* sads) {
    constexpr int kSide = 2 * R + 1;
    const int b = L.blksize;
    const int wside = b + 2 * R;
    const int t = threadIdx.x;
    for (int i = t; i < b * b; i += blockDim.x) {
        const int py = i / b, px = i - py * b;
        const int sx = clamp_to(ox + px, L.width), sy = clamp_to(oy + py, L.height);
        centre_tile[i] = L.pyramid[centre_base + static_cast<int64_t>(sy) * L.width + sx];
    }
    const int wx0 = ox + cdx - R, wy0 = oy + cdy - R;
    for (int i = t; i < wside * wside; i += blockDim.x) {
        const int wy = i / wside, wx = i - wy * wside;
        const int sx = clamp_to(wx0 + wx, L.width), sy = clamp_to(wy0 + wy, L.height);
        window[i] = L.pyramid[nbr_base + static_cast<int64_t>(sy) * L.width + sx];
    }
    __syncthreads();
    for (int c = t; c < kSide * kSide; c += blockDim.x) {
        const int dy = c / kSide, dx = c - dy * kSide;
        float sad = 0.0f;
        for (int iy = 0; iy < b; ++iy) {
            const float* wrow = window + (iy + dy) * wside + dx;
            const float* crow = centre_tile + iy * b;
            for (int ix = 0; ix < b; ++ix) sad = __fadd_rn(sad, fabsf(__fsub_rn(crow[ix], wrow[ix])));
        }
        sads[c] = sad;
    }
    __syncthreads();
}

// The winner of a scored window around (cdx, cdy) (block_match.rs:720-785): the lowest SAD with the
// first row-major index, the centre winning a tie; the mean sums every SAD in row-major order;
// the edge bar is the lowest SAD off the outer ring (1e30 at radius 0) when the winner sits on it.
template <int R>
__device__ __forceinline__ WinBest window_result(const float* sads, int best_index, int cdx, int cdy, bool want_mean,
                                                 bool want_bar) {
    constexpr int kSide = 2 * R + 1;
    constexpr int kCand = kSide * kSide;
    WinBest r{cdx, cdy, kNoSad, 0.0f, 0.0f, cdx, cdy};
    if (best_index >= 0) {
        r.sad = sads[best_index];
        r.dx = cdx + best_index % kSide - R;
        r.dy = cdy + best_index / kSide - R;
    }
    const float centre_sad = sads[R * kSide + R];
    if (centre_sad <= r.sad) {
        r.sad = centre_sad;
        r.dx = cdx;
        r.dy = cdy;
    }
    if (want_mean) {
        float total = 0.0f;
        for (int i = 0; i < kCand; ++i) total = __fadd_rn(total, sads[i]);
        r.mean = __fmul_rn(total, __fdiv_rn(1.0f, static_cast<float>(kCand)));
    }
    if (want_bar && (abs(r.dx - cdx) == R || abs(r.dy - cdy) == R)) {
        float bar = kNoSad;
        for (int y = 1; y < kSide - 1; ++y)
            for (int x = 1; x < kSide - 1; ++x) bar = fminf(bar, sads[y * kSide + x]);
        r.bar = bar;
    }
    return r;
}

template <int R>
struct WindowScratch {
    float centre_tile[kMaxBlk * kMaxBlk];
    float window[(kMaxBlk + 2 * R) * (kMaxBlk + 2 * R)];
    float sads[(2 * R + 1) * (2 * R + 1)];
    unsigned long long warp_keys[((2 * R + 1) * (2 * R + 1) + 31) / 32];
    int best_index;
};

// One window around (cdx, cdy), the result at thread 0; every thread must call it.
template <int R>
__device__ __forceinline__ WinBest window_best(const SearchLevel& L, int64_t centre_base, int64_t nbr_base, int ox,
                                               int oy, int cdx, int cdy, WindowScratch<R>& w, bool want_mean,
                                               bool want_bar) {
    score_window<R>(L, centre_base, nbr_base, ox, oy, cdx, cdy, w.centre_tile, w.window, w.sads);
    window_argmin<R>(w.sads, w.warp_keys, &w.best_index);
    WinBest r{cdx, cdy, kNoSad, 0.0f, 0.0f, cdx, cdy};
    if (threadIdx.x == 0) r = window_result<R>(w.sads, w.best_index, cdx, cdy, want_mean, want_bar);
    return r;
}

struct SearchArgs {
    SearchLevel L;
    const uint32_t* neighbour_slots;  // null: the slots are `slots`
    uint32_t slots[kMaxNeighbours];
    int centre_slot;
    int32_t* mv_field;
    int mv_stride;
    // Coarse only: how coarse blocks map onto the fine grid.
    int level_scale, fine_blocks_x, fine_blocks_y, fine_step;
    // Fine only.
    int use_seed;
    float* confidence;
    int conf_stride;
    const float* noise;
    int sad_floor_word;
    float thsad;
    // Fine only, with escalation: the state the first pass records for it (escalate.rs:84-155):
    // sections `esc_section` floats apart of kept SAD, edge bar, and the winning window's centre.
    float* esc_state;
    int64_t esc_section;
    // The camera model (candidates.rs): 6 prediction words per neighbour, or null; its window wins
    // by more than 1/8 of noise word `sad_floor_word`, times `floor_scale` on the coarse level.
    const float* predictions;
    float floor_scale;
    // Fine only: winning SADs, then `sad_means` values on, the windows' mean SADs (conf layout).
    float* sad_out;
    int64_t sad_means;
};

__device__ __forceinline__ uint32_t search_slot(const SearchArgs& a, int n) {
    return a.neighbour_slots ? a.neighbour_slots[n] : a.slots[n];
}

// The model's bias: 1/8 of the window's SAD floor, scaled to the level (block_match.rs:156-159).
__device__ __forceinline__ float model_bias(const SearchArgs& a, float level_scale_factor) {
    if (!a.predictions || !a.noise) return 0.0f;
    return __fmul_rn(__fmul_rn(kModelCandidateBias, a.noise[a.sad_floor_word]), level_scale_factor);
}

// block_match.rs:520-578 (`search_candidates`) over the window around (sdx, sdy) and, when the
// camera model adds one, the window around its point, which replaces the first only when its SAD
// plus `bias` is lower. The result is valid at thread 0; every thread must call it.
template <int R>
__device__ __forceinline__ WinBest search_candidates(const SearchArgs& a, int bx, int by, int n, int sdx, int sdy,
                                                     int scale, float bias, bool want_mean, bool want_bar) {
    __shared__ WindowScratch<R> w;
    const int64_t cb = a.L.level_base + static_cast<int64_t>(a.centre_slot) * a.L.slot_pixels;
    const int64_t nb = a.L.level_base + static_cast<int64_t>(search_slot(a, n)) * a.L.slot_pixels;
    const int ox = bx * a.L.step, oy = by * a.L.step;
    WinBest best = window_best<R>(a.L, cb, nb, ox, oy, sdx, sdy, w, want_mean, want_bar);
    int mdx, mdy;
    if (model_window(a.predictions, n, ox, oy, a.L.blksize, scale, a.L.width, a.L.height, R, sdx, sdy, &mdx, &mdy)) {
        const WinBest ch = window_best<R>(a.L, cb, nb, ox, oy, mdx, mdy, w, want_mean, want_bar);
        if (threadIdx.x == 0 && __fadd_rn(ch.sad, bias) < best.sad) best = ch;
    }
    return best;
}

// block_match.rs:190-214: every fine block inside coarse block (bx, by)'s region takes the scaled
// winner; the last coarse block on each axis reaches the fine grid's edge.
__device__ __forceinline__ void seed_fine_blocks(const SearchArgs& a, int bx, int by, int n, int dx, int dy) {
    const int s = a.L.step * a.level_scale;
    const int c0 = min(bx * s / a.fine_step, a.fine_blocks_x);
    const int c1 = bx == a.L.blocks_x - 1 ? a.fine_blocks_x : min((bx + 1) * s / a.fine_step, a.fine_blocks_x);
    const int r0 = min(by * s / a.fine_step, a.fine_blocks_y);
    const int r1 = by == a.L.blocks_y - 1 ? a.fine_blocks_y : min((by + 1) * s / a.fine_step, a.fine_blocks_y);
    int32_t* mv = a.mv_field + static_cast<int64_t>(n) * a.mv_stride;
    for (int r = r0; r < r1; ++r)
        for (int c = c0; c < c1; ++c) {
            mv[(r * a.fine_blocks_x + c) * 2] = dx * a.level_scale;
            mv[(r * a.fine_blocks_x + c) * 2 + 1] = dy * a.level_scale;
        }
}

__device__ __forceinline__ float match_confidence(float sad, float floor, float thsad) {
    float excess = __fsub_rn(sad, floor);
    if (excess < 0.0f) excess = 0.0f;
    const float t2 = __fmul_rn(thsad, thsad);
    const float e2 = __fmul_rn(excess, excess);
    const float c = __fdiv_rn(__fsub_rn(t2, e2), __fadd_rn(t2, e2));
    return c < 0.0f ? 0.0f : c;
}

// The outputs of one fine block (block_match.rs:480-510 and escalate.rs:140-155): the vector, the
// escalation state, the SAD and window mean, and the confidence.
__device__ __forceinline__ void write_fine(const SearchArgs& a, int bx, int by, int n, const WinBest& b) {
    int32_t* mv = a.mv_field + static_cast<int64_t>(n) * a.mv_stride + (by * a.L.blocks_x + bx) * 2;
    mv[0] = b.dx;
    mv[1] = b.dy;
    const int64_t slot = static_cast<int64_t>(n) * a.conf_stride + by * a.L.blocks_x + bx;
    if (a.esc_state) {
        a.esc_state[slot] = b.sad;
        a.esc_state[a.esc_section + slot] = b.bar;
        a.esc_state[2 * a.esc_section + slot] = static_cast<float>(b.cdx);
        a.esc_state[3 * a.esc_section + slot] = static_cast<float>(b.cdy);
    }
    if (a.sad_out) {
        a.sad_out[slot] = b.sad;
        a.sad_out[a.sad_means + slot] = b.mean;
    }
    if (a.confidence) a.confidence[slot] = match_confidence(b.sad, a.noise[a.sad_floor_word], a.thsad);
}

template <int R>
__global__ void __launch_bounds__(((2 * R + 1) * (2 * R + 1) + 31) / 32 * 32) coarse_kernel(SearchArgs a) {
    const int bx = blockIdx.x, by = blockIdx.y, n = blockIdx.z;
    const WinBest b = search_candidates<R>(a, bx, by, n, 0, 0, a.level_scale, model_bias(a, a.floor_scale), false, false);
    if (threadIdx.x != 0) return;
    seed_fine_blocks(a, bx, by, n, b.dx, b.dy);
}

template <int R>
__global__ void __launch_bounds__(((2 * R + 1) * (2 * R + 1) + 31) / 32 * 32) fine_kernel(SearchArgs a) {
    const int bx = blockIdx.x, by = blockIdx.y, n = blockIdx.z;
    const int32_t* mv = a.mv_field + static_cast<int64_t>(n) * a.mv_stride + (by * a.L.blocks_x + bx) * 2;
    const int sdx = a.use_seed ? mv[0] : 0;
    const int sdy = a.use_seed ? mv[1] : 0;
    const WinBest b = search_candidates<R>(a, bx, by, n, sdx, sdy, 1, model_bias(a, 1.0f), a.sad_out != nullptr,
                                           a.esc_state != nullptr);
    if (threadIdx.x != 0) return;
    write_fine(a, bx, by, n, b);
}

// Register-blocked search for the common block sizes: one warp per (block, neighbour), several
// blocks per CTA. Each work item is one candidate row and three adjacent offsets along it (five for
// the wide coarse window of the camera model's first search); per block row it holds BLK + 2 (or
// BLK + 4) window values in registers and scores the offsets from them, so a SAD term costs well
// under one shared load instead of two. Every SAD is still the
// sequential row-major sum, so the vectors are the generic kernels' bit for bit.
template <int BLK, int R>
struct Blocked {
    static constexpr int kSide = 2 * R + 1;
    static constexpr int kWide = R > kMaxRadius ? 5 : 3;  // offsets per work item
    static constexpr int kGroups = (kSide + kWide - 1) / kWide;
    static constexpr int kItems = kSide * kGroups;
    static constexpr int kRows = BLK + 2 * R;
    static constexpr int kReach = kGroups * kWide + BLK - 1;             // columns the last group reads
    static constexpr int kStride = (kReach > kRows ? kReach : kRows) | 1;  // odd: spreads the banks
    static constexpr int kWarps = BLK >= 32 ? 2 : 4;
    static constexpr int kWindow = kStride * kRows;
};

template <int BLK, int R>
__device__ __forceinline__ void blocked_window(const SearchLevel& L, int64_t centre_base, int64_t nbr_base, int ox,
                                               int oy, int cdx, int cdy, float* centre_tile, float* window,
                                               float* sads, int lane, unsigned long long* best_key) {
    using B = Blocked<BLK, R>;
    for (int i = lane; i < BLK * BLK; i += 32) {
        const int py = i / BLK, px = i % BLK;
        centre_tile[i] = L.pyramid[centre_base + static_cast<int64_t>(clamp_to(oy + py, L.height)) * L.width +
                                   clamp_to(ox + px, L.width)];
    }
    const int wx0 = ox + cdx - R, wy0 = oy + cdy - R;
    for (int i = lane; i < B::kWindow; i += 32) {
        const int wy = i / B::kStride, wx = i % B::kStride;
        window[i] = L.pyramid[nbr_base + static_cast<int64_t>(clamp_to(wy0 + wy, L.height)) * L.width +
                              clamp_to(wx0 + wx, L.width)];
    }
    __syncwarp();
    for (int item = lane; item < B::kItems; item += 32) {
        const int dy = item / B::kGroups, dx0 = (item % B::kGroups) * B::kWide;
        float part[B::kWide];
#pragma unroll
        for (int k = 0; k < B::kWide; ++k) part[k] = 0.0f;
        for (int iy = 0; iy < BLK; ++iy) {
            const float* wrow = window + (iy + dy) * B::kStride + dx0;
            // The block row in registers, four samples per shared load (rows start 16-byte aligned).
            const float4* crow = reinterpret_cast<const float4*>(centre_tile + iy * BLK);
            float c[BLK];
#pragma unroll
            for (int q = 0; q < BLK / 4; ++q) {
                const float4 v = crow[q];
                c[4 * q] = v.x;
                c[4 * q + 1] = v.y;
                c[4 * q + 2] = v.z;
                c[4 * q + 3] = v.w;
            }
            float w[BLK + B::kWide - 1];
#pragma unroll
            for (int k = 0; k < BLK + B::kWide - 1; ++k) w[k] = wrow[k];
#pragma unroll
            for (int ix = 0; ix < BLK; ++ix) {
#pragma unroll
                for (int k = 0; k < B::kWide; ++k) part[k] = __fadd_rn(part[k], fabsf(__fsub_rn(c[ix], w[ix + k])));
            }
        }
#pragma unroll
        for (int k = 0; k < B::kWide; ++k)
            if (dx0 + k < B::kSide) sads[dy * B::kSide + dx0 + k] = part[k];
    }
    __syncwarp();
    unsigned long long key = ~0ull;
    for (int i = lane; i < B::kSide * B::kSide; i += 32) {
        const float v = sads[i];
        if (v < kNoSad) {
            const unsigned long long k = (static_cast<unsigned long long>(__float_as_uint(v)) << 32) | static_cast<unsigned>(i);
            key = k < key ? k : key;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
        key = other < key ? other : key;
    }
    *best_key = key;
}

template <int BLK, int R, bool COARSE>
__global__ void __launch_bounds__(Blocked<BLK, R>::kWarps * 32) blocked_kernel(SearchArgs a) {
    using B = Blocked<BLK, R>;
    __shared__ __align__(16) float centre_tiles[B::kWarps][BLK * BLK];
    __shared__ float windows[B::kWarps][B::kWindow];
    __shared__ float sad_buf[B::kWarps][B::kSide * B::kSide];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bx = blockIdx.x * B::kWarps + warp, by = blockIdx.y, n = blockIdx.z;
    if (bx >= a.L.blocks_x) return;  // the whole warp leaves; only warp-scoped syncs follow
    const int64_t centre_base = a.L.level_base + static_cast<int64_t>(a.centre_slot) * a.L.slot_pixels;
    const int64_t nbr_base = a.L.level_base + static_cast<int64_t>(search_slot(a, n)) * a.L.slot_pixels;
    const int ox = bx * a.L.step, oy = by * a.L.step;
    int cdx = 0, cdy = 0;
    if (!COARSE && a.use_seed) {
        const int32_t* mv = a.mv_field + static_cast<int64_t>(n) * a.mv_stride + (by * a.L.blocks_x + bx) * 2;
        cdx = mv[0];
        cdy = mv[1];
    }
    const bool want_mean = !COARSE && a.sad_out != nullptr, want_bar = !COARSE && a.esc_state != nullptr;
    unsigned long long key;
    blocked_window<BLK, R>(a.L, centre_base, nbr_base, ox, oy, cdx, cdy, centre_tiles[warp], windows[warp],
                           sad_buf[warp], lane, &key);
    WinBest best{cdx, cdy, kNoSad, 0.0f, 0.0f, cdx, cdy};
    if (lane == 0) best = window_result<R>(sad_buf[warp], key == ~0ull ? -1 : static_cast<int>(key & 0xffffffffu), cdx,
                                           cdy, want_mean, want_bar);
    int mdx, mdy;
    const int scale = COARSE ? a.level_scale : 1;
    if (model_window(a.predictions, n, ox, oy, BLK, scale, a.L.width, a.L.height, R, cdx, cdy, &mdx, &mdy)) {
        blocked_window<BLK, R>(a.L, centre_base, nbr_base, ox, oy, mdx, mdy, centre_tiles[warp], windows[warp],
                               sad_buf[warp], lane, &key);
        if (lane == 0) {
            const WinBest ch = window_result<R>(sad_buf[warp], key == ~0ull ? -1 : static_cast<int>(key & 0xffffffffu),
                                                mdx, mdy, want_mean, want_bar);
            if (__fadd_rn(ch.sad, model_bias(a, COARSE ? a.floor_scale : 1.0f)) < best.sad) best = ch;
        }
    }
    if (lane != 0) return;
    if (COARSE) {
        seed_fine_blocks(a, bx, by, n, best.dx, best.dy);
        return;
    }
    write_fine(a, bx, by, n, best);
}

// The fine pass at radius 0 (the HQ confidence pass scores every block where it stands): one thread
// per (block, neighbour). The single candidate's SAD is the same sequential row-major sum the
// windowed kernels take, so vectors, SADs and confidences are theirs bit for bit; a SAD that is not
// below the 1e30 start leaves the search's 1e30 (block_match.rs:735-742).
__device__ __forceinline__ float point_sad(const SearchArgs& a, int64_t centre_base, int64_t nbr_base, int ox, int oy,
                                           int cdx, int cdy) {
    const int b = a.L.blksize;
    float sad = 0.0f;
    for (int iy = 0; iy < b; ++iy) {
        const int64_t crow = centre_base + static_cast<int64_t>(clamp_to(oy + iy, a.L.height)) * a.L.width;
        const int64_t wrow = nbr_base + static_cast<int64_t>(clamp_to(oy + cdy + iy, a.L.height)) * a.L.width;
#pragma unroll 8
        for (int ix = 0; ix < b; ++ix) {
            const float c = __ldg(a.L.pyramid + crow + clamp_to(ox + ix, a.L.width));
            const float w = __ldg(a.L.pyramid + wrow + clamp_to(ox + cdx + ix, a.L.width));
            sad = __fadd_rn(sad, fabsf(__fsub_rn(c, w)));
        }
    }
    return sad;
}

__global__ void __launch_bounds__(128) zero_radius_fine_kernel(SearchArgs a) {
    const int bx = blockIdx.x * blockDim.x + threadIdx.x, by = blockIdx.y, n = blockIdx.z;
    if (bx >= a.L.blocks_x) return;
    const int32_t* mv = a.mv_field + static_cast<int64_t>(n) * a.mv_stride + (by * a.L.blocks_x + bx) * 2;
    const int cdx = a.use_seed ? mv[0] : 0;
    const int cdy = a.use_seed ? mv[1] : 0;
    const int64_t centre_base = a.L.level_base + static_cast<int64_t>(a.centre_slot) * a.L.slot_pixels;
    const int64_t nbr_base = a.L.level_base + static_cast<int64_t>(search_slot(a, n)) * a.L.slot_pixels;
    const int ox = bx * a.L.step, oy = by * a.L.step;
    // A window of one candidate: its SAD is the mean, and its winner always sits on the outer ring
    // with nothing inside it (block_match.rs:803-820).
    const float raw = point_sad(a, centre_base, nbr_base, ox, oy, cdx, cdy);
    WinBest best{cdx, cdy, raw <= kNoSad ? raw : kNoSad, raw, kNoSad, cdx, cdy};
    int mdx, mdy;
    if (model_window(a.predictions, n, ox, oy, a.L.blksize, 1, a.L.width, a.L.height, 0, cdx, cdy, &mdx, &mdy)) {
        const float mraw = point_sad(a, centre_base, nbr_base, ox, oy, mdx, mdy);
        const float msad = mraw <= kNoSad ? mraw : kNoSad;
        if (__fadd_rn(msad, model_bias(a, 1.0f)) < best.sad) best = WinBest{mdx, mdy, msad, mraw, kNoSad, mdx, mdy};
    }
    write_fine(a, bx, by, n, best);
}

template <int BLK, int R>
cudaError_t launch_blocked(bool coarse, const SearchArgs& a, dim3 grid, cudaStream_t s) {
    using B = Blocked<BLK, R>;
    dim3 g((grid.x + B::kWarps - 1) / B::kWarps, grid.y, grid.z);
    if (coarse) {
        blocked_kernel<BLK, R, true><<<g, B::kWarps * 32, 0, s>>>(a);
    } else {
        if constexpr (R <= kMaxRadius) {
            blocked_kernel<BLK, R, false><<<g, B::kWarps * 32, 0, s>>>(a);
        } else {
            return cudaErrorInvalidValue;
        }
    }
    return cudaGetLastError();
}

template <int R>
cudaError_t launch_search(bool coarse, const SearchArgs& a, dim3 grid, cudaStream_t s) {
    if (R >= 1) {
        switch (a.L.blksize) {
            case 8: return launch_blocked<8, R>(coarse, a, grid, s);
            case 16: return launch_blocked<16, R>(coarse, a, grid, s);
            case 32: return launch_blocked<32, R>(coarse, a, grid, s);
            default: break;
        }
    }
    if (R == 0 && !coarse) {
        zero_radius_fine_kernel<<<dim3((grid.x + 127) / 128, grid.y, grid.z), 128, 0, s>>>(a);
        return cudaGetLastError();
    }
    constexpr int kCand = (2 * R + 1) * (2 * R + 1);
    const int threads = ((kCand + 31) / 32) * 32;
    if (coarse) {
        coarse_kernel<R><<<grid, threads, 0, s>>>(a);
    } else {
        if constexpr (R <= kMaxRadius) {
            fine_kernel<R><<<grid, threads, 0, s>>>(a);
        } else {
            return cudaErrorInvalidValue;
        }
    }
    return cudaGetLastError();
}

// ---- search escalation (motion/escalate.rs, motion/kernels/escalate.rs) --------------------------
//
// With a ceiling above the first radius, blocks that fail their first window search again around
// the same centre at the ceiling. The state holds four sections of neighbours * conf_stride floats
// (kept SAD, edge bar then failure flag, winning window's centre x and y) and the SAD floor after
// them. Every stage reads only what the launch before it wrote, so the result does not depend on the
// order blocks run in.

constexpr float kEscalateBelowConfidence = 0.5f;  // escalate.rs:14-17
constexpr int kNeighbourDisagreement = 4;         // escalate.rs:19-23
constexpr float kEscalateSadMargin = 0.125f;      // escalate.rs:25-31
constexpr unsigned kFloorSamples = 4096, kFloorThreads = 256, kFloorRankDivisor = 4;
constexpr unsigned kFloorBinShift = 16, kInfinityBin = 0x7F80;
constexpr float kExactMatchSad = 1.0e-6f, kFlatShare = 0.25f;
enum { kStateSad = 0, kStateFlag = 1, kStateCentreX = 2, kStateCentreY = 3, kStateSections = 4 };

struct EscalateArgs {
    SearchLevel L;   // level 0
    SearchLevel Lc;  // the coarse level, when `widen`
    const uint32_t* neighbour_slots;
    uint32_t slots[kMaxNeighbours];
    int centre_slot, neighbours, use_seed, widen, scale;
    int32_t* mv_field;
    int mv_stride;
    float* confidence;
    int conf_stride;
    const float* noise;
    int sad_floor_word, reads_floor;
    float thsad;
    float* state;
    const float* predictions;  // the coarse search's camera-model window, or null
    float floor_scale;         // the SAD floor from a fine block to a coarse one
    float* sad_out;            // winning SADs (conf layout), replaced when a block improves; or null
};

__device__ __forceinline__ uint32_t escalate_slot(const EscalateArgs& e, int n, int bx, int by) {
    return static_cast<uint32_t>(n) * e.conf_stride + by * e.L.blocks_x + bx;
}

__device__ __forceinline__ int64_t escalate_section(const EscalateArgs& e) {
    return static_cast<int64_t>(e.neighbours) * e.conf_stride;
}

__device__ unsigned count_keys(const unsigned* keys, unsigned lo, unsigned hi, unsigned* counter) {
    if (threadIdx.x == 0) *counter = 0;
    __syncthreads();
    unsigned c = 0;
    for (unsigned i = threadIdx.x; i < kFloorSamples; i += blockDim.x) {
        const unsigned k = keys[i];
        c += (k >= lo && k <= hi) ? 1u : 0u;
    }
    atomicAdd(counter, c);
    __syncthreads();
    const unsigned total = *counter;
    __syncthreads();
    return total;
}

// escalate.rs:259-297 (`ranked_bin`): the lowest bin at or above `lower` that one in `divisor` of
// the keys from `lower` up fall at or below. Uniform across the CTA; at most 15 halvings.
__device__ unsigned ranked_bin(const unsigned* keys, unsigned lower, unsigned divisor, unsigned* counter) {
    const unsigned valid = count_keys(keys, lower, 0xFFFFFFFFu, counter);
    unsigned low = lower, high = kInfinityBin;
    while (low < high) {
        const unsigned middle = low + (high - low) / 2;
        if (divisor * count_keys(keys, lower, middle, counter) >= valid)
            high = middle;
        else
            low = middle + 1;
    }
    return low;
}

// escalate.rs:168-257 (`mc_measure_floor`): one CTA.
__global__ void __launch_bounds__(kFloorThreads) floor_kernel(EscalateArgs e) {
    __shared__ unsigned keys[kFloorSamples];
    __shared__ unsigned counter;
    const int64_t sec = escalate_section(e);
    float* floor_word = e.state + kStateSections * sec;
    if (e.reads_floor) {
        const float reading = e.noise[e.sad_floor_word];
        if (reading > 0.0f) {
            if (threadIdx.x == 0) *floor_word = reading;
            return;  // uniform: every thread read the same word
        }
    }
    const unsigned blocks = static_cast<unsigned>(e.L.blocks_x * e.L.blocks_y);
    const unsigned total = static_cast<unsigned>(e.neighbours) * blocks;
    const unsigned sample_step = (total + kFloorSamples - 1) / kFloorSamples;
    const unsigned sample_count = (total + sample_step - 1) / sample_step;
    for (unsigned s = threadIdx.x; s < kFloorSamples; s += blockDim.x) {
        const unsigned flat = min(s, sample_count - 1) * sample_step;
        const unsigned n = flat / blocks, b = flat % blocks;
        const float kept = e.state[kStateSad * sec + static_cast<int64_t>(n) * e.conf_stride + b];
        const bool counted = s < sample_count && kept > kExactMatchSad;
        keys[s] = counted ? (__float_as_uint(kept) >> kFloorBinShift) : 0u;
    }
    __syncthreads();
    const unsigned valid = count_keys(keys, 1u, 0xFFFFFFFFu, &counter);
    const unsigned median_bin = ranked_bin(keys, 1u, 2u, &counter);
    const float median = __uint_as_float(median_bin << kFloorBinShift);
    const float flat_limit = __fmul_rn(median, kFlatShare);
    const unsigned grainy = max(__float_as_uint(flat_limit) >> kFloorBinShift, 1u);
    const unsigned floor_bin = ranked_bin(keys, grainy, kFloorRankDivisor, &counter);
    if (threadIdx.x == 0) *floor_word = valid == 0 ? 0.0f : __uint_as_float(floor_bin << kFloorBinShift);
}

// escalate.rs:321-395 (`mc_flag_failures`): low confidence, an edge winner that beats its bar by
// more than the margin, or a vector more than 4 pixels from every grid neighbour's.
__global__ void __launch_bounds__(64) flag_kernel(EscalateArgs e) {
    const int bx = blockIdx.x * blockDim.x + threadIdx.x, by = blockIdx.y, n = blockIdx.z;
    if (bx >= e.L.blocks_x) return;
    const int64_t sec = escalate_section(e);
    const uint32_t slot = escalate_slot(e, n, bx, by);
    const float floor = e.state[kStateSections * sec];
    const float kept = e.state[kStateSad * sec + slot];
    const bool low = match_confidence(kept, floor, e.thsad) < kEscalateBelowConfidence;
    const float margin = __fmul_rn(kEscalateSadMargin, floor);
    const bool on_edge = __fadd_rn(kept, margin) < e.state[kStateFlag * sec + slot];
    const int32_t* f = e.mv_field + static_cast<int64_t>(n) * e.mv_stride;
    const int bxn = e.L.blocks_x, byn = e.L.blocks_y;
    const int own = (by * bxn + bx) * 2;
    int closest = INT_MAX;
    auto gap = [&](int o) { closest = min(closest, max(abs(f[o] - f[own]), abs(f[o + 1] - f[own + 1]))); };
    if (bx > 0) gap(own - 2);
    if (bx + 1 < bxn) gap(own + 2);
    if (by > 0) gap(own - 2 * bxn);
    if (by + 1 < byn) gap(own + 2 * bxn);
    if (closest == INT_MAX) closest = 0;
    e.state[kStateFlag * sec + slot] = (low || on_edge || closest > kNeighbourDisagreement) ? 1.0f : 0.0f;
}

// escalate.rs:400-640 (`mc_escalate_search`, `coarse_search`).
template <int C>
__global__ void __launch_bounds__(((2 * C + 1) * (2 * C + 1) + 31) / 32 * 32) escalate_kernel(EscalateArgs e) {
    __shared__ WindowScratch<C> w;
    __shared__ int coarse_vec[2];
    const int bx = blockIdx.x, by = blockIdx.y, n = blockIdx.z;
    const int64_t sec = escalate_section(e);
    const uint32_t slot = escalate_slot(e, n, bx, by);
    if (e.state[kStateFlag * sec + slot] == 0.0f) return;  // uniform across the CTA
    const int cdx = static_cast<int>(e.state[kStateCentreX * sec + slot]);
    const int cdy = static_cast<int>(e.state[kStateCentreY * sec + slot]);
    const float sad_floor = e.state[kStateSections * sec];
    const float margin = __fmul_rn(kEscalateSadMargin, sad_floor);
    const uint32_t nslot = e.neighbour_slots ? e.neighbour_slots[n] : e.slots[n];
    int kx = 0, ky = 0;
    if (e.widen) {
        // The coarse level again at the ceiling around no motion and, with the camera model, its
        // prediction, which wins by more than 1/8 of the floor scaled to the coarse block.
        const int64_t cb = e.Lc.level_base + static_cast<int64_t>(e.centre_slot) * e.Lc.slot_pixels;
        const int64_t nb = e.Lc.level_base + static_cast<int64_t>(nslot) * e.Lc.slot_pixels;
        const int ox = bx * e.L.step / e.scale, oy = by * e.L.step / e.scale;
        WinBest cbest = window_best<C>(e.Lc, cb, nb, ox, oy, 0, 0, w, false, false);
        int mdx, mdy;
        if (model_window(e.predictions, n, ox, oy, e.Lc.blksize, e.scale, e.Lc.width, e.Lc.height, C, 0, 0, &mdx, &mdy)) {
            const WinBest ch = window_best<C>(e.Lc, cb, nb, ox, oy, mdx, mdy, w, false, false);
            const float bias = __fmul_rn(__fmul_rn(kModelCandidateBias, sad_floor), e.floor_scale);
            if (threadIdx.x == 0 && __fadd_rn(ch.sad, bias) < cbest.sad) cbest = ch;
        }
        if (threadIdx.x == 0) {
            coarse_vec[0] = cbest.dx * e.scale;
            coarse_vec[1] = cbest.dy * e.scale;
        }
        __syncthreads();
        kx = coarse_vec[0];
        ky = coarse_vec[1];
    }
    const int64_t cb = static_cast<int64_t>(e.centre_slot) * e.L.slot_pixels;
    const int64_t nb = static_cast<int64_t>(nslot) * e.L.slot_pixels;
    WinBest best = window_best<C>(e.L, cb, nb, bx * e.L.step, by * e.L.step, cdx, cdy, w, false, false);
    if (e.widen && (kx != cdx || ky != cdy)) {  // uniform: every thread holds the same vectors
        const WinBest ch = window_best<C>(e.L, cb, nb, bx * e.L.step, by * e.L.step, kx, ky, w, false, false);
        if (threadIdx.x == 0 && __fadd_rn(ch.sad, margin) < best.sad) best = ch;
    }
    if (threadIdx.x != 0) return;
    if (__fadd_rn(best.sad, margin) < e.state[kStateSad * sec + slot]) {
        int32_t* mv = e.mv_field + static_cast<int64_t>(n) * e.mv_stride + (by * e.L.blocks_x + bx) * 2;
        mv[0] = best.dx;
        mv[1] = best.dy;
        e.state[kStateSad * sec + slot] = best.sad;
        if (e.sad_out) e.sad_out[slot] = best.sad;
        if (e.confidence) e.confidence[slot] = match_confidence(best.sad, e.noise[e.sad_floor_word], e.thsad);
    }
}

template <int R>
cudaError_t launch_escalate(int radius, const EscalateArgs& e, dim3 grid, cudaStream_t s) {
    if (radius == R) {
        constexpr int kCand = (2 * R + 1) * (2 * R + 1);
        escalate_kernel<R><<<grid, ((kCand + 31) / 32) * 32, 0, s>>>(e);
        return cudaGetLastError();
    }
    if constexpr (R < kMaxRadius) {
        return launch_escalate<R + 1>(radius, e, grid, s);
    } else {
        return cudaErrorInvalidValue;
    }
}

cudaError_t dispatch_search(int radius, bool coarse, const SearchArgs& a, dim3 grid, cudaStream_t s) {
    switch (radius) {
        case 0: return launch_search<0>(coarse, a, grid, s);
        case 1: return launch_search<1>(coarse, a, grid, s);
        case 2: return launch_search<2>(coarse, a, grid, s);
        case 3: return launch_search<3>(coarse, a, grid, s);
        case 4: return launch_search<4>(coarse, a, grid, s);
        case 5: return launch_search<5>(coarse, a, grid, s);
        case 6: return launch_search<6>(coarse, a, grid, s);
        case 7: return launch_search<7>(coarse, a, grid, s);
        case 8: return launch_search<8>(coarse, a, grid, s);
        case kAcquisitionRadius: return coarse ? launch_search<kAcquisitionRadius>(true, a, grid, s) : cudaErrorInvalidValue;
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

int64_t pyramid_slot_pixels(int width, int height, int level) {
    int w = width, h = height;
    for (int l = 0; l < level; ++l) {
        w = w / 2 > 1 ? w / 2 : 1;
        h = h / 2 > 1 ? h / 2 : 1;
    }
    return (static_cast<int64_t>(w) * h + 7) / 8 * 8;
}

void pyramid_level_dims(int width, int height, int level, int* w, int* h) {
    *w = width;
    *h = height;
    for (int l = 0; l < level; ++l) {
        *w = *w / 2 > 1 ? *w / 2 : 1;
        *h = *h / 2 > 1 ? *h / 2 : 1;
    }
}

int64_t pyramid_level_base(int width, int height, int frame_count, int level) {
    int64_t base = 0;
    for (int l = 0; l < level; ++l) base += static_cast<int64_t>(frame_count) * pyramid_slot_pixels(width, height, l);
    return base;
}

int64_t pyramid_floats(int width, int height, int frame_count, int levels) {
    return pyramid_level_base(width, height, frame_count, levels);
}

cudaError_t launch_pyramid_build(const float* ring, int channels, int width, int height, int frame_count,
                                 int ring_slot, int levels, float* pyramid, int pyramid_slot, cudaStream_t s) {
    const int64_t pixels = static_cast<int64_t>(width) * height;
    float* dst0 = pyramid + static_cast<int64_t>(pyramid_slot) * pyramid_slot_pixels(width, height, 0);
    const int64_t src_elems = static_cast<int64_t>(ring_slot) * pixels * channels;
    pyramid_level0_kernel<<<static_cast<unsigned>((pixels + 255) / 256), 256, 0, s>>>(ring, dst0, pixels, channels,
                                                                                      src_elems);
    for (int l = 1; l < levels; ++l) {
        int sw, sh, dw, dh;
        pyramid_level_dims(width, height, l - 1, &sw, &sh);
        pyramid_level_dims(width, height, l, &dw, &dh);
        const float* src = pyramid + pyramid_level_base(width, height, frame_count, l - 1) +
                           static_cast<int64_t>(pyramid_slot) * pyramid_slot_pixels(width, height, l - 1);
        float* dst = pyramid + pyramid_level_base(width, height, frame_count, l) +
                     static_cast<int64_t>(pyramid_slot) * pyramid_slot_pixels(width, height, l);
        dim3 block(16, 16), grid((dw + 15) / 16, (dh + 15) / 16);
        pyramid_down_kernel<<<grid, block, 0, s>>>(src, dst, sw, sh, dw, dh);
    }
    return cudaGetLastError();
}

cudaError_t launch_motion_search(const MotionLaunch& m, cudaStream_t s) {
    if (!m.neighbour_slots && m.neighbours > kMaxNeighbours) return cudaErrorInvalidValue;
    if (m.predictions && !m.noise) return cudaErrorInvalidValue;
    const int step = m.blksize - m.overlap;
    const int blocks_x = (m.width + step - 1) / step > 1 ? (m.width + step - 1) / step : 1;
    const int blocks_y = (m.height + step - 1) / step > 1 ? (m.height + step - 1) / step : 1;
    const bool coarse = m.levels > 1 && !m.seeded;
    const bool seeded = coarse || m.seeded;
    const int factor = m.coarse_block_factor > 0 ? m.coarse_block_factor : 1;
    // analyse.rs:118-157 (`coarse_level`): the smallest level, its blocks `factor` times the content
    // a fine block covers there, and the SAD floor's scale from a fine block to a coarse one.
    SearchLevel Lc{};
    int scale = 1;
    float floor_scale = 1.0f;
    if (m.levels > 1) {
        const int level = m.levels - 1;
        scale = 1 << level;
        pyramid_level_dims(m.width, m.height, level, &Lc.width, &Lc.height);
        Lc.pyramid = m.pyramid;
        Lc.level_base = pyramid_level_base(m.width, m.height, m.frame_count, level);
        Lc.slot_pixels = pyramid_slot_pixels(m.width, m.height, level);
        Lc.blksize = (m.blksize / scale > 2 ? m.blksize / scale : 2) * factor;
        Lc.step = step / scale > 1 ? step / scale : 1;
        Lc.blocks_x = (Lc.width + Lc.step - 1) / Lc.step > 1 ? (Lc.width + Lc.step - 1) / Lc.step : 1;
        Lc.blocks_y = (Lc.height + Lc.step - 1) / Lc.step > 1 ? (Lc.height + Lc.step - 1) / Lc.step : 1;
        if (Lc.blksize > kMaxBlk) return cudaErrorInvalidValue;
        const float coarse_area = static_cast<float>(Lc.blksize * Lc.blksize);
        const float fine_area = static_cast<float>(m.blksize * m.blksize);
        floor_scale = coarse_area / fine_area / static_cast<float>(scale);
    }
    if (coarse) {
        SearchArgs a{};
        a.L = Lc;
        a.neighbour_slots = m.neighbour_slots;
        for (int i = 0; i < kMaxNeighbours; ++i) a.slots[i] = m.inline_slots[i];
        a.centre_slot = m.centre_slot;
        a.mv_field = m.mv_field;
        a.mv_stride = m.mv_stride;
        a.level_scale = scale;
        a.fine_blocks_x = blocks_x;
        a.fine_blocks_y = blocks_y;
        a.fine_step = step;
        a.noise = m.noise;
        a.sad_floor_word = m.sad_floor_word;
        a.predictions = m.predictions;
        a.floor_scale = floor_scale;
        dim3 grid(Lc.blocks_x, Lc.blocks_y, m.neighbours);
        if (cudaError_t e = dispatch_search(m.coarse_radius, true, a, grid, s)) return e;
        // analyse.rs:268-277 (`keep_seeds`): the coarse field, before the fine pass overwrites it.
        if (m.keep_seeds)
            if (cudaError_t e = cudaMemcpyAsync(m.keep_seeds, m.mv_field,
                                                static_cast<size_t>(m.neighbours) * m.mv_stride * sizeof(int32_t),
                                                cudaMemcpyDeviceToDevice, s))
                return e;
    }
    SearchArgs a{};
    a.L.pyramid = m.pyramid;
    a.L.width = m.width;
    a.L.height = m.height;
    a.L.level_base = 0;
    a.L.slot_pixels = pyramid_slot_pixels(m.width, m.height, 0);
    a.L.blksize = m.blksize;
    a.L.step = step;
    a.L.blocks_x = blocks_x;
    a.L.blocks_y = blocks_y;
    a.neighbour_slots = m.neighbour_slots;
    for (int i = 0; i < kMaxNeighbours; ++i) a.slots[i] = m.inline_slots[i];
    a.centre_slot = m.centre_slot;
    a.mv_field = m.mv_field;
    a.mv_stride = m.mv_stride;
    a.use_seed = seeded ? 1 : 0;
    a.confidence = m.confidence;
    a.conf_stride = m.conf_stride;
    a.noise = m.noise;
    a.sad_floor_word = m.sad_floor_word;
    a.thsad = m.thsad;
    a.predictions = m.predictions;
    a.floor_scale = 1.0f;
    a.sad_out = m.sad;
    a.sad_means = static_cast<int64_t>(m.neighbours) * m.conf_stride;
    if (a.L.blksize > kMaxBlk) return cudaErrorInvalidValue;
    dim3 grid(blocks_x, blocks_y, m.neighbours);
    const bool escalates = m.escalation && m.ceiling > m.search_radius;
    if (!escalates) return dispatch_search(m.search_radius, false, a, grid, s);
    if (m.ceiling > kMaxRadius || m.thsad <= 0.0f || !m.noise) return cudaErrorInvalidValue;
    // analyse.rs:234-262 and escalate.rs:19-57: the first pass records each block's kept SAD, edge
    // bar and winning window's centre; then the floor, the failure flags, and the failures searched
    // again at the ceiling (the coarse level too, when a coarse pass seeded the search and the
    // ceiling reaches past its radius, escalate.rs:203-205).
    EscalateArgs e{};
    e.L = a.L;
    e.neighbour_slots = m.neighbour_slots;
    for (int i = 0; i < kMaxNeighbours; ++i) e.slots[i] = m.inline_slots[i];
    e.centre_slot = m.centre_slot;
    e.neighbours = m.neighbours;
    e.use_seed = seeded ? 1 : 0;
    e.widen = coarse && m.ceiling > m.coarse_radius ? 1 : 0;
    e.scale = scale;
    e.Lc = Lc;
    e.mv_field = m.mv_field;
    e.mv_stride = m.mv_stride;
    e.confidence = m.confidence;
    e.conf_stride = m.conf_stride;
    e.noise = m.noise;
    e.sad_floor_word = m.sad_floor_word;
    e.reads_floor = m.esc_reads_floor;
    e.thsad = m.thsad;
    e.state = m.escalation;
    e.predictions = m.predictions;
    e.floor_scale = floor_scale;
    e.sad_out = m.sad;
    a.esc_state = e.state;
    a.esc_section = static_cast<int64_t>(m.neighbours) * m.conf_stride;
    if (cudaError_t err = dispatch_search(m.search_radius, false, a, grid, s)) return err;
    floor_kernel<<<1, kFloorThreads, 0, s>>>(e);
    flag_kernel<<<dim3((blocks_x + 63) / 64, blocks_y, m.neighbours), 64, 0, s>>>(e);
    return launch_escalate<0>(m.ceiling, e, grid, s);
}

size_t escalation_state_floats(int neighbours, int conf_stride) {
    return static_cast<size_t>(kStateSections) * neighbours * conf_stride + 1;
}

namespace {
// motion/kernels/compensate.rs:6-44 (`mc_warp`): pixel (x, y) of neighbour n takes the vector of
// block (min(x / step, bx - 1), min(y / step, by - 1)) and copies the source pixel at the clamped
// (x + dx, y + dy), every channel; the reference ring follows the same vectors when given.
__global__ void __launch_bounds__(256) warp_kernel(WarpLaunch w) {
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    if (x >= w.width || y >= w.height) return;
    const int n = blockIdx.z;
    const int64_t slot = w.slots[n];
    const int bc = min(x / w.step, w.blocks_x - 1), br = min(y / w.step, w.blocks_y - 1);
    const int32_t* mv = w.mv_field + static_cast<int64_t>(n) * w.mv_stride + 2 * (br * w.blocks_x + bc);
    const int sx = clamp_to(x + mv[0], w.width), sy = clamp_to(y + mv[1], w.height);
    const int64_t src = slot * w.frame_elems + (static_cast<int64_t>(sy) * w.width + sx) * w.channels;
    const int64_t dst = slot * w.frame_elems + (static_cast<int64_t>(y) * w.width + x) * w.channels;
    for (int c = 0; c < w.channels; ++c) w.dst_ring[dst + c] = __ldg(w.src_ring + src + c);
    if (w.src_ref)
        for (int c = 0; c < w.channels; ++c) w.dst_ref[dst + c] = __ldg(w.src_ref + src + c);
}

__global__ void chain_compose_kernel(const int32_t* __restrict__ pair_ring, int32_t* __restrict__ mv_field,
                                     int mv_stride, int centre, int d, int head_mod, int dir_stride,
                                     int slot_stride, int step, int width, int height, int blocks_x, int blocks_y) {
    const int bx = blockIdx.x * blockDim.x + threadIdx.x, by = blockIdx.y, n = blockIdx.z;
    if (bx >= blocks_x || by >= blocks_y) return;
    const int logical = n < centre ? n : n + 1;
    const int k = logical - centre;
    const bool forward = k > 0;
    const int steps = forward ? k : -k;
    const int slots = 2 * d;
    const int start_gap = forward ? centre : centre - 1;
    const int start = ((head_mod + start_gap) % slots + slots) % slots;
    int pos_x = bx * step + step / 2, pos_y = by * step + step / 2;
    int acc_x = 0, acc_y = 0;
    for (int i = 0; i < steps; ++i) {
        const int slot = forward ? (start + i) % slots : (start + slots - i) % slots;
        const int cx = clamp_to(pos_x, width), cy = clamp_to(pos_y, height);
        const int hc = min(cx / step, blocks_x - 1), hr = min(cy / step, blocks_y - 1);
        const int base = slot * slot_stride + (forward ? 0 : dir_stride) + (hr * blocks_x + hc) * 2;
        const int hop_x = pair_ring[base], hop_y = pair_ring[base + 1];
        acc_x += hop_x;
        acc_y += hop_y;
        pos_x += hop_x;
        pos_y += hop_y;
    }
    int32_t* out = mv_field + static_cast<int64_t>(n) * mv_stride + (by * blocks_x + bx) * 2;
    out[0] = acc_x;
    out[1] = acc_y;
}
}  // namespace

cudaError_t launch_chain_compose(const int32_t* pair_ring, int32_t* mv_field, int mv_stride, int centre, int d,
                                 int head_mod, int dir_stride, int slot_stride, int step, int width, int height,
                                 int blocks_x, int blocks_y, cudaStream_t s) {
    if (d < 1) return cudaErrorInvalidValue;
    dim3 grid((blocks_x + 63) / 64, blocks_y, 2 * d);
    chain_compose_kernel<<<grid, 64, 0, s>>>(pair_ring, mv_field, mv_stride, centre, d, head_mod, dir_stride,
                                             slot_stride, step, width, height, blocks_x, blocks_y);
    return cudaGetLastError();
}

cudaError_t launch_warp(const WarpLaunch& w, cudaStream_t s) {
    if (!w.src_ring || !w.dst_ring || !w.mv_field || (w.src_ref && !w.dst_ref) || w.neighbours < 1 ||
        w.neighbours > WarpLaunch::kMaxSlots || w.channels < 1 || w.channels > 2 || w.step < 1 || w.blocks_x < 1 ||
        w.blocks_y < 1)
        return cudaErrorInvalidValue;
    dim3 grid((w.width + 31) / 32, (w.height + 7) / 8, w.neighbours);
    warp_kernel<<<grid, dim3(32, 8), 0, s>>>(w);
    return cudaGetLastError();
}

namespace {

// chroma_map.rs:6-18 (`scale_down`): divided by 2^shift, rounding half away from zero.
__device__ __forceinline__ int scale_down(int v, int shift) {
    if (shift == 0) return v;
    const int factor = 1 << shift, half = 1 << (shift - 1);
    const int rounded = (abs(v) + half) / factor;
    return v < 0 ? -rounded : rounded;
}

__global__ void __launch_bounds__(64) map_luma_fields_kernel(MapLaunch m, int covers_x, int covers_y) {
    const int col = blockIdx.x * 8 + threadIdx.x;
    const int row = blockIdx.y * 8 + threadIdx.y;
    if (col >= m.chroma_bx || row >= m.chroma_by) return;
    const int field = blockIdx.z;
    const int origin_x = (col * m.chroma_step) << m.shift_x;
    const int origin_y = (row * m.chroma_step) << m.shift_y;
    const int start_col = origin_x / m.luma_step, start_row = origin_y / m.luma_step;
    const int last_col = min(start_col + covers_x - 1, m.luma_bx - 1);
    const int last_row = min(start_row + covers_y - 1, m.luma_by - 1);
    const int first_col = min(start_col, last_col), first_row = min(start_row, last_row);
    const int32_t* luma = m.luma + static_cast<int64_t>(field) * m.luma_stride;
    const int n = covers_x * covers_y;
    // chroma_map.rs:20-46 (`lower_median`): the live entry whose rank among the live entries holds
    // the lower median, per component; entries past the grid repeat the last block but do not count.
    auto value = [&](int i, int comp) {
        const int c = first_col + i % covers_x, r = first_row + i / covers_x;
        return luma[2 * (min(r, last_row) * m.luma_bx + min(c, last_col)) + comp];
    };
    auto live = [&](int i) { return first_col + i % covers_x <= last_col && first_row + i / covers_x <= last_row; };
    int count = 0;
    for (int i = 0; i < n; ++i) count += live(i) ? 1 : 0;
    const int middle = (count - 1) / 2;
    int out[2];
    for (int comp = 0; comp < 2; ++comp) {
        int median = value(0, comp);
        for (int i = 0; i < n; ++i) {
            const int vi = value(i, comp);
            int below = 0, equal = 0;
            for (int j = 0; j < n; ++j) {
                if (!live(j)) continue;
                const int vj = value(j, comp);
                below += vj < vi ? 1 : 0;
                equal += vj == vi ? 1 : 0;
            }
            if (live(i) && below <= middle && middle < below + equal) median = vi;
        }
        out[comp] = median;
    }
    int32_t* dst = m.chroma + static_cast<int64_t>(field) * m.chroma_stride + 2 * (row * m.chroma_bx + col);
    dst[0] = scale_down(out[0], m.shift_x);
    dst[1] = scale_down(out[1], m.shift_y);
}

}  // namespace

cudaError_t launch_map_luma_fields(const MapLaunch& m, cudaStream_t s) {
    if (!m.luma || !m.chroma || m.fields < 1 || m.luma_step < 1 || m.chroma_step < 1 || m.shift_x < 0 ||
        m.shift_x > 1 || m.shift_y < 0 || m.shift_y > 1)
        return cudaErrorInvalidValue;
    // chroma_map.rs:65-68: the luma blocks along each axis of the area a chroma block covers.
    const int area_x = m.chroma_blksize << m.shift_x, area_y = m.chroma_blksize << m.shift_y;
    const int covers_x = std::max(area_x - m.luma_blksize, 0) / m.luma_step + 1;
    const int covers_y = std::max(area_y - m.luma_blksize, 0) / m.luma_step + 1;
    dim3 grid((m.chroma_bx + 7) / 8, (m.chroma_by + 7) / 8, m.fields);
    map_luma_fields_kernel<<<grid, dim3(8, 8), 0, s>>>(m, covers_x, covers_y);
    return cudaGetLastError();
}

}  // namespace avd
