// NL4D collaborative filter for sm_100a: group search, 2D DCT + Haar hard/pooled threshold,
// inverse transforms and fixed-point aggregation, one launch per pass.
//
// What it computes (av-denoise-core/src/collab/kernels/fused/mod.rs:170-891): for every reference
// patch (8x8 on a step-4 grid of the centre frame) the best 8 positions of the centre frame's
// spatial window (self match pinned first, ties keep the earlier position), optionally grown into
// volumes along the neighbour frames' motion (fused/trajectory.rs), a 2D DCT per member, a Haar
// along the stack (or time and volumes), a hard or pooled threshold against lambda x the
// propagated noise, the inverse transforms, and a Kaiser-tapered fixed-point scatter of every
// member into its own frame's accumulator region, weighted by 1 / (retained variance).
//
// How (B200): one 8-lane group per reference patch, lane `sub` owning column `sub` of every patch
// the group touches, so every candidate read and every scatter is an 8-wide coalesced access.
// Cross-lane sums use the xor-1/2/4 shuffle butterfly and the 8x8 transposes a per-group shared
// region, both scoped to the group's own 8 lanes (`__shfl_*_sync` with the group's mask and
// `__syncwarp(mask)`), so groups of one warp may take different trip counts through their
// clipped windows: no block barrier is ever needed. The group's 8 members x 8 values stay in
// registers through the transforms. Accumulation is integer atomics, so the output does not
// depend on scheduling. Every multiply and add is rounded on its own (no fused multiply-add),
// in the restatement's order, so the floats, and with them every threshold decision and member
// choice, agree bit for bit with the CPU oracle.

#include <cuda_runtime.h>

#include <cstdint>

#include "colour_lookup.cuh"
#include "kernels.h"

namespace avd {

namespace {

constexpr int P = 8;
constexpr int STEP = 4;
constexpr int MAX_K = 8;
constexpr int kGroups = 16;  // reference patches per CTA
constexpr int kThreads = kGroups * 8;
constexpr float kUnfilled = 3.0e38f;
constexpr float kSelfPin = -1.0e38f;
constexpr float kReciprocalFloor = 1e-12f;
constexpr float kAccumClamp = 5.0f;
constexpr float kWeightGain = 5.0f;
constexpr float kVarianceFloor = 1.0e-20f;
constexpr float kFrac1Sqrt2 = 0.70710678118654752440f;
constexpr int kCurveBins = 16;

// The orthonormal 8-point DCT-II taps, c_row * cos(pi * (2 col + 1) row / 16), in f32.
__constant__ float c_dct[8][8];

struct GroupCtx {
    unsigned mask;  // this group's 8 lanes of the warp
    int sub;        // lane within the group
};

__device__ __forceinline__ float reduce8(const GroupCtx& g, float v) {
    v += __shfl_xor_sync(g.mask, v, 1);
    v += __shfl_xor_sync(g.mask, v, 2);
    v += __shfl_xor_sync(g.mask, v, 4);
    return v;
}

__device__ __forceinline__ uint32_t pack_pos_t(uint32_t x, uint32_t y, uint32_t t) {
    return (t << 26) | (y << 13) | x;
}

__device__ __forceinline__ uint32_t clamp_top_left(int v, uint32_t max_pos) {
    return v < 0 ? 0u : (v > static_cast<int>(max_pos) ? max_pos : static_cast<uint32_t>(v));
}

// The lane's share of the distance from `ref` (its 8 x C column) to the candidate at (x, y).
template <int C>
__device__ __forceinline__ float column_ssd(const float (&ref)[P * C], const float* __restrict__ frame, int width,
                                            uint32_t x, uint32_t y, int sub) {
    float s = 0.0f;
    const float* p = frame + (static_cast<size_t>(y) * width + x + sub) * C;
#pragma unroll
    for (int r = 0; r < P; ++r) {
#pragma unroll
        for (int c = 0; c < C; ++c) {
            float d = ref[r * C + c] - __ldg(p + static_cast<size_t>(r) * width * C + c);
            s = __fadd_rn(s, __fmul_rn(d, d));
        }
    }
    return s;
}

__device__ __forceinline__ void dct8_fwd(float (&line)[P]) {
    float s[4], d[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        s[k] = line[k] + line[7 - k];
        d[k] = line[k] - line[7 - k];
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        float even = 0.0f, odd = 0.0f;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            even = __fadd_rn(even, __fmul_rn(s[k], c_dct[2 * m][k]));
            odd = __fadd_rn(odd, __fmul_rn(d[k], c_dct[2 * m + 1][k]));
        }
        line[2 * m] = even;
        line[2 * m + 1] = odd;
    }
}

__device__ __forceinline__ void dct8_inv(float (&line)[P]) {
    float snap[P];
#pragma unroll
    for (int j = 0; j < P; ++j) snap[j] = line[j];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        float even = 0.0f, odd = 0.0f;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            even = __fadd_rn(even, __fmul_rn(snap[2 * m], c_dct[2 * m][k]));
            odd = __fadd_rn(odd, __fmul_rn(snap[2 * m + 1], c_dct[2 * m + 1][k]));
        }
        line[k] = even + odd;
        line[7 - k] = even - odd;
    }
}

// An 8x8 transpose across the group's lanes through its own shared region of kRegion floats; the
// index skew of one float every 32 keeps the column reads off a shared bank.
constexpr int kRegion = 72;
__device__ __forceinline__ void transpose8(const GroupCtx& g, float* region, float (&v)[P]) {
#pragma unroll
    for (int i = 0; i < P; ++i) region[i * 8 + g.sub + (i * 8 + g.sub) / 32] = v[i];
    __syncwarp(g.mask);
#pragma unroll
    for (int i = 0; i < P; ++i) v[i] = region[g.sub * 8 + i + (g.sub * 8 + i) / 32];
    __syncwarp(g.mask);
}


// fused/pooled.rs: keep a coefficient on the mean energy of itself and its four frequency
// neighbours; lane `sub` holds vertical frequency `sub`, slot i horizontal frequency i. Returns
// the lane's retained variance.
__device__ __forceinline__ float pooled_threshold(const GroupCtx& g, float (&s)[MAX_K][P], const float (&v)[MAX_K],
                                                  const float (&prof)[P], int k_use, float threshold,
                                                  float dc_lambda, bool wiener, uint64_t& bits) {
    const int sub = g.sub;
    const bool dc_lane = sub == 0, has_up = sub > 0, has_down = sub < 7;
    const float vertical = 1.0f + (has_up ? 1.0f : 0.0f) + (has_down ? 1.0f : 0.0f);
    const float bar = threshold * threshold;
    const float first_col = bar * (vertical + (sub == 1 ? 0.0f : 1.0f));
    const float second_col = bar * (vertical + (dc_lane ? 1.0f : 2.0f));
    const float middle_col = bar * (vertical + 2.0f);
    const float last_col = bar * (vertical + 1.0f);
    const float prof_sub = prof[sub];
    float retained = 0.0f;
#pragma unroll
    for (int j = 0; j < MAX_K; ++j) {
        const float lane_var = v[j] * prof_sub;
        const float lane_inv = 1.0f / fmaxf(lane_var, kVarianceFloor);
        float e0 = s[j][0] * s[j][0] * lane_inv * (1.0f / fmaxf(prof[0], kVarianceFloor));
        float current = dc_lane ? 0.0f : e0;
        float previous = 0.0f;
        float kept_profile = 0.0f;
#pragma unroll
        for (int i = 0; i < P; ++i) {
            const float coeff = s[j][i];
            float next = 0.0f;
            if (i < 7) next = s[j][i + 1] * s[j][i + 1] * lane_inv * (1.0f / fmaxf(prof[i + 1], kVarianceFloor));
            const float shuffled_up = __shfl_up_sync(g.mask, current, 1, 8);
            const float shuffled_down = __shfl_down_sync(g.mask, current, 1, 8);
            float sum = current + (has_down ? shuffled_down : 0.0f) + (has_up ? shuffled_up : 0.0f);
            if (i > 0) sum += previous;
            if (i < 7) sum += next;
            const float col_bar = i == 0 ? first_col : (i == 1 ? second_col : (i == 7 ? last_col : middle_col));
            bool keep = sum >= col_bar;
            if (i == 0) {
                const bool own = fabsf(coeff) >= dc_lambda * sqrtf(lane_var * prof[0]);
                keep = dc_lane ? own : keep;
                if (j == 0) keep = keep || dc_lane;
            }
            const bool live = j < k_use;
            if (wiener && live && keep) {
                const float cv = lane_var * prof[i];
                const float zz = coeff * coeff;
                const float den = zz + cv;
                const float gain = den > 0.0f ? zz / den : 1.0f;
                kept_profile += (gain * gain) * prof[i];
                s[j][i] = gain * coeff;
            } else {
                kept_profile += keep ? prof[i] : 0.0f;
                if (live && !keep) s[j][i] = 0.0f;
            }
            if (keep && live) bits |= uint64_t{1} << (j * 8 + i);
            previous = current;
            current = next;
        }
        if (j < k_use) retained = __fadd_rn(retained, __fmul_rn(kept_profile, lane_var));
    }
    return retained;
}

// The Haar ladder over the stack of k_use members (transforms.rs:124-191) and its variance shadow.
__device__ __forceinline__ void haar_level(float (&s)[MAX_K][P], int len, bool inverse) {
    const int half = len / 2;
#pragma unroll
    for (int pos = 0; pos < P; ++pos) {
        float snap[MAX_K];
#pragma unroll
        for (int k = 0; k < MAX_K; ++k) snap[k] = s[k][pos];
#pragma unroll
        for (int p = 0; p < MAX_K / 2; ++p) {
            if (p >= half) break;
            if (!inverse) {
                s[p][pos] = (snap[2 * p] + snap[2 * p + 1]) * kFrac1Sqrt2;
                s[half + p][pos] = (snap[2 * p] - snap[2 * p + 1]) * kFrac1Sqrt2;
            } else {
                s[2 * p][pos] = (snap[p] + snap[half + p]) * kFrac1Sqrt2;
                s[2 * p + 1][pos] = (snap[p] - snap[half + p]) * kFrac1Sqrt2;
            }
        }
    }
}

__device__ __forceinline__ void variance_level(float (&v)[MAX_K], int len) {
    const int half = len / 2;
    float snap[MAX_K];
#pragma unroll
    for (int k = 0; k < MAX_K; ++k) snap[k] = v[k];
#pragma unroll
    for (int p = 0; p < MAX_K / 2; ++p) {
        if (p >= half) break;
        const float mean = (snap[2 * p] + snap[2 * p + 1]) * 0.5f;
        v[p] = mean;
        v[half + p] = mean;
    }
}

// fused/grid.rs: strided Haar levels (time inside a volume, then across volumes).
template <int START, int STRIDE, int LEN>
__device__ __forceinline__ void strided_level(float (&vals)[MAX_K], bool inverse, bool variance) {
    constexpr int half = LEN / 2;
    float snap[LEN];
#pragma unroll
    for (int k = 0; k < LEN; ++k) snap[k] = vals[START + k * STRIDE];
#pragma unroll
    for (int p = 0; p < half; ++p) {
        if (variance) {
            const float mean = (snap[2 * p] + snap[2 * p + 1]) * 0.5f;
            vals[START + p * STRIDE] = mean;
            vals[START + (half + p) * STRIDE] = mean;
        } else if (!inverse) {
            vals[START + p * STRIDE] = (snap[2 * p] + snap[2 * p + 1]) * kFrac1Sqrt2;
            vals[START + (half + p) * STRIDE] = (snap[2 * p] - snap[2 * p + 1]) * kFrac1Sqrt2;
        } else {
            vals[START + 2 * p * STRIDE] = (snap[p] + snap[half + p]) * kFrac1Sqrt2;
            vals[START + (2 * p + 1) * STRIDE] = (snap[p] - snap[half + p]) * kFrac1Sqrt2;
        }
    }
}

template <int START, int STRIDE, int LEN>
__device__ __forceinline__ void strided_fwd(float (&vals)[MAX_K], bool variance) {
    if constexpr (LEN >= 4) strided_level<START, STRIDE, 4>(vals, false, variance);
    if constexpr (LEN >= 2) strided_level<START, STRIDE, 2>(vals, false, variance);
}

template <int START, int STRIDE, int LEN>
__device__ __forceinline__ void strided_inv(float (&vals)[MAX_K]) {
    if constexpr (LEN >= 2) strided_level<START, STRIDE, 2>(vals, true, false);
    if constexpr (LEN >= 4) strided_level<START, STRIDE, 4>(vals, true, false);
}

template <int GF, int V = 0>
__device__ __forceinline__ void volumes_fwd(float (&vals)[MAX_K], bool variance) {
    if constexpr (V < MAX_K / GF) {
        strided_fwd<V * GF, 1, GF>(vals, variance);
        volumes_fwd<GF, V + 1>(vals, variance);
    }
}

template <int GF, int F = 0>
__device__ __forceinline__ void frames_fwd(float (&vals)[MAX_K], bool variance) {
    if constexpr (F < GF) {
        strided_fwd<F, GF, MAX_K / GF>(vals, variance);
        frames_fwd<GF, F + 1>(vals, variance);
    }
}

template <int GF, int V = 0>
__device__ __forceinline__ void volumes_inv(float (&vals)[MAX_K]) {
    if constexpr (V < MAX_K / GF) {
        strided_inv<V * GF, 1, GF>(vals);
        volumes_inv<GF, V + 1>(vals);
    }
}

template <int GF, int F = 0>
__device__ __forceinline__ void frames_inv(float (&vals)[MAX_K]) {
    if constexpr (F < GF) {
        strided_inv<F, GF, MAX_K / GF>(vals);
        frames_inv<GF, F + 1>(vals);
    }
}

template <int GF>
__device__ __forceinline__ void grid_fwd(float (&s)[MAX_K][P]) {
#pragma unroll
    for (int pos = 0; pos < P; ++pos) {
        float vals[MAX_K];
#pragma unroll
        for (int m = 0; m < MAX_K; ++m) vals[m] = s[m][pos];
        volumes_fwd<GF>(vals, false);
        frames_fwd<GF>(vals, false);
#pragma unroll
        for (int m = 0; m < MAX_K; ++m) s[m][pos] = vals[m];
    }
}

template <int GF>
__device__ __forceinline__ void grid_inv(float (&s)[MAX_K][P]) {
#pragma unroll
    for (int pos = 0; pos < P; ++pos) {
        float vals[MAX_K];
#pragma unroll
        for (int m = 0; m < MAX_K; ++m) vals[m] = s[m][pos];
        frames_inv<GF>(vals);
        volumes_inv<GF>(vals);
#pragma unroll
        for (int m = 0; m < MAX_K; ++m) s[m][pos] = vals[m];
    }
}

template <int GF>
__device__ __forceinline__ void grid_variance(float (&v)[MAX_K]) {
    volumes_fwd<GF>(v, true);
    frames_fwd<GF>(v, true);
}

// aggregate.rs:147-160.
__device__ __forceinline__ int32_t to_fixed(float value, float scale) {
    return static_cast<int32_t>(roundf(fminf(fmaxf(value, -kAccumClamp), kAccumClamp) * scale));
}

__device__ __forceinline__ int32_t to_fixed_weight(float weight, float scale) {
    return static_cast<int32_t>(roundf(fminf(fmaxf(weight, 0.0f), 1.0f) * scale * kWeightGain));
}

__device__ __forceinline__ uint32_t covering_lo(uint32_t patch_start, uint32_t blksize, uint32_t step) {
    const uint32_t overhang = max(patch_start + P, blksize) - blksize;
    return (overhang + step - 1) / step;
}

// fused/trajectory.rs (clipped walk): for each neighbour frame the best candidate over one refine
// rectangle per covering motion block (blocks under c_min skipped, rectangles already searched and
// positions the group holds skipped), inserted into the volume's sorted tail. COVERS (the covering
// blocks per axis, ceil(blksize / step)) is a template argument so the rectangles searched so far
// stay in registers. A skipped candidate can only matter if it would beat the frame's best so far,
// so the skip test runs for those alone; the winner is the same.
template <int C, int GF, int FIRST, int COVERS>
__device__ __forceinline__ void trajectory_search(const GroupCtx& g, const CollabLaunch& a, const float (&anchor)[P * C],
                                                  uint32_t ax, uint32_t ay, float scale, float (&grid_d)[MAX_K],
                                                  uint32_t (&grid_pos)[MAX_K]) {
    constexpr int TAIL = GF - 1;
    constexpr int RECTS = COVERS * COVERS;
    const uint32_t max_x = a.width - P, max_y = a.height - P;
    const uint32_t bx_hi = min(ax / a.blk_step, static_cast<uint32_t>(a.blocks_x - 1));
    const uint32_t by_hi = min(ay / a.blk_step, static_cast<uint32_t>(a.blocks_y - 1));
    const uint32_t bx_lo = min(covering_lo(ax, a.blksize, a.blk_step), bx_hi);
    const uint32_t by_lo = min(covering_lo(ay, a.blksize, a.blk_step), by_hi);
    for (int t = 0; t < 2 * a.radius; ++t) {
        const int slot = static_cast<int>(a.neighbour_slots[t]);
        const float* frame = a.ring + static_cast<size_t>(slot) * a.frame_elems;
        const uint32_t packed_t = t + 1;
        float frame_d = kUnfilled;
        uint32_t frame_pos = 0;
        uint32_t sl[RECTS], sr[RECTS], st[RECTS], sb[RECTS];
#pragma unroll
        for (int i = 0; i < RECTS; ++i) {
            sl[i] = 1;
            sr[i] = 0;
            st[i] = 1;
            sb[i] = 0;
        }
#pragma unroll
        for (int iy = 0; iy < COVERS; ++iy)
#pragma unroll
            for (int ix = 0; ix < COVERS; ++ix) {
                const uint32_t bx = bx_lo + ix, by = by_lo + iy;
                if (bx > bx_hi || by > by_hi) continue;
                const uint32_t block = by * a.blocks_x + bx;
                if (!(__ldg(a.confidence + t * a.conf_stride + block) >= a.c_min)) continue;
                const int mvx = __ldg(a.mv_field + t * a.mv_stride + block * 2);
                const int mvy = __ldg(a.mv_field + t * a.mv_stride + block * 2 + 1);
                const uint32_t left = clamp_top_left(static_cast<int>(ax) + mvx - a.refine, max_x);
                const uint32_t right = clamp_top_left(static_cast<int>(ax) + mvx + a.refine, max_x);
                const uint32_t top = clamp_top_left(static_cast<int>(ay) + mvy - a.refine, max_y);
                const uint32_t bottom = clamp_top_left(static_cast<int>(ay) + mvy + a.refine, max_y);
                bool contained = false;
#pragma unroll
                for (int i = 0; i < RECTS; ++i)
                    contained |= left >= sl[i] && right <= sr[i] && top >= st[i] && bottom <= sb[i];
                if (!contained) {
                    for (uint32_t cy = top; cy <= bottom; ++cy)
                        for (uint32_t cx = left; cx <= right; ++cx) {
                            const float d = reduce8(g, column_ssd<C>(anchor, frame, a.width, cx, cy, g.sub)) * scale;
                            if (!(d < frame_d)) continue;
                            bool skip = false;
#pragma unroll
                            for (int i = 0; i < RECTS; ++i)
                                skip |= cy >= st[i] && cy <= sb[i] && cx >= sl[i] && cx <= sr[i];
                            const uint32_t packed = pack_pos_t(cx, cy, packed_t);
#pragma unroll
                            for (int k = 0; k < FIRST; ++k) skip |= grid_pos[k] == packed;
                            if (skip) continue;
                            frame_d = d;
                            frame_pos = packed;
                        }
                }
                sl[iy * COVERS + ix] = left;
                sr[iy * COVERS + ix] = right;
                st[iy * COVERS + ix] = top;
                sb[iy * COVERS + ix] = bottom;
            }
        float carry_d = frame_d;
        uint32_t carry_pos = frame_pos;
#pragma unroll
        for (int j = 0; j < TAIL; ++j) {
            const float held_d = grid_d[FIRST + j];
            const uint32_t held_pos = grid_pos[FIRST + j];
            if (carry_d < held_d) {
                grid_d[FIRST + j] = carry_d;
                grid_pos[FIRST + j] = carry_pos;
                carry_d = held_d;
                carry_pos = held_pos;
            }
        }
    }
}

template <int C, int GF, int COVERS, int VOL = 0>
__device__ __forceinline__ void search_volumes(const GroupCtx& g, const CollabLaunch& a, const uint32_t (&member_pos)[MAX_K],
                                               float scale, float (&grid_d)[MAX_K], uint32_t (&grid_pos)[MAX_K]) {
    if constexpr (VOL < MAX_K / GF) {
        constexpr int FIRST = VOL * GF;
        const uint32_t anchor_packed = member_pos[VOL];
        const uint32_t ax = anchor_packed & 0x1FFFu, ay = (anchor_packed >> 13) & 0x1FFFu;
        grid_pos[FIRST] = anchor_packed;
        grid_d[FIRST] = 0.0f;
#pragma unroll
        for (int j = 1; j < GF; ++j) {
            grid_pos[FIRST + j] = 0;
            grid_d[FIRST + j] = kUnfilled;
        }
        float anchor[P * C];
        const float* centre = a.ring + static_cast<size_t>(a.centre_slot) * a.frame_elems;
#pragma unroll
        for (int r = 0; r < P; ++r)
#pragma unroll
            for (int c = 0; c < C; ++c)
                anchor[r * C + c] = __ldg(centre + ((static_cast<size_t>(ay) + r) * a.width + ax + g.sub) * C + c);
        trajectory_search<C, GF, FIRST + 1, COVERS>(g, a, anchor, ax, ay, scale, grid_d, grid_pos);
        search_volumes<C, GF, COVERS, VOL + 1>(g, a, member_pos, scale, grid_d, grid_pos);
    }
}

// Keyed top-8 insert: the reference visits the window row by row and keeps ties in visiting order
// (fused/plane_ops.rs:38-53), so its list is the 8 smallest (distance, visiting index) pairs. The
// search here visits columns, comparing the pair, which keeps exactly the same list.
__device__ __forceinline__ bool key_less(float d, uint32_t i, float bd, uint32_t bi) {
    return d < bd || (d == bd && i < bi);
}

__device__ __forceinline__ void shift_insert8_key(const GroupCtx& g, float& best_d, uint32_t& best_i, float d,
                                                  uint32_t i) {
    const float prev_d = __shfl_up_sync(g.mask, best_d, 1, 8);
    const uint32_t prev_i = __shfl_up_sync(g.mask, best_i, 1, 8);
    if (key_less(d, i, best_d, best_i)) {
        if (g.sub == 0 || !key_less(d, i, prev_d, prev_i)) {
            best_d = d;
            best_i = i;
        } else {
            best_d = prev_d;
            best_i = prev_i;
        }
    }
}

template <int C>
__device__ __forceinline__ void load_row(float (&dst)[C], const float* __restrict__ colp, uint32_t row, int width) {
#pragma unroll
    for (int c = 0; c < C; ++c) dst[c] = __ldg(colp + static_cast<size_t>(row) * width * C + c);
}

// The group sums of eight candidates at once, each lane's eight column distances in `v`: the same
// pairwise tree as reduce8 (partners xor 1, then 2, then 4), each level keeping half the candidates
// on each side, so every total has the bits reduce8 gives it. Lane `sub` ends with the total of
// candidate (sub & 1) * 4 + (sub & 2) + ((sub >> 2) & 1).
__device__ __forceinline__ float reduce_scatter8(const GroupCtx& g, const float (&v)[8]) {
    const bool b0 = g.sub & 1, b1 = g.sub & 2, b2 = g.sub & 4;
    float u[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float give = b0 ? v[j] : v[4 + j];
        const float keep = b0 ? v[4 + j] : v[j];
        u[j] = __fadd_rn(keep, __shfl_xor_sync(g.mask, give, 1));
    }
    float w[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const float give = b1 ? u[j] : u[2 + j];
        const float keep = b1 ? u[2 + j] : u[j];
        w[j] = __fadd_rn(keep, __shfl_xor_sync(g.mask, give, 2));
    }
    const float give = b2 ? w[0] : w[1];
    const float keep = b2 ? w[1] : w[0];
    return __fadd_rn(keep, __shfl_xor_sync(g.mask, give, 4));
}

__device__ __forceinline__ int scattered_candidate(int sub) { return (sub & 1) * 4 + (sub & 2) + ((sub >> 2) & 1); }

// Eight candidate rows jb..jb+7 of window column `col` (the lane's sample column `colp`): `rows`
// holds window rows jb..jb+6 on entry and jb+8..jb+14 on exit. Each candidate's distance is its
// column sums in row order, the group's pairwise sum (reduce8's tree), times the channel scale;
// the candidates that beat the list's worst key join it one at a time, in any order (the list is
// the 8 smallest (distance, visiting index) pairs whatever the order they arrive in).
template <int C>
__device__ __forceinline__ void centre_batch(const GroupCtx& g, const float (&cur)[P * C], float (&rows)[15][C],
                                             const float* __restrict__ colp, int width, uint32_t top, uint32_t jb,
                                             uint32_t hh, uint32_t col, uint32_t ww, bool self_col,
                                             uint32_t self_row, float scale, float& best_d, uint32_t& best_i,
                                             float& worst_d, uint32_t& worst_i) {
#pragma unroll
    for (int x = 0; x < 8; ++x) {
        if (jb + x < hh) {
            load_row<C>(rows[7 + x], colp, top + jb + 7 + x, width);
        } else {
#pragma unroll
            for (int c = 0; c < C; ++c) rows[7 + x][c] = 0.0f;
        }
    }
    float v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float sum = 0.0f;
#pragma unroll
        for (int r = 0; r < P; ++r)
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const float d = cur[r * C + c] - rows[k + r][c];
                sum = __fadd_rn(sum, __fmul_rn(d, d));
            }
        v[k] = sum;
    }
    const uint32_t j = jb + static_cast<uint32_t>(scattered_candidate(g.sub));
    float d = reduce_scatter8(g, v) * scale;
    if (self_col && j == self_row) d = kSelfPin;
    const uint32_t i = j * ww + col;
    const bool wins = j < hh && d < kUnfilled && key_less(d, i, worst_d, worst_i);
    unsigned m = __ballot_sync(g.mask, wins) & g.mask;
    while (m) {
        const int src = __ffs(m) - 1;
        m &= m - 1;
        const float dd = __shfl_sync(g.mask, d, src);
        const uint32_t ii = __shfl_sync(g.mask, i, src);
        if (key_less(dd, ii, worst_d, worst_i)) {  // uniform: every lane holds the same words
            shift_insert8_key(g, best_d, best_i, dd, ii);
            worst_d = __shfl_sync(g.mask, best_d, 7, 8);
            worst_i = __shfl_sync(g.mask, best_i, 7, 8);
        }
    }
#pragma unroll
    for (int r = 0; r < 7; ++r)
#pragma unroll
        for (int c = 0; c < C; ++c) rows[r][c] = rows[8 + r][c];
}

// Member words per reference patch: 8 packed positions, then k_use | use_grid << 8.
constexpr int kMemberWords = 9;

template <int C, int GF, int COVERS>
__global__ void __launch_bounds__(kThreads, C == 1 ? 5 : 4) collab_search_kernel(CollabLaunch a) {
    const int lane = threadIdx.x & 31;
    const int group = threadIdx.x >> 3;
    GroupCtx g;
    g.sub = threadIdx.x & 7;
    g.mask = 0xFFu << (lane & ~7);

    const uint32_t refs_x = (a.width - P + STEP - 1) / STEP + 1;
    const uint32_t ix = blockIdx.x * kGroups + group;
    if (ix >= refs_x) return;  // the group's 8 lanes leave together; no barrier spans groups
    const uint32_t iy = blockIdx.y;
    const uint32_t max_x = a.width - P, max_y = a.height - P;
    const uint32_t rx = min(ix * STEP, max_x), ry = min(iy * STEP, max_y);
    const float scale = C == 1 ? 3.0f : 1.5f;
    const float* centre = a.ring + static_cast<size_t>(a.centre_slot) * a.frame_elems;

    float cur[P * C];
#pragma unroll
    for (int r = 0; r < P; ++r)
#pragma unroll
        for (int c = 0; c < C; ++c) cur[r * C + c] = __ldg(centre + ((static_cast<size_t>(ry) + r) * a.width + rx + g.sub) * C + c);

    // Centre search (fused/centre.rs:213-258) over the clipped window, column by column, eight
    // candidate rows at a time with the column's rows in registers: one load per candidate and lane,
    // one reduce-scatter of the group per eight candidates.
    const uint32_t left = clamp_top_left(static_cast<int>(rx) - a.spatial_radius, max_x);
    const uint32_t right = clamp_top_left(static_cast<int>(rx) + a.spatial_radius, max_x);
    const uint32_t top = clamp_top_left(static_cast<int>(ry) - a.spatial_radius, max_y);
    const uint32_t bottom = clamp_top_left(static_cast<int>(ry) + a.spatial_radius, max_y);
    const uint32_t ww = right - left + 1, hh = bottom - top + 1;
    float best_d = kUnfilled, worst_d = kUnfilled;
    uint32_t best_i = 0xFFFFFFFFu, worst_i = 0xFFFFFFFFu;
    for (uint32_t cx = left; cx <= right; ++cx) {
        const float* colp = centre + static_cast<size_t>(cx + g.sub) * C;
        const bool self_col = cx == rx;
        const uint32_t col = cx - left, self_row = ry - top;
        float rows[15][C];
#pragma unroll
        for (int r = 0; r < P - 1; ++r) load_row<C>(rows[r], colp, top + r, a.width);
        for (uint32_t jb = 0; jb < hh; jb += 8)
            centre_batch<C>(g, cur, rows, colp, a.width, top, jb, hh, col, ww, self_col, self_row, scale, best_d,
                            best_i, worst_d, worst_i);
    }
    const uint32_t n_live = ww * hh;
    int k_use = 1;
    while (static_cast<uint32_t>(k_use * 2) <= n_live && k_use * 2 <= a.k_max) k_use *= 2;
    uint32_t member_pos[MAX_K];
#pragma unroll
    for (int m = 0; m < MAX_K; ++m) {
        const uint32_t i = __shfl_sync(g.mask, best_i, m, 8);
        member_pos[m] = i == 0xFFFFFFFFu ? 0u : pack_pos_t(left + i % ww, top + i / ww, 0);
    }

    bool use_grid = false;
    if constexpr (GF > 1) {
        if (a.k_max == MAX_K) {
            float grid_d[MAX_K];
            uint32_t grid_pos[MAX_K];
            search_volumes<C, GF, COVERS>(g, a, member_pos, scale, grid_d, grid_pos);
            use_grid = k_use == MAX_K;
#pragma unroll
            for (int v = 0; v < MAX_K / GF; ++v) use_grid = use_grid && grid_d[v * GF + GF - 1] < kUnfilled;
            if (use_grid) {
#pragma unroll
                for (int m = 0; m < MAX_K; ++m) member_pos[m] = grid_pos[m];
                k_use = MAX_K;
            }
        }
    }
    uint32_t* words = a.members + static_cast<size_t>(iy * refs_x + ix) * kMemberWords;
    uint32_t mine = member_pos[0];
#pragma unroll
    for (int m = 1; m < MAX_K; ++m) mine = g.sub == m ? member_pos[m] : mine;
    words[g.sub] = mine;
    if (g.sub == 0) words[MAX_K] = static_cast<uint32_t>(k_use) | (use_grid ? 0x100u : 0u);
}

// What filter_group (fused/mod.rs:559-850) settles before its transforms: the members and their
// ring slots, the group size and layout, and each channel's threshold multiplier.
struct GroupPlan {
    uint32_t member_pos[MAX_K];
    int member_slot[MAX_K];
    int k_use;
    bool use_grid;
    float first_lambda, second_lambda;
};

template <int C>
__device__ __forceinline__ void plan_group(const CollabLaunch& a, const GroupCtx& g, uint32_t ix, uint32_t iy,
                                           uint32_t refs_x, GroupPlan& plan) {
    const uint32_t max_x = a.width - P, max_y = a.height - P;
    const uint32_t rx = min(ix * STEP, max_x), ry = min(iy * STEP, max_y);
    const float* centre = a.ring + static_cast<size_t>(a.centre_slot) * a.frame_elems;
    float cur[P * C];
#pragma unroll
    for (int r = 0; r < P; ++r)
#pragma unroll
        for (int c = 0; c < C; ++c) cur[r * C + c] = __ldg(centre + ((static_cast<size_t>(ry) + r) * a.width + rx + g.sub) * C + c);
    const uint32_t* words = a.members + static_cast<size_t>(iy * refs_x + ix) * kMemberWords;
#pragma unroll
    for (int m = 0; m < MAX_K; ++m) plan.member_pos[m] = __ldg(words + m);
    const uint32_t meta = __ldg(words + MAX_K);
    plan.k_use = static_cast<int>(meta & 0xFFu);
    plan.use_grid = (meta & 0x100u) != 0;
#pragma unroll
    for (int m = 0; m < MAX_K; ++m) {
        const uint32_t t = plan.member_pos[m] >> 26;
        plan.member_slot[m] = t > 0 ? static_cast<int>(__ldg(a.neighbour_slots + t - 1)) : a.centre_slot;
    }
    float col_first = 0.0f, col_second = 0.0f;
#pragma unroll
    for (int r = 0; r < P; ++r) {
        col_first += cur[r * C];
        if (C > 1) col_second += cur[r * C + 1];
    }
    const float patch_luma = reduce8(g, col_first) / 64.0f;
    const float patch_second = C > 1 ? reduce8(g, col_second) / 64.0f : 0.0f;
    const float bins = static_cast<float>(kCurveBins);
    const float curve_pos = fminf(fmaxf(__fsub_rn(__fmul_rn(patch_luma, bins), 0.5f), 0.0f), bins - 1.0f);
    const uint32_t lower = min(static_cast<uint32_t>(curve_pos), static_cast<uint32_t>(kCurveBins - 2));
    const float fraction = curve_pos - static_cast<float>(lower);
    const bool curve_valid = __ldg(a.noise + a.curve_valid_word) != 0.0f;
    float ratio = 0.0f;
    if (curve_valid) {
        const float lo = __ldg(a.noise_curve + lower), hi = __ldg(a.noise_curve + lower + 1);
        ratio = __fadd_rn(lo, __fmul_rn(__fsub_rn(hi, lo), fraction));
    }
    // fused/colour.rs:48-83 (`threshold_gains`): a luma patch reads the gain at its own mean luma and
    // its block's Cb and Cr, a chroma patch at its own Cb and Cr and its block's luma.
    float first_gain = 1.0f, second_gain = 1.0f;
    if (a.colour_on) {
        const uint32_t bx = (rx + P / 2) / 16, by = (ry + P / 2) / 16;
        const float* m = a.colour_means + (by * static_cast<uint32_t>(a.colour_blocks_x) + bx) * 3;
        if (C == 1) {
            first_gain = exp_mirror(colour::table_value(a.colour_gains, __fmul_rn(patch_luma, a.colour_scale),
                                                        __ldg(m + 1), __ldg(m + 2)));
        } else {
            const float cb = __fsub_rn(__fmul_rn(patch_luma, a.colour_scale), 128.0f);
            const float cr = __fsub_rn(__fmul_rn(patch_second, a.colour_scale), 128.0f);
            colour::gain_pair(a.colour_gains, a.colour_gains + colour::kCells, __ldg(m), cb, cr, &first_gain,
                              &second_gain);
        }
    }
    // fused/mod.rs:643-660: a luma gain joins the curve's scale (together clamped to 0.33..6), a
    // chroma gain scales its channel's threshold.
    float curve_gain = 1.0f, first_channel_gain = first_gain, scale_max = 3.0f;
    if (C == 1) {
        curve_gain = first_gain;
        first_channel_gain = 1.0f;
        scale_max = a.colour_on ? 6.0f : 3.0f;
    }
    const float curve_scale = fminf(fmaxf(__fmul_rn(ratio, curve_gain), 0.33f), scale_max);
    const float flat_scale = fminf(fmaxf(curve_gain, 0.33f), scale_max);
    const float luma_scale = curve_valid ? curve_scale : flat_scale;
    plan.first_lambda = __fmul_rn(__fmul_rn(a.lambda_ht, luma_scale), first_channel_gain);
    plan.second_lambda = __fmul_rn(a.lambda_ht, second_gain);
}

// The 2D DCT of every member (column DCT, transpose, row DCT), then the member-axis transform.
template <int GF>
__device__ __forceinline__ void stack_forward(const GroupCtx& g, float* region, float (&s)[MAX_K][P], int k_use,
                                              bool use_grid) {
#pragma unroll
    for (int m = 0; m < MAX_K; ++m) {
        dct8_fwd(s[m]);
        transpose8(g, region, s[m]);
        dct8_fwd(s[m]);
    }
    if (GF > 1 && use_grid) {
        grid_fwd<(GF > 1 ? GF : 2)>(s);
    } else {
        if (k_use >= 8) haar_level(s, 8, false);
        if (k_use >= 4) haar_level(s, 4, false);
        if (k_use >= 2) haar_level(s, 2, false);
    }
}

template <int GF>
__device__ __forceinline__ void stack_inverse(const GroupCtx& g, float* region, float (&s)[MAX_K][P], int k_use,
                                              bool use_grid) {
    if (GF > 1 && use_grid) {
        grid_inv<(GF > 1 ? GF : 2)>(s);
    } else {
        if (k_use >= 2) haar_level(s, 2, true);
        if (k_use >= 4) haar_level(s, 4, true);
        if (k_use >= 8) haar_level(s, 8, true);
    }
#pragma unroll
    for (int m = 0; m < MAX_K; ++m) {
        dct8_inv(s[m]);
        transpose8(g, region, s[m]);
        dct8_inv(s[m]);
    }
}

// Channel c of every member into the stack (lane `sub` column `sub`), with the propagated noise
// variance of each member-axis coefficient, then the forward transforms.
template <int C, int GF>
__device__ __forceinline__ void group_spectrum(const CollabLaunch& a, const GroupCtx& g, float* region,
                                               const GroupPlan& plan, int c, float (&s)[MAX_K][P],
                                               float (&mv)[MAX_K]) {
    const float sig = __ldg(a.noise + a.sigma_word + c);
    const float base_sig2 = sig * sig;
#pragma unroll
    for (int m = 0; m < MAX_K; ++m) {
        const uint32_t mx = plan.member_pos[m] & 0x1FFFu, my = (plan.member_pos[m] >> 13) & 0x1FFFu;
        const float* src = a.ring + static_cast<size_t>(plan.member_slot[m]) * a.frame_elems;
        mv[m] = base_sig2;
#pragma unroll
        for (int r = 0; r < P; ++r) s[m][r] = __ldg(src + ((static_cast<size_t>(my) + r) * a.width + mx + g.sub) * C + c);
    }
    if (GF > 1 && plan.use_grid) {
        grid_variance<(GF > 1 ? GF : 2)>(mv);
    } else {
        if (plan.k_use >= 8) variance_level(mv, 8);
        if (plan.k_use >= 4) variance_level(mv, 4);
        if (plan.k_use >= 2) variance_level(mv, 2);
    }
    stack_forward<GF>(g, region, s, plan.k_use, plan.use_grid);
}

// The threshold (pooled or per coefficient) and, with `a.wiener`, the empirical Wiener gain
// z^2 / (z^2 + v) on every kept coefficient (an extension: the reference stops at the threshold).
// Returns the lane's retained variance (sum of g^2 v over its kept coefficients) and sets bit
// j * 8 + i of `bits` for every kept coefficient of a live member-axis slot j.
__device__ __forceinline__ float threshold_group(const CollabLaunch& a, const GroupCtx& g, float (&s)[MAX_K][P],
                                                 const float (&mv)[MAX_K], const float (&prof)[P], int k_use,
                                                 float channel_lambda, uint64_t& bits) {
    bits = 0;
    if (a.pooled)
        return pooled_threshold(g, s, mv, prof, k_use, channel_lambda * a.pool_ratio, channel_lambda, a.wiener != 0,
                                bits);
    float retained = 0.0f;
    const float prof_sub = __ldg(a.dct_profile + g.sub);
#pragma unroll
    for (int i = 0; i < P; ++i) {
        const float factor = prof[i] * prof_sub;
#pragma unroll
        for (int j = 0; j < MAX_K; ++j) {
            if (j < k_use) {
                const float cv = mv[j] * factor;
                bool keep = fabsf(s[j][i]) >= channel_lambda * sqrtf(cv);
                if (j == 0 && i == 0 && g.sub == 0) keep = true;
                if (keep && a.wiener) {
                    const float zz = s[j][i] * s[j][i];
                    const float den = zz + cv;
                    const float gain = den > 0.0f ? zz / den : 1.0f;
                    s[j][i] = gain * s[j][i];
                    retained += (gain * gain) * cv;
                } else if (keep) {
                    retained += cv;
                } else {
                    s[j][i] = 0.0f;
                }
                if (keep) bits |= uint64_t{1} << (j * 8 + i);
            }
        }
    }
    return retained;
}

__device__ __forceinline__ float group_weight_of(float sum) {
    return (isnan(sum) || isinf(sum)) ? 0.0f : 1.0f / fmaxf(sum, kReciprocalFloor);
}

template <int C, int GF>
__global__ void __launch_bounds__(kThreads, 3) collab_filter_kernel(CollabLaunch a) {
    __shared__ float transpose_buf[kGroups * kRegion];
    const int lane = threadIdx.x & 31;
    const int group = threadIdx.x >> 3;
    GroupCtx g;
    g.sub = threadIdx.x & 7;
    g.mask = 0xFFu << (lane & ~7);
    float* region = transpose_buf + group * kRegion;

    const uint32_t refs_x = (a.width - P + STEP - 1) / STEP + 1;
    const uint32_t ix = blockIdx.x * kGroups + group;
    if (ix >= refs_x) return;
    const uint32_t iy = blockIdx.y;
    GroupPlan plan;
    plan_group<C>(a, g, ix, iy, refs_x, plan);
    float prof[P];
#pragma unroll
    for (int i = 0; i < P; ++i) prof[i] = __ldg(a.dct_profile + i);
    const float weight_scale = __ldg(a.noise + a.weight_scale_word);
    const uint32_t ref_idx = iy * refs_x + ix;
    const int64_t plane = static_cast<int64_t>(a.width) * a.height;
    float scaled_weight = 0.0f;
    float kaiser_r[P];
#pragma unroll
    for (int r = 0; r < P; ++r) kaiser_r[r] = __ldg(a.kaiser + r);
    const float kaiser_sub = __ldg(a.kaiser + g.sub);

#pragma unroll 1
    for (int c = 0; c < C; ++c) {
        float s[MAX_K][P];
        float mv[MAX_K];
        group_spectrum<C, GF>(a, g, region, plan, c, s, mv);
        uint64_t bits;
        const float retained =
            threshold_group(a, g, s, mv, prof, plan.k_use, c == 0 ? plan.first_lambda : plan.second_lambda, bits);
        const float weight = group_weight_of(reduce8(g, retained));
        if (c == 0) {
            if (g.sub == 0) a.group_weight[ref_idx] = weight;
            scaled_weight = weight * weight_scale;
        }
        stack_inverse<GF>(g, region, s, plan.k_use, plan.use_grid);
        // aggregate.rs:176-211 (`scatter_patch`).
#pragma unroll
        for (int m = 0; m < MAX_K; ++m) {
            if (m >= plan.k_use) break;
            const uint32_t mx = plan.member_pos[m] & 0x1FFFu, my = (plan.member_pos[m] >> 13) & 0x1FFFu;
#pragma unroll
            for (int r = 0; r < P; ++r) {
                const float w = scaled_weight * (kaiser_r[r] * kaiser_sub);
                const int64_t pixel = plan.member_slot[m] * plane + (static_cast<int64_t>(my) + r) * a.width + mx + g.sub;
                atomicAdd(a.accum + pixel * C + c, to_fixed(s[m][r] * w, a.accum_scale));
                if (c == 0) atomicAdd(a.wsum + pixel, to_fixed_weight(w, a.accum_scale));
            }
        }
    }
}

// The adjoint of one pass with its groups and keep decisions held fixed (an extension: the
// reference has none). The pass is read as a smooth function of the ring and the noise levels:
// per group Y = M g Z (Z the forward transform of the members, M the keep mask, g the Wiener
// gain or 1), weight w = ws / R with R channel 0's retained variance, and every member pixel adds
// clamp(w K est, -5, 5) to A and clamp(w K, 0, 1) to W (A and W in real units: the accumulators
// hold A x accum_scale and W x accum_scale x 5). Given dL/dA and dL/dW it adds dL/d(ring) and
// writes each reference patch's share of dL/d(sigma_c), the weight-scale word read as proportional
// to sigma_0^2 as the engine derives it (aggregate.rs:79-99), so that with the hard threshold a
// group weight does not move with sigma at all (R moves as sigma_0^2 too). The
// keep masks are recomputed from the ring with the filter's own arithmetic, so they are the
// forward's bit for bit. Z waits in shared memory for the Wiener terms, one float per thread and
// coefficient, thread-minor so a warp's stores hit 32 banks.
template <int C, int GF>
__global__ void __launch_bounds__(kThreads, 2) collab_adjoint_kernel(CollabLaunch a, CollabAdjointLaunch b) {
    __shared__ float transpose_buf[kGroups * kRegion];
    __shared__ float spectrum[MAX_K * P * kThreads];
    const int lane = threadIdx.x & 31;
    const int group = threadIdx.x >> 3;
    GroupCtx g;
    g.sub = threadIdx.x & 7;
    g.mask = 0xFFu << (lane & ~7);
    float* region = transpose_buf + group * kRegion;

    const uint32_t refs_x = (a.width - P + STEP - 1) / STEP + 1;
    const uint32_t ix = blockIdx.x * kGroups + group;
    if (ix >= refs_x) return;
    const uint32_t iy = blockIdx.y;
    GroupPlan plan;
    plan_group<C>(a, g, ix, iy, refs_x, plan);
    float prof[P];
#pragma unroll
    for (int i = 0; i < P; ++i) prof[i] = __ldg(a.dct_profile + i);
    const float prof_sub = prof[g.sub];
    const float weight_scale = __ldg(a.noise + a.weight_scale_word);
    const uint32_t ref_idx = iy * refs_x + ix;
    const int64_t plane = static_cast<int64_t>(a.width) * a.height;
    float kaiser_r[P];
#pragma unroll
    for (int r = 0; r < P; ++r) kaiser_r[r] = __ldg(a.kaiser + r);
    const float kaiser_sub = __ldg(a.kaiser + g.sub);

    // Channel 0's weight first when a second channel is processed before it.
    float weight = 0.0f, retained0 = 0.0f;
    if (C > 1) {
        float s[MAX_K][P];
        float mv[MAX_K];
        group_spectrum<C, GF>(a, g, region, plan, 0, s, mv);
        uint64_t bits;
        retained0 = reduce8(g, threshold_group(a, g, s, mv, prof, plan.k_use, plan.first_lambda, bits));
        weight = group_weight_of(retained0);
    }
    float dweight = 0.0f;  // this lane's share of dL/d(w ws)
#pragma unroll 1
    for (int step = 0; step < C; ++step) {
        const int c = C - 1 - step;  // channel 0 last: its retained variance carries every channel's dL/dw
        float s[MAX_K][P];
        float mv[MAX_K];
        group_spectrum<C, GF>(a, g, region, plan, c, s, mv);
#pragma unroll
        for (int j = 0; j < MAX_K; ++j)
#pragma unroll
            for (int i = 0; i < P; ++i) spectrum[(j * P + i) * kThreads + threadIdx.x] = s[j][i];
        uint64_t bits;
        const float retained =
            threshold_group(a, g, s, mv, prof, plan.k_use, c == 0 ? plan.first_lambda : plan.second_lambda, bits);
        if (C == 1) {
            retained0 = reduce8(g, retained);
            weight = group_weight_of(retained0);
        }
        const float scaled_weight = weight * weight_scale;
        stack_inverse<GF>(g, region, s, plan.k_use, plan.use_grid);
        // Back through the scatter: s becomes d est, and each pixel adds its share of dL/dw.
#pragma unroll
        for (int m = 0; m < MAX_K; ++m) {
            const uint32_t mx = plan.member_pos[m] & 0x1FFFu, my = (plan.member_pos[m] >> 13) & 0x1FFFu;
#pragma unroll
            for (int r = 0; r < P; ++r) {
                const float window = kaiser_r[r] * kaiser_sub;
                const float w = scaled_weight * window;
                float d_est = 0.0f;
                if (m < plan.k_use) {
                    const int64_t pixel =
                        plan.member_slot[m] * plane + (static_cast<int64_t>(my) + r) * a.width + mx + g.sub;
                    float d_w = 0.0f;
                    const float e = s[m][r];
                    if (fabsf(e * w) < kAccumClamp) {
                        const float ga = __ldg(b.grad_accum + pixel * C + c);
                        d_est = ga * w;
                        d_w = ga * e;
                    }
                    if (c == 0 && w > 0.0f && w < 1.0f) d_w += __ldg(b.grad_wsum + pixel);
                    dweight += d_w * window;
                }
                s[m][r] = d_est;
            }
        }
        stack_forward<GF>(g, region, s, plan.k_use, plan.use_grid);  // s = dL/dY
        const float sig = __ldg(a.noise + a.sigma_word + c);
        float d_retained = 0.0f, d_sigma = 0.0f;
        if (c == 0) {
            const float total = reduce8(g, dweight);
            const bool live = !(isnan(retained0) || isinf(retained0)) && retained0 > kReciprocalFloor;
            d_retained = live ? -total * weight_scale * weight * weight : 0.0f;
            if (g.sub == 0 && sig > 0.0f) d_sigma = total * 2.0f * scaled_weight / sig;  // through the word
        }
        const bool wiener = a.wiener != 0;
#pragma unroll
        for (int j = 0; j < MAX_K; ++j)
#pragma unroll
            for (int i = 0; i < P; ++i) {
                const bool keep = (bits >> (j * 8 + i)) & 1u;
                const float var_unit = prof[i] * prof_sub;  // v / sigma^2
                const float v = mv[j] * var_unit;
                const float dy = s[j][i];
                float dz = dy, dv = c == 0 ? d_retained : 0.0f;
                if (wiener) {
                    const float z = spectrum[(j * P + i) * kThreads + threadIdx.x];
                    const float den = z * z + v;
                    if (den > 0.0f) {
                        const float gain = z * z / den;
                        const float inv = 1.0f / den;
                        dz = dy * gain * (z * z + 3.0f * v) * inv;
                        dv = -dy * gain * z * inv;
                        if (c == 0) {
                            dz += d_retained * 4.0f * gain * z * v * v * inv * inv;
                            dv += d_retained * gain * gain * (z * z - v) * inv;
                        }
                    }
                }
                s[j][i] = keep ? dz : 0.0f;
                if (keep) d_sigma += dv * 2.0f * sig * var_unit;
            }
        stack_inverse<GF>(g, region, s, plan.k_use, plan.use_grid);  // s = dL/dX
#pragma unroll
        for (int m = 0; m < MAX_K; ++m) {
            if (m >= plan.k_use) break;
            const uint32_t mx = plan.member_pos[m] & 0x1FFFu, my = (plan.member_pos[m] >> 13) & 0x1FFFu;
            float* dst = b.grad_ring + static_cast<size_t>(plan.member_slot[m]) * a.frame_elems;
#pragma unroll
            for (int r = 0; r < P; ++r)
                atomicAdd(dst + ((static_cast<size_t>(my) + r) * a.width + mx + g.sub) * C + c, s[m][r]);
        }
        d_sigma = reduce8(g, d_sigma);
        if (g.sub == 0) b.grad_sigma_refs[static_cast<size_t>(ref_idx) * C + c] = d_sigma;
    }
}

template <int C, int GF, int COVERS>
cudaError_t launch_cgc(const CollabLaunch& a, cudaStream_t stream) {
    const uint32_t refs_x = (a.width - P + STEP - 1) / STEP + 1;
    const uint32_t refs_y = (a.height - P + STEP - 1) / STEP + 1;
    dim3 grid((refs_x + kGroups - 1) / kGroups, refs_y);
    collab_search_kernel<C, GF, COVERS><<<grid, kThreads, 0, stream>>>(a);
    collab_filter_kernel<C, GF><<<grid, kThreads, 0, stream>>>(a);
    return cudaGetLastError();
}

template <int C, int GF>
cudaError_t launch_cg(const CollabLaunch& a, cudaStream_t stream) {
    if (GF == 1) return launch_cgc<C, GF, 1>(a, stream);  // no volumes: the walk never runs
    switch ((a.blksize + a.blk_step - 1) / a.blk_step) {
        case 1: return launch_cgc<C, GF, 1>(a, stream);
        case 2: return launch_cgc<C, GF, 2>(a, stream);
        case 3: return launch_cgc<C, GF, 3>(a, stream);
        default: return launch_cgc<C, GF, 4>(a, stream);
    }
}

cudaError_t upload_taps() {
    static bool done = false;
    if (done) return cudaSuccess;
    float taps[8][8];
    for (int row = 0; row < 8; ++row)
        for (int col = 0; col < 8; ++col) {
            const double scale = row == 0 ? 1.0 / 2.8284271247461903 : 0.5;
            taps[row][col] = static_cast<float>(scale * cos(3.14159265358979323846 * (2.0 * col + 1.0) * row / 16.0));
        }
    cudaError_t e = cudaMemcpyToSymbol(c_dct, taps, sizeof(taps));
    if (e == cudaSuccess) done = true;
    return e;
}

template <int C, int GF>
cudaError_t launch_adjoint_cg(const CollabLaunch& a, const CollabAdjointLaunch& b, cudaStream_t stream) {
    const uint32_t refs_x = (a.width - P + STEP - 1) / STEP + 1;
    const uint32_t refs_y = (a.height - P + STEP - 1) / STEP + 1;
    dim3 grid((refs_x + kGroups - 1) / kGroups, refs_y);
    collab_adjoint_kernel<C, GF><<<grid, kThreads, 0, stream>>>(a, b);
    return cudaGetLastError();
}

}  // namespace

size_t collab_member_words(int width, int height) {
    if (width < P || height < P) return 0;
    const size_t rx = (width - P + STEP - 1) / STEP + 1, ry = (height - P + STEP - 1) / STEP + 1;
    return rx * ry * kMemberWords;
}

cudaError_t launch_collab_adjoint(const CollabLaunch& a, const CollabAdjointLaunch& b, cudaStream_t stream) {
    if (!a.members || !b.grad_accum || !b.grad_wsum || !b.grad_ring || !b.grad_sigma_refs)
        return cudaErrorInvalidValue;
    if (a.width < P || a.height < P || a.radius < 0 || a.radius > 8) return cudaErrorInvalidValue;
    cudaError_t e = upload_taps();
    if (e != cudaSuccess) return e;
    const int gf = a.radius == 0 ? 1 : (a.radius == 1 ? 2 : 4);
    if (a.channels == 1) {
        if (gf == 1) return launch_adjoint_cg<1, 1>(a, b, stream);
        if (gf == 2) return launch_adjoint_cg<1, 2>(a, b, stream);
        return launch_adjoint_cg<1, 4>(a, b, stream);
    }
    if (a.channels == 2) {
        if (gf == 1) return launch_adjoint_cg<2, 1>(a, b, stream);
        if (gf == 2) return launch_adjoint_cg<2, 2>(a, b, stream);
        return launch_adjoint_cg<2, 4>(a, b, stream);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_collab(const CollabLaunch& a, cudaStream_t stream) {
    if (!a.members) return cudaErrorInvalidValue;
    if (a.width < P || a.height < P || a.k_max < 1 || a.k_max > MAX_K || a.radius < 0 || a.radius > 8)
        return cudaErrorInvalidValue;
    if ((a.blksize + a.blk_step - 1) / max(a.blk_step, 1) > 4 || a.blk_step < 1) return cudaErrorInvalidValue;
    cudaError_t e = upload_taps();
    if (e != cudaSuccess) return e;
    const int gf = a.radius == 0 ? 1 : (a.radius == 1 ? 2 : 4);
    if (a.channels == 1) {
        if (gf == 1) return launch_cg<1, 1>(a, stream);
        if (gf == 2) return launch_cg<1, 2>(a, stream);
        return launch_cg<1, 4>(a, stream);
    }
    if (a.channels == 2) {
        if (gf == 1) return launch_cg<2, 1>(a, stream);
        if (gf == 2) return launch_cg<2, 2>(a, stream);
        return launch_cg<2, 4>(a, stream);
    }
    return cudaErrorInvalidValue;
}

}  // namespace avd
