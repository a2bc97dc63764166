// The truemotion stage that ends a motion search, for sm_100a: every block picks its vector again
// from a few candidates under a penalty toward its neighbourhood's consensus.
//
// Reference behaviour (av-denoise-core/src/motion/truemotion):
//   kernels/truemotion/candidates.rs:124-176  the component-wise lower median of the on-grid blocks
//                       of the 3x3 neighbourhood (the block's own vector when it has none);
//   candidates.rs:178-306  the distinct candidates in order: own, median, left, right, up, down,
//                       zero, (the camera model's prediction), the block's coarse seed and its four
//                       diagonal blocks' seeds;
//   score.rs:7-61       each candidate's SAD over the block at level 0, every row summed left to
//                       right, then the rows top to bottom, coordinates clamped to the frame;
//   mod.rs:230-276      cost = SAD + lambda * |v - median|_1, plus surcharge * SAD off the median;
//                       lambda = lambda_base + lambda_noise * floor, faded by
//                       level^2 / (level^2 + max(median SAD - floor, 0)^2);
//   mod.rs:292-345      the early settle on the own vector and the median;
//   mod.rs:347-441      the lowest cost (a tie keeps the earlier entry), then, when the winner is not
//                       the block's own vector, the ring within the refine radius around it, each
//                       replacing the best only when strictly cheaper;
//   mod.rs:448-463, 492-535  the vector, and the confidence max(0, (T^2 - e^2) / (T^2 + e^2)).
// With the camera model's predictions its point at the block joins the list after zero; with a SAD
// output every rescored block writes its winning SAD. A second pass, after a search that escalates,
// reads the change flags of the first.
//
// Layout and design: one warp per (block, neighbour), four per CTA, each with its own slice of
// shared memory: the staged 3x3 field and seeds, the candidate list, a |difference| tile and the
// row sums. Candidates are scored in chunks of 32 / blksize: lane l owns column l mod blksize of
// candidate l / blksize, keeps that column of the centre block in registers, and walks down the
// rows (so each load instruction reads whole row segments) writing |centre - neighbour| into the
// tile (rows padded to an odd stride); then each lane sums one tile row left to right, and one lane
// per candidate adds its rows top to bottom, so every SAD is the reference's sum bit for bit. The
// candidate logic runs on lane 0 from the staged words. The block size is a template argument for
// 8, 16 and 32 (0 = any other, the centre block then read from shared memory). The file is built
// with -fmad=false so no multiply-add is fused.

#include <cuda_runtime.h>

#include <cstdint>

#include "camera_model.cuh"
#include "kernels.h"

namespace avd {

namespace {

constexpr int kWarps = 4;
constexpr int kMaxBlk = 32;
constexpr int kListCap = 13;  // mod.rs:10-14 (TRUEMOTION_CANDIDATES)

template <int BLK>
struct WarpSlice {
    static constexpr int kB = BLK ? BLK : kMaxBlk;
    float centre[BLK ? 1 : kB * kB];  // the generic block size's centre block
    float diffs[32 * (kB + 1)];       // 32 rows of |centre - neighbour|, odd stride
    float row_sums[kListCap * kB];
    float sads[kListCap];
    int list[2 * kListCap];
    int staged[36];  // the 3x3 field, then the 3x3 seeds, (dx, dy) per block, 0 off the grid
    int count;
};

// The centre block's column that a lane owns, in registers for the templated block sizes.
template <int BLK>
struct CentreColumn {
    float v[BLK ? BLK : 1];
};

__device__ __forceinline__ int clamp_to(int v, int limit) { return v < 0 ? 0 : (v >= limit ? limit - 1 : v); }

__device__ __forceinline__ bool on_grid(int c, int r, int bx, int by) { return c >= 0 && r >= 0 && c < bx && r < by; }

__device__ __forceinline__ int push_unique(int* list, int count, int dx, int dy) {
    for (int e = 0; e < count; ++e)
        if (list[2 * e] == dx && list[2 * e + 1] == dy) return count;
    list[2 * count] = dx;
    list[2 * count + 1] = dy;
    return count + 1;
}

__device__ __forceinline__ float penalised_cost(float sad, int vx, int vy, int mx, int my, float lambda,
                                                float surcharge) {
    const int deviation = abs(vx - mx) + abs(vy - my);
    float cost = sad + lambda * static_cast<float>(deviation);
    if (deviation != 0 && surcharge > 0.0f) cost += surcharge * sad;
    return cost;
}

// Scores list entries [first, count) into `sads` with the whole warp.
template <int BLK>
__device__ __forceinline__ void score(WarpSlice<BLK>& w, const CentreColumn<BLK>& cc, int first, int count,
                                      const TruemotionLaunch& t, const float* __restrict__ nbr, int ox, int oy,
                                      int lane) {
    const int B = BLK ? BLK : t.blksize;
    const int stride = B + 1;
    const int per = 32 / B;  // candidates per chunk of at most 32 rows
    const int my_cand = lane / B, ix = lane - my_cand * B;
    for (int c0 = first; c0 < count; c0 += per) {
        const int nc = min(per, count - c0);
        if (my_cand < nc) {
            const int e = c0 + my_cand;
            const int mvx = w.list[2 * e], mvy = w.list[2 * e + 1];
            const float* column = nbr + clamp_to(ox + ix + mvx, t.width);
            float* d = w.diffs + my_cand * B * stride + ix;
            if (BLK) {
#pragma unroll
                for (int r = 0; r < (BLK ? BLK : 1); ++r) {
                    const float nv = __ldg(column + static_cast<int64_t>(clamp_to(oy + r + mvy, t.height)) * t.width);
                    d[r * stride] = fabsf(cc.v[r] - nv);
                }
            } else {
                for (int r = 0; r < B; ++r) {
                    const float nv = __ldg(column + static_cast<int64_t>(clamp_to(oy + r + mvy, t.height)) * t.width);
                    d[r * stride] = fabsf(w.centre[r * B + ix] - nv);
                }
            }
        }
        __syncwarp();
        if (lane < nc * B) {
            const float* d = w.diffs + lane * stride;
            float s = 0.0f;
            for (int ix = 0; ix < B; ++ix) s += d[ix];
            w.row_sums[(c0 - first) * B + lane] = s;
        }
        __syncwarp();
    }
    for (int e = first + lane; e < count; e += 32) {
        float sad = 0.0f;
        for (int iy = 0; iy < B; ++iy) sad += w.row_sums[(e - first) * B + iy];
        w.sads[e] = sad;
    }
    __syncwarp();
}

template <int BLK>
__global__ void __launch_bounds__(kWarps * 32) truemotion_kernel(TruemotionLaunch t) {
    __shared__ WarpSlice<BLK> slices[kWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int blocks = t.blocks_x * t.blocks_y;
    const int blk = blockIdx.x * kWarps + warp;
    if (blk >= blocks) return;  // whole warps leave; only warp-level barriers follow
    WarpSlice<BLK>& w = slices[warp];
    const int n = blockIdx.y;
    const int col = blk % t.blocks_x, row = blk / t.blocks_x;
    const int ox = col * t.step, oy = row * t.step;
    const int B = BLK ? BLK : t.blksize;
    const uint32_t nslot = t.neighbour_slots ? t.neighbour_slots[n] : t.inline_slots[n];
    const float* centre = t.pyramid + static_cast<int64_t>(t.centre_slot) * t.slot_pixels;
    const float* nbr = t.pyramid + static_cast<int64_t>(nslot) * t.slot_pixels;
    const int32_t* field = t.mv_in + static_cast<int64_t>(n) * t.mv_stride;
    const int32_t* seeds = t.seeds ? t.seeds + static_cast<int64_t>(n) * t.mv_stride : nullptr;
    // mod.rs:483-520, 656-680: a block whose 3x3 neighbourhood kept every vector last pass would
    // pick what it holds again, and its confidence from that pass still stands.
    if (t.changes_in) {
        bool changed = false;
        if (lane < 9) {
            const int c = col + lane % 3 - 1, r = row + lane / 3 - 1;
            changed = on_grid(c, r, t.blocks_x, t.blocks_y) &&
                      __ldg(t.changes_in + static_cast<int64_t>(n) * t.conf_stride + r * t.blocks_x + c) != 0u;
        }
        if (!__any_sync(0xffffffffu, changed)) {
            if (lane == 0) {
                int32_t* out = t.mv_out + static_cast<int64_t>(n) * t.mv_stride + 2 * blk;
                out[0] = field[2 * blk];
                out[1] = field[2 * blk + 1];
                if (t.changes_out) t.changes_out[static_cast<int64_t>(n) * t.conf_stride + blk] = 0u;
            }
            return;  // the whole warp leaves together
        }
    }

    CentreColumn<BLK> cc;
    if (BLK) {
        const int cx = clamp_to(ox + lane % (BLK ? BLK : 1), t.width);
#pragma unroll
        for (int r = 0; r < (BLK ? BLK : 1); ++r)
            cc.v[r] = __ldg(centre + static_cast<int64_t>(clamp_to(oy + r, t.height)) * t.width + cx);
    } else {
        for (int p = lane; p < B * B; p += 32) {
            const int py = p / B, px = p - (p / B) * B;
            w.centre[p] = __ldg(centre + static_cast<int64_t>(clamp_to(oy + py, t.height)) * t.width +
                                clamp_to(ox + px, t.width));
        }
    }
    // candidates.rs:18-66 (`stage_neighbourhood`): the 3x3 field and seeds, one word per lane.
    for (int word = lane; word < 36; word += 32) {
        const bool reads_seeds = word >= 18;
        const int fw = word % 18, pos = fw / 2, comp = fw % 2;
        const int c = col + pos % 3 - 1, r = row + pos / 3 - 1;
        int value = 0;
        if (on_grid(c, r, t.blocks_x, t.blocks_y) && (!reads_seeds || seeds)) {
            const int64_t i = 2 * (static_cast<int64_t>(r) * t.blocks_x + c) + comp;
            value = reads_seeds ? __ldg(seeds + i) : __ldg(field + i);
        }
        w.staged[word] = value;
    }
    __syncwarp();

    // Lane 0: the median and the candidate list (candidates.rs:124-306).
    int own_x = 0, own_y = 0, med_x = 0, med_y = 0, median_entry = 0;
    if (lane == 0) {
        const int* sf = w.staged;
        const int* ss = w.staged + 18;
        own_x = sf[8];
        own_y = sf[9];
        int xs[8], ys[8], cnt = 0;
        for (int pos = 0; pos < 9; ++pos) {
            if (pos == 4) continue;
            const int c = col + pos % 3 - 1, r = row + pos / 3 - 1;
            if (!on_grid(c, r, t.blocks_x, t.blocks_y)) continue;
            // insertion into the sorted runs of each component
            int vx = sf[2 * pos], vy = sf[2 * pos + 1];
            int j = cnt;
            while (j > 0 && xs[j - 1] > vx) {
                xs[j] = xs[j - 1];
                --j;
            }
            xs[j] = vx;
            j = cnt;
            while (j > 0 && ys[j - 1] > vy) {
                ys[j] = ys[j - 1];
                --j;
            }
            ys[j] = vy;
            ++cnt;
        }
        med_x = cnt ? xs[(cnt - 1) / 2] : own_x;
        med_y = cnt ? ys[(cnt - 1) / 2] : own_y;
        int count = 0;
        count = push_unique(w.list, count, own_x, own_y);
        count = push_unique(w.list, count, med_x, med_y);
        const int sdx[4] = {-1, 1, 0, 0}, sdy[4] = {0, 0, -1, 1};
        for (int s = 0; s < 4; ++s) {
            const int c = col + sdx[s], r = row + sdy[s];
            if (on_grid(c, r, t.blocks_x, t.blocks_y)) {
                const int pos = 3 * (sdy[s] + 1) + sdx[s] + 1;
                count = push_unique(w.list, count, sf[2 * pos], sf[2 * pos + 1]);
            }
        }
        count = push_unique(w.list, count, 0, 0);
        if (t.predictions && predicts_motion(t.predictions + n * kAffineWords)) {
            int mdx, mdy;
            model_point(t.predictions + n * kAffineWords, ox, oy, B, 1, t.width, t.height, &mdx, &mdy);
            count = push_unique(w.list, count, mdx, mdy);
        }
        if (seeds) {
            count = push_unique(w.list, count, ss[8], ss[9]);
            for (int corner = 0; corner < 4; ++corner) {
                const int ddx = (corner % 2) * 2 - 1, ddy = (corner / 2) * 2 - 1;
                if (on_grid(col + ddx, row + ddy, t.blocks_x, t.blocks_y)) {
                    const int pos = 3 * (ddy + 1) + ddx + 1;
                    count = push_unique(w.list, count, ss[2 * pos], ss[2 * pos + 1]);
                }
            }
        }
        for (int e = count - 1; e >= 0; --e)
            if (w.list[2 * e] == med_x && w.list[2 * e + 1] == med_y) median_entry = e;
        w.count = count;
    }
    __syncwarp();
    const int listed = w.count;
    const int head = listed < 2 ? listed : 2;
    score<BLK>(w, cc, 0, head, t, nbr, ox, oy, lane);

    // Lane 0 decides; the lanes follow its broadcast outcome through the remaining scoring.
    int outcome = 0;
    float lambda = 0.0f, best_cost = 0.0f, best_sad = 0.0f;
    int best_x = 0, best_y = 0;
    if (lane == 0) {
        const float median_sad = w.sads[median_entry];
        float floor = 0.0f;
        if (t.reads_floor) {
            const float reading = __ldg(t.noise + t.sad_field);
            if (reading > 0.0f) floor = reading;
        }
        lambda = t.lambda_base + t.lambda_noise * floor;
        if (t.fade_level > 0.0f) {
            const float excess = fmaxf(median_sad - floor, 0.0f);
            const float level_sq = t.fade_level * t.fade_level;
            const float fade = __fdiv_rn(level_sq, level_sq + excess * excess);
            lambda *= fade;
        }
        const float own_cost = penalised_cost(w.sads[0], own_x, own_y, med_x, med_y, lambda, t.surcharge);
        const float median_cost = penalised_cost(median_sad, med_x, med_y, med_x, med_y, lambda, t.surcharge);
        if (listed == 1 || (median_entry == 0 && own_cost <= lambda)) {
            outcome = 1;
        } else if (median_entry == 1) {
            if (own_cost <= median_cost && own_cost <= lambda) outcome = 1;
            else if (median_cost < own_cost && median_cost <= lambda) outcome = 2;
        }
        best_x = own_x;
        best_y = own_y;
        best_cost = own_cost;
        best_sad = w.sads[0];
        if (outcome == 2) {
            best_x = med_x;
            best_y = med_y;
            best_cost = median_cost;
            best_sad = median_sad;
        }
    }
    outcome = __shfl_sync(0xffffffffu, outcome, 0);
    if (outcome == 0) {
        score<BLK>(w, cc, head, listed, t, nbr, ox, oy, lane);
        if (lane == 0) {
            int bi = 0;
            for (int e = 1; e < listed; ++e) {
                const float cost =
                    penalised_cost(w.sads[e], w.list[2 * e], w.list[2 * e + 1], med_x, med_y, lambda, t.surcharge);
                if (cost < best_cost) {
                    best_cost = cost;
                    bi = e;
                }
            }
            best_x = w.list[2 * bi];
            best_y = w.list[2 * bi + 1];
            best_sad = w.sads[bi];
        }
    }
    int refines = 0;
    if (lane == 0) {
        refines = outcome != 1 && t.refine_radius > 0 && !(best_x == own_x && best_y == own_y);
        if (refines) {
            int count = 0;
            for (int ry = -t.refine_radius; ry <= t.refine_radius; ++ry)
                for (int rx = -t.refine_radius; rx <= t.refine_radius; ++rx) {
                    if (rx == 0 && ry == 0) continue;
                    w.list[2 * count] = best_x + rx;
                    w.list[2 * count + 1] = best_y + ry;
                    ++count;
                }
            w.count = count;
        }
    }
    __syncwarp();
    refines = __shfl_sync(0xffffffffu, refines, 0);
    if (refines) {
        const int ring = w.count;
        score<BLK>(w, cc, 0, ring, t, nbr, ox, oy, lane);
        if (lane == 0) {
            for (int e = 0; e < ring; ++e) {
                const int vx = w.list[2 * e], vy = w.list[2 * e + 1];
                const float cost = penalised_cost(w.sads[e], vx, vy, med_x, med_y, lambda, t.surcharge);
                if (cost < best_cost) {
                    best_cost = cost;
                    best_sad = w.sads[e];
                    best_x = vx;
                    best_y = vy;
                }
            }
        }
    }
    if (lane == 0) {
        int32_t* out = t.mv_out + static_cast<int64_t>(n) * t.mv_stride + 2 * blk;
        out[0] = best_x;
        out[1] = best_y;
        if (t.confidence) {
            float excess = best_sad - __ldg(t.noise + t.sad_field);
            if (excess < 0.0f) excess = 0.0f;
            const float t2 = t.thsad * t.thsad, e2 = excess * excess;
            float c = __fdiv_rn(t2 - e2, t2 + e2);
            if (c < 0.0f) c = 0.0f;
            t.confidence[static_cast<int64_t>(n) * t.conf_stride + blk] = c;
        }
        if (t.sad) t.sad[static_cast<int64_t>(n) * t.conf_stride + blk] = best_sad;
        if (t.changes_out)
            t.changes_out[static_cast<int64_t>(n) * t.conf_stride + blk] =
                (best_x == field[2 * blk] && best_y == field[2 * blk + 1]) ? 0u : 1u;
    }
}

}  // namespace

cudaError_t launch_truemotion(const TruemotionLaunch& t, cudaStream_t s) {
    if (!t.pyramid || !t.mv_in || !t.mv_out || t.mv_in == t.mv_out || t.blksize < 1 || t.blksize > kMaxBlk ||
        t.neighbours < 1 || (!t.neighbour_slots && t.neighbours > TruemotionLaunch::kMaxInlineSlots) ||
        t.refine_radius < 0 || t.refine_radius > 1 || t.blocks_x < 1 || t.blocks_y < 1 ||
        (t.confidence && !t.noise) || (t.reads_floor && !t.noise))
        return cudaErrorInvalidValue;
    const int blocks = t.blocks_x * t.blocks_y;
    dim3 grid((blocks + kWarps - 1) / kWarps, t.neighbours);
    if (t.blksize == 16) truemotion_kernel<16><<<grid, kWarps * 32, 0, s>>>(t);
    else if (t.blksize == 8) truemotion_kernel<8><<<grid, kWarps * 32, 0, s>>>(t);
    else if (t.blksize == 32) truemotion_kernel<32><<<grid, kWarps * 32, 0, s>>>(t);
    else truemotion_kernel<0><<<grid, kWarps * 32, 0, s>>>(t);
    return cudaGetLastError();
}

}  // namespace avd
