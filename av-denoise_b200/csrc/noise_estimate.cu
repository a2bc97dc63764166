// The automatic noise estimate on sm_100a, without motion compensation: per-block temporal residual
// statistics, one frame's reading and the window fold into the derived words and offset tables.
//
// Reference behaviour (av-denoise-core/src/noise):
//   kernels/stats.rs:141-620   `nlm_temporal_noise_stats`: per 16x16 block the per-channel sums of
//                              d = new - prev and d^2 and the lag-1 channel-0 product, each summed
//                              over the block's 256 threads in thread order; each channel's texture
//                              from 4x4 cell means (stats.rs:599-650); with a motion field, the
//                              compensated variant's vector check; with the luma fields, each 8x8
//                              quarter's residual sums, luma sum, minimum, maximum and flatness.
//   kernels/sample.rs:143-803  `noise_block_derive`, `noise_block_accept`, `noise_sample_finish`:
//                              the static gate, the outlier ceiling, the moved-texture threshold, the
//                              kept sigmas' median and lower quartile, the median correlation; with
//                              the luma fields, the noise curve (kernels/curve.rs:37-133): the static
//                              quarters' median sigma and the 16 luma bins' medians, interpolated.
//   kernels/window.rs:1-498, kernels/derive.rs:1-192
//                              `noise_window_fold`: four chains' medians over the window, the stream
//                              state, the derived words and both NLM offset tables.
//
// Design. The reference runs the reading as 9 launches over three tagged radix-select batches. Here
// one CTA of 1024 threads builds the whole reading: it derives every block's values into a small
// global scratch (L2-resident: at 3840x2160 that is 32,400 blocks), answers each order statistic
// with an exact 4-pass 8-bit radix select (one warp scans each query's histogram), and writes the
// reading words into the frame's history slot. The fold is one CTA as well. Order statistics are
// exact, so the results equal the reference's tagged selects; every other step rounds each multiply
// and add on its own (this file is built with -fmad=false), as the oracle does.

#include <cstdint>

#include "kernels.h"

namespace avd {
namespace {

constexpr int kNB = 16;
constexpr int kNoiseChannels = 2;
constexpr int kReadingThreads = 1024;
constexpr int kReadingWords = 30;
constexpr uint32_t kExcluded = 0xFFFFFFFFu;
constexpr float kStaticGate = 1.5f / 255.0f;
constexpr float kRhoSigmaGate = 0.3f / 255.0f;
constexpr float kOutlierFactor = 5.0f;
constexpr float kSigmaFloor = 0.1f / 255.0f;
constexpr float kSqrt2 = 1.41421356237309504880f;
// The luma quarter fields (noise/temporal.rs:20-62) and the noise curve (noise/curve.rs:21-50).
constexpr int kQuarterBase = 3, kQuarterFields = 6;
constexpr int Q_SUM_D = 0, Q_SUM_D2 = 1, Q_LUMA_SUM = 2, Q_FLATNESS = 3, Q_LUMA_MIN = 4, Q_LUMA_MAX = 5;
constexpr float kUnmeasuredFlatness = 3.0e38f;
constexpr int kCurveBins = 16;
constexpr uint32_t kMinBinQuarters = 32, kMinPopulatedBins = 3;
constexpr float kClipLow = 4.0f / 255.0f, kClipHigh = 251.0f / 255.0f, kFlatFactor = 0.5f;
constexpr float kFlatFloor = (1.0f / 255.0f) * (1.0f / 255.0f);
constexpr float kQuarterStaticGate = 2.0f * kStaticGate;

// Reading, fold-settings, state and derived word layouts (noise/reading.rs, fold.rs, derived.rs).
constexpr int R_VALID = 2, R_SIGMA = 4, R_SIGMA_LOW = 6, R_RHO = 8, R_STATIC = 9, R_ACCEPTED = 10,
              R_CURVE_VALID = 11, R_QUARTER_MEDIAN = 12, R_POPULATED = 13, R_RATIOS = 14;
constexpr int F_SIGMA_SCALE = 0, F_CURVE_APPLIES = 1, F_G_MAX = 2, F_W_FLOOR = 3, F_H2_AUTO = 4, F_H2_PIV = 5,
              F_H2_FIXED = 6, F_PILOT = 7, F_OFFSET_PV = 8, F_MAIN_OFFSET = 9, F_SAD = 10, F_CONF_SAD = 11,
              F_IMM = 12, F_SEG = 13;
constexpr int S_MEDIAN = 0, S_LOW = 3, S_LOW_UNB = 6, S_TEMPORAL = 9, S_RHO_VALID = 12, S_RHO = 13, S_CURVE = 14,
              S_QUARTER = 15, S_RATIOS = 16;
constexpr int D_SIGMA = 0, D_WEIGHT = 2, D_CURVE = 3, D_SAD = 4, D_CONF_SAD = 5, D_H2 = 6, D_PILOT_H2 = 7,
              D_OFFSET = 8, D_INPUT_OFFSET = 9, D_RHO = 10;

__host__ __device__ constexpr int record_len(int c) { return 3 * c + 26; }
__host__ __device__ constexpr int texture_lane(int channels, int c) {
    return c == 0 ? 2 * channels + 1 : 2 * channels + 3 + 24 + c - 1;
}

// kernels/select.rs:31-46: a float's order-preserving key and back.
__device__ __forceinline__ uint32_t order_key(float v) {
    const uint32_t b = __float_as_uint(v);
    return b >= 0x80000000u ? b ^ 0xFFFFFFFFu : b ^ 0x80000000u;
}
__device__ __forceinline__ float key_value(uint32_t k) {
    return __uint_as_float(k >= 0x80000000u ? k ^ 0x80000000u : k ^ 0xFFFFFFFFu);
}

// ---- temporal stats ---------------------------------------------------------------------------

// The motion field a compensated read follows: (dx, dy) per block of a blocks_x x blocks_y grid at
// `step`, each noise block taking the vector of the motion block covering its origin.
struct StatsMotion {
    const int32_t* field;
    int blocks_x, blocks_y, step;
};

template <int C, bool COMP, bool LF>
__global__ void __launch_bounds__(256) temporal_stats_kernel(const float* __restrict__ next,
                                                             const float* __restrict__ prev, int width, int height,
                                                             StatsMotion motion, float* __restrict__ records) {
    constexpr int L = 2 * C + 1;
    // The lane scratch, then the cell tile; the compensated variant's four variance runs of 256
    // threads each alias the start of it before the lanes are written.
    constexpr int kScratch = 256 * L + 256 > 1024 ? 256 * L + 256 : 1024;
    __shared__ float smem[kScratch];
    __shared__ float cells[16];
    float* scratch = smem;
    float* tile = smem + 256 * L;
    const int t = threadIdx.x, lx = t % kNB, ly = t / kNB;
    const int x0 = blockIdx.x * kNB, y0 = blockIdx.y * kNB;
    const int gx = x0 + lx, gy = y0 + ly;
    const int bw = min(kNB, width - x0), bh = min(kNB, height - y0);
    float* out = records + (static_cast<int64_t>(blockIdx.y) * gridDim.x + blockIdx.x) * record_len(C);
    auto at = [&](int x, int y, int c) { return (static_cast<int64_t>(y) * width + x) * C + c; };

    int sx = 0, sy = 0;
    bool matched = true, moved = false;
    if (COMP) {
        // kernels/stats.rs:224-330: the block follows its vector only when the channel-0 residual
        // variance along it is at most half the zero-vector variance (or nothing of it matches).
        const int col = min(x0 / motion.step, motion.blocks_x - 1), row = min(y0 / motion.step, motion.blocks_y - 1);
        const int vx = motion.field[(row * motion.blocks_x + col) * 2];
        const int vy = motion.field[(row * motion.blocks_x + col) * 2 + 1];
        float zr = 0.0f, vr = 0.0f;
        if (gx < width && gy < height) {
            const float nl = next[at(gx, gy, 0)];
            zr = nl - prev[at(gx, gy, 0)];
            const int mx = gx + vx, my = gy + vy;
            if (mx >= 0 && mx < width && my >= 0 && my < height) vr = nl - prev[at(mx, my, 0)];
        }
        smem[t] = zr;
        smem[256 + t] = zr * zr;
        smem[512 + t] = vr;
        smem[768 + t] = vr * vr;
        __syncthreads();
#pragma unroll
        for (int stride = 128; stride >= 1; stride >>= 1) {
            if (t < stride) {
#pragma unroll
                for (int r = 0; r < 4; ++r) smem[r * 256 + t] += smem[r * 256 + t + stride];
            }
            __syncthreads();
        }
        const float zero_sum = smem[0], zero_sq = smem[256], vec_sum = smem[512], vec_sq = smem[768];
        __syncthreads();
        const int left = x0 + vx, top = y0 + vy, right = left + bw, bottom = top + bh;
        const int ow = max(min(right, width) - max(left, 0), 0), oh = max(min(bottom, height) - max(top, 0), 0);
        const float matched_pixels = static_cast<float>(ow * oh), block_pixels = static_cast<float>(bw * bh);
        const float zero_mean = zero_sum / block_pixels;
        const float zero_var = zero_sq / block_pixels - zero_mean * zero_mean;
        const float safe = fmaxf(matched_pixels, 1.0f);
        const float vec_mean = vec_sum / safe;
        const float vec_var = vec_sq / safe - vec_mean * vec_mean;
        const bool follows = (vx != 0 || vy != 0) && (matched_pixels == 0.0f || vec_var <= 0.5f * zero_var);
        if (follows) {
            sx = vx;
            sy = vy;
            matched = left >= 0 && right <= width && top >= 0 && bottom <= height;
        }
        moved = follows && matched;
    }
    const bool valid = gx < width && gy < height && matched;

    float nv[C], d[C], prev_luma = 0.0f;
#pragma unroll
    for (int c = 0; c < C; ++c) {
        nv[c] = 0.0f;
        d[c] = 0.0f;
        if (valid) {
            nv[c] = next[at(gx, gy, c)];
            const float p = prev[at(gx + sx, gy + sy, c)];
            d[c] = nv[c] - p;
            if (c == 0) prev_luma = p;
        }
        scratch[t * L + c] = d[c];
        scratch[t * L + C + c] = d[c] * d[c];
    }
    __syncthreads();
    // The lag pair never crosses the block's in-frame edge (lx + 1 < bw <= 16 keeps t + 1 in range).
    const float lag = (valid && lx + 1 < bw) ? d[0] * scratch[(t + 1) * L] : 0.0f;
    scratch[t * L + 2 * C] = lag;
    __syncthreads();
    if (t < L) {
        float total = 0.0f;
        for (int i = 0; i < 256; ++i) total += scratch[i * L + t];
        out[t] = total;
    }
    // The moved lane, then the quarter lanes as zero without the luma fields.
    if (t == 2 * C + 2) out[t] = moved ? 1.0f : 0.0f;
    if (!LF && t > 2 * C + 2 && t < 2 * C + 27) out[t] = 0.0f;
#pragma unroll
    for (int c = 0; c < C; ++c) {
        __syncthreads();
        tile[t] = valid ? nv[c] : 0.0f;
        __syncthreads();
        if (t < 16) {
            const int cx = t % 4, cy = t / 4;
            float cell = 0.0f;
#pragma unroll
            for (int dy = 0; dy < 4; ++dy)
#pragma unroll
                for (int dx = 0; dx < 4; ++dx) cell += tile[(4 * cy + dy) * kNB + 4 * cx + dx];
            cells[t] = cell / 16.0f;
        }
        __syncthreads();
        if (t == 0) {
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
            out[texture_lane(C, c)] = pairs ? energy / static_cast<float>(pairs) : 0.0f;
        }
    }
    if constexpr (LF) {
        // kernels/stats.rs:476-606: each quarter's 64 pixels sit at slots quarter * 64 + position
        // and fold in halving rounds of 32..1; an invalid pixel seeds the sum with 0, the minimum
        // with 1e30 and the maximum with -1e30. The flatness averages the pixels' mean of new and
        // previous luma over 2x2 cells of an 8x8 grid, scores each cell's squared difference to its
        // right and lower neighbour inside its quarter, folds each quarter's 16 scores in halving
        // rounds of 8..1 and divides by its 24 pairs.
        __shared__ float qsum[256], qlo[256], qhi[256], qrd[256], qrq[256], qcells[64], qpairs[64];
        const int quarter = (ly / 8) * 2 + lx / 8, qpos = (ly % 8) * 8 + lx % 8, slot = quarter * 64 + qpos;
        qsum[slot] = valid ? nv[0] : 0.0f;
        qlo[slot] = valid ? nv[0] : 1.0e30f;
        qhi[slot] = valid ? nv[0] : -1.0e30f;
        qrd[slot] = d[0];
        qrq[slot] = d[0] * d[0];
        tile[t] = valid ? 0.5f * (nv[0] + prev_luma) : 0.0f;
        __syncthreads();
#pragma unroll
        for (int stride = 32; stride >= 1; stride >>= 1) {
            if (qpos < stride) {
                qsum[slot] += qsum[slot + stride];
                qrd[slot] += qrd[slot + stride];
                qrq[slot] += qrq[slot + stride];
                qlo[slot] = fminf(qlo[slot], qlo[slot + stride]);
                qhi[slot] = fmaxf(qhi[slot], qhi[slot + stride]);
            }
            __syncthreads();
        }
        if (t < 64) {
            const int cy = t / 8, cx = t % 8;
            float cell = 0.0f;
#pragma unroll
            for (int dy = 0; dy < 2; ++dy)
#pragma unroll
                for (int dx = 0; dx < 2; ++dx) cell += tile[(2 * cy + dy) * kNB + 2 * cx + dx];
            qcells[t] = cell / 4.0f;
        }
        __syncthreads();
        if (t < 64) {
            const int cy = t / 8, cx = t % 8;
            const float here = qcells[t];
            float energy = 0.0f;
            if (cx % 4 != 3) {
                const float s = here - qcells[t + 1];
                energy += s * s;
            }
            if (cy % 4 != 3) {
                const float s = here - qcells[t + 8];
                energy += s * s;
            }
            qpairs[((cy / 4) * 2 + cx / 4) * 16 + (cy % 4) * 4 + cx % 4] = energy;
        }
        __syncthreads();
#pragma unroll
        for (int stride = 8; stride >= 1; stride >>= 1) {
            if (t < 64 && t % 16 < stride) qpairs[t] += qpairs[t + stride];
            __syncthreads();
        }
        if (qpos == 0) {
            float* f = out + 2 * C + kQuarterBase + quarter * kQuarterFields;
            const bool full = bw >= (quarter % 2 + 1) * 8 && bh >= (quarter / 2 + 1) * 8;
            // An unmatched block reads as no measurable noise: its seeds and sentinel give way to zeros.
            f[Q_SUM_D] = matched ? qrd[slot] : 0.0f;
            f[Q_SUM_D2] = matched ? qrq[slot] : 0.0f;
            f[Q_LUMA_SUM] = matched ? qsum[slot] : 0.0f;
            f[Q_FLATNESS] = matched ? (full ? qpairs[quarter * 16] / 24.0f : kUnmeasuredFlatness) : 0.0f;
            f[Q_LUMA_MIN] = matched ? qlo[slot] : 0.0f;
            f[Q_LUMA_MAX] = matched ? qhi[slot] : 0.0f;
        }
    }
}

// ---- the reading ------------------------------------------------------------------------------

// The per-block values the reading works from (global scratch, one array per field), then one
// sigma and one tag per 8x8 quarter for the noise curve.
struct BlockScratch {
    float* sigma[kNoiseChannels];
    float* texture[kNoiseChannels];
    float* mean0;
    float* var0;
    float* mean_lag;
    float* pairs;
    float* rho;
    uint32_t* flags;  // per channel: bit 0 candidate, bit 1 measurable, bit 2 kept, bit 3 accepted; bit 8 moved,
                      // bit 9 has_rho
    float* quarter_sigma;
    uint32_t* quarter_tag;  // bit 8: in the static quarter set; bits 0-7: its luma bin, or kNoBin
};

constexpr uint32_t kNoBin = 0xFFu, kQuarterMember = 0x100u;
constexpr int kBinQueries = 2 * kCurveBins;

enum SetKind : int { kSetReference, kSetTexture, kSetKept, kSetRho, kSetQuarter };

struct ReadingShared {
    uint32_t hist[kBinQueries][256];
    uint32_t prefix[kBinQueries], rank[kBinQueries];
    uint32_t ref_n[kNoiseChannels], excl_n[kNoiseChannels], tex_n[kNoiseChannels], kept_n[kNoiseChannels],
        acc_n[kNoiseChannels], rho_n;
    uint32_t ref_min[kNoiseChannels], ref_max[kNoiseChannels];
    float ceiling[kNoiseChannels], threshold[kNoiseChannels];
    uint32_t trusted[kNoiseChannels];
    uint32_t result[kBinQueries];
    uint32_t quarter_n, bin_n[kCurveBins];
};

__device__ __forceinline__ uint32_t set_key(const BlockScratch& s, int kind, int c, int i) {
    if (kind == kSetQuarter)
        return (s.quarter_tag[i] & kQuarterMember) ? order_key(s.quarter_sigma[i]) : kExcluded;
    const uint32_t f = s.flags[i] >> (4 * c);
    switch (kind) {
        case kSetReference: return ((f & 3u) == 3u) ? order_key(s.sigma[c][i]) : kExcluded;
        case kSetTexture:
            return ((f & 3u) == 3u && (s.flags[i] & 0x100u)) ? order_key(s.texture[c][i]) : kExcluded;
        case kSetKept: return (f & 4u) ? order_key(s.sigma[c][i]) : kExcluded;
        default: return (s.flags[i] & 0x200u) ? order_key(s.rho[i]) : kExcluded;
    }
}

// Exact order statistics by four 8-bit radix passes: query q asks for the element of rank
// sh.rank[q] among the elements that `element(i, key, first)` assigns to it (element i joins queries
// first..first+span-1 with `key`, or none when it returns false). One histogram per query, one warp
// scanning each query's histogram; sh.result[q] receives the key. Lanes of a warp that add to the
// same histogram word add once, by their count: the keys of one set share their top bits, so plain
// shared atomics would serialise on a few words.
template <typename Element>
__device__ void radix_select(int n, int nq, int span, ReadingShared& sh, Element element) {
    const int t = threadIdx.x;
    if (t < nq) sh.prefix[t] = 0;
    uint32_t mask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int i = t; i < nq * 256; i += blockDim.x) (&sh.hist[0][0])[i] = 0;
        __syncthreads();
        for (int base = 0; base < n; base += blockDim.x) {
            const int i = base + t;
            uint32_t key = 0;
            int first = 0;
            const bool in = i < n && element(i, key, first);
            for (int k = 0; k < span; ++k) {
                const int q = first + k;
                const bool hit = in && (key & mask) == sh.prefix[q];
                const uint32_t word = hit ? static_cast<uint32_t>(q) * 256u + ((key >> shift) & 0xFFu) : 0xFFFFFFFFu;
                const uint32_t peers = __match_any_sync(0xFFFFFFFFu, word);
                if (hit && (t & 31) == __ffs(peers) - 1)
                    atomicAdd(&sh.hist[0][0] + word, static_cast<uint32_t>(__popc(peers)));
            }
        }
        __syncthreads();
        const int warp = t / 32, lane = t % 32;
        for (int q = warp; q < nq; q += blockDim.x / 32) {
            const uint32_t* h = sh.hist[q];
            uint32_t mine = 0;
            for (int b = 0; b < 8; ++b) mine += h[lane * 8 + b];
            uint32_t incl = mine;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                if (lane >= o) incl += v;
            }
            const uint32_t below = incl - mine, rank = sh.rank[q];
            if (rank >= below && rank < incl) {
                uint32_t seen = below, b = 0;
                for (; b < 8; ++b) {
                    if (rank < seen + h[lane * 8 + b]) break;
                    seen += h[lane * 8 + b];
                }
                sh.prefix[q] |= static_cast<uint32_t>(lane * 8 + b) << shift;
                sh.rank[q] = rank - seen;
            }
        }
        mask |= 0xFFu << shift;
        __syncthreads();
    }
    if (t < nq) sh.result[t] = sh.prefix[t];
    __syncthreads();
}

// The keys of ranks[0..nq) among one set's elements (all ranks below the set's count).
__device__ void select_ranks(const BlockScratch& s, int kind, int c, int n, const uint32_t* ranks, int nq,
                             ReadingShared& sh) {
    if (static_cast<int>(threadIdx.x) < nq) sh.rank[threadIdx.x] = ranks[threadIdx.x];
    radix_select(n, nq, nq, sh, [&](int i, uint32_t& key, int& first) {
        key = set_key(s, kind, c, i);
        first = 0;
        return key != kExcluded;
    });
}

__device__ __forceinline__ float quartile_from_pair(float low, float high, uint32_t count) {
    const uint32_t last = max(count, 1u) - 1u;
    const float fraction = static_cast<float>(last % 4u) * 0.25f;
    return low + fraction * (high - low);
}
__device__ __forceinline__ float median_from_pair(float low, float high) { return (low + high) * 0.5f; }

// The median pair and quartile pair of a set of n elements (all four zero for an empty set).
__device__ void set_pairs(const BlockScratch& s, int kind, int c, int nb, uint32_t n, float out[4],
                          ReadingShared& sh) {
    if (n == 0) {
        out[0] = out[1] = out[2] = out[3] = 0.0f;
        return;
    }
    const uint32_t ranks[4] = {(n - 1) / 2, n / 2, (n - 1) / 4, (n + 2) / 4};
    select_ranks(s, kind, c, nb, ranks, 4, sh);
    for (int q = 0; q < 4; ++q) out[q] = key_value(sh.result[q]);
    __syncthreads();
}

// kernels/sample.rs:95-104 (`static_quarter_sigma`) and kernels/curve.rs:93-133: quarter q of block
// i's sigma, whether it passes the static gates and, if it also lies flat and unclipped, its bin.
struct QuarterRead {
    float sigma;
    bool passes;
    uint32_t bin;
};

__device__ QuarterRead read_quarter(const float* r, int C, int bw, int bh, int q, float flat_limit) {
    const int qw = min(max(bw - (q % 2) * 8, 0), 8), qh = min(max(bh - (q / 2) * 8, 0), 8);
    const float pixels = static_cast<float>(qw * qh);
    const float* f = r + 2 * C + kQuarterBase + q * kQuarterFields;
    const float divisor = pixels > 0.0f ? pixels : 1.0f;
    const float mean = f[Q_SUM_D] / divisor;
    const float ms = f[Q_SUM_D2] / divisor;
    QuarterRead out;
    out.sigma = sqrtf(fmaxf(ms - mean * mean, 0.0f)) / kSqrt2;
    out.passes = pixels > 0.0f && fabsf(mean) < kQuarterStaticGate && out.sigma > kRhoSigmaGate;
    const float mean_luma = f[Q_LUMA_SUM] / divisor;
    const float scaled = fmaxf(mean_luma * static_cast<float>(kCurveBins), 0.0f);
    const uint32_t bin = static_cast<uint32_t>(fminf(scaled, static_cast<float>(kCurveBins - 1)));
    const bool textured = f[Q_FLATNESS] > flat_limit;
    const bool clipped = f[Q_LUMA_MIN] < kClipLow || f[Q_LUMA_MAX] > kClipHigh;
    out.bin = (textured || clipped) ? kNoBin : bin;
    return out;
}

template <int C>
__global__ void __launch_bounds__(kReadingThreads) noise_reading_kernel(const float* __restrict__ records, int width,
                                                                       int height, BlockScratch s, uint32_t min_accepted,
                                                                       bool curve, float* __restrict__ reading) {
    __shared__ ReadingShared sh;
    const int t = threadIdx.x;
    const int bxn = (width + kNB - 1) / kNB, byn = (height + kNB - 1) / kNB, nb = bxn * byn;
    if (t < kNoiseChannels) {
        sh.ref_n[t] = sh.excl_n[t] = sh.tex_n[t] = sh.kept_n[t] = sh.acc_n[t] = 0;
        sh.ref_min[t] = 0xFFFFFFFFu;
        sh.ref_max[t] = 0u;
    }
    if (t == 0) sh.rho_n = 0;
    __syncthreads();

    // Block derive (sample.rs:143-276).
    for (int i = t; i < nb; i += blockDim.x) {
        const int bx = i % bxn, by = i / bxn;
        const int bw = min(kNB, width - bx * kNB), bh = min(kNB, height - by * kNB);
        const float pixels = static_cast<float>(bw * bh), pairs = static_cast<float>(bh * (bw - 1));
        const float* r = records + static_cast<int64_t>(i) * record_len(C);
        const bool moved = r[2 * C + 2] != 0.0f;
        uint32_t flags = moved ? 0x100u : 0u;
#pragma unroll
        for (int c = 0; c < C; ++c) {
            const float mean = r[c] / pixels;
            const float ms = r[C + c] / pixels;
            const float var = fmaxf(ms - mean * mean, 0.0f);
            const float sigma = sqrtf(var) / kSqrt2;
            const bool candidate = fabsf(mean) < kStaticGate;
            const bool measurable = sigma > kRhoSigmaGate;
            s.sigma[c][i] = sigma;
            s.texture[c][i] = r[texture_lane(C, c)];
            flags |= ((candidate ? 1u : 0u) | (measurable ? 2u : 0u)) << (4 * c);
            if (candidate && measurable) {
                atomicAdd(&sh.ref_n[c], 1u);
                const uint32_t k = order_key(sigma);
                atomicMin(&sh.ref_min[c], k);
                atomicMax(&sh.ref_max[c], k);
                if (moved) atomicAdd(&sh.tex_n[c], 1u);
            } else if (candidate) {
                atomicAdd(&sh.excl_n[c], 1u);
            }
            if (c == 0) {
                s.mean0[i] = mean;
                s.var0[i] = var;
            }
        }
        s.pairs[i] = pairs;
        s.mean_lag[i] = pairs > 0.0f ? r[2 * C] / pairs : 0.0f;
        s.flags[i] = flags;
    }
    __threadfence_block();
    __syncthreads();

    // The outlier ceilings and moved-texture thresholds (sample.rs:310-360).
    for (int c = 0; c < C; ++c) {
        const uint32_t n = sh.ref_n[c];
        float ql = 0.0f, qh = 0.0f;
        if (n > 0) {
            const uint32_t ranks[2] = {(n - 1) / 4, (n + 2) / 4};
            select_ranks(s, kSetReference, c, nb, ranks, 2, sh);
            ql = key_value(sh.result[0]);
            qh = key_value(sh.result[1]);
        }
        float threshold = 0.0f;
        const uint32_t tn = sh.tex_n[c];
        if (tn > 0) {
            const uint32_t ranks[1] = {(tn - 1) * 2 / 5};
            select_ranks(s, kSetTexture, c, nb, ranks, 1, sh);
            threshold = key_value(sh.result[0]);
        }
        if (t == 0) {
            const float q = quartile_from_pair(ql, qh, n);
            sh.ceiling[c] = n > 0 ? q * kOutlierFactor : 0.0f;
            const bool spread = n > 0 && key_value(sh.ref_max[c]) > key_value(sh.ref_min[c]);
            sh.trusted[c] = (sh.excl_n[c] == 0 || spread) ? 1u : 0u;
            sh.threshold[c] = threshold;
        }
        __syncthreads();
    }

    // Block accept (sample.rs:362-500).
    for (int i = t; i < nb; i += blockDim.x) {
        uint32_t flags = s.flags[i];
        const bool moved = flags & 0x100u;
        bool accepted0 = false;
#pragma unroll
        for (int c = 0; c < C; ++c) {
            const float sigma = s.sigma[c][i];
            const bool candidate = (flags >> (4 * c)) & 1u;
            const bool acc = sh.trusted[c] && candidate && sigma <= sh.ceiling[c] && sigma > kRhoSigmaGate;
            const bool textured = moved && sh.tex_n[c] > 0 && s.texture[c][i] > sh.threshold[c];
            if (acc) {
                flags |= 8u << (4 * c);
                atomicAdd(&sh.acc_n[c], 1u);
            }
            if (acc && !textured) {
                flags |= 4u << (4 * c);
                atomicAdd(&sh.kept_n[c], 1u);
            }
            if (c == 0) accepted0 = acc;
        }
        const bool has_rho = accepted0 && s.pairs[i] > 0.0f;
        const float variance = has_rho ? s.var0[i] : 1.0f;
        const float mean0 = s.mean0[i];
        const float rho = (s.mean_lag[i] - mean0 * mean0) / variance;
        if (has_rho) {
            flags |= 0x200u;
            s.rho[i] = fminf(fmaxf(rho, 0.0f), 1.0f);
            atomicAdd(&sh.rho_n, 1u);
        }
        s.flags[i] = flags;
    }
    __threadfence_block();
    __syncthreads();

    // The sample (sample.rs:562-710).
    float kept[kNoiseChannels][4] = {};
    for (int c = 0; c < C; ++c) set_pairs(s, kSetKept, c, nb, sh.kept_n[c], kept[c], sh);
    float rho_pair[4];
    set_pairs(s, kSetRho, 0, nb, sh.rho_n, rho_pair, sh);

    // The noise curve (kernels/sample.rs:482-510, kernels/curve.rs:37-133, sample.rs:717-803): the
    // quarters of channel-0 accepted blocks that pass the static gates form the quarter set; those
    // that are also flat (against a gate from channel 0's kept sigma median) and unclipped join the
    // bin of their mean luma. The set's median and each bin's median are exact selects.
    float quarter_median = 0.0f;
    float bin_median[kCurveBins];
    if (curve) {
        const float sigma_median = median_from_pair(kept[0][0], kept[0][1]);
        const float flat_limit = fmaxf(kFlatFactor * sigma_median * sigma_median, kFlatFloor);
        if (t < kCurveBins) sh.bin_n[t] = 0;
        if (t == 0) sh.quarter_n = 0;
        __syncthreads();
        const int nq = 4 * nb;
        for (int base = 0; base < nq; base += blockDim.x) {
            const int i = base + t;
            uint32_t tag = kNoBin;
            if (i < nq) {
                const int blk = i / 4, bx = blk % bxn, by = blk / bxn;
                const int bw = min(kNB, width - bx * kNB), bh = min(kNB, height - by * kNB);
                const QuarterRead qr =
                    read_quarter(records + static_cast<int64_t>(blk) * record_len(C), C, bw, bh, i % 4, flat_limit);
                if (qr.passes && (s.flags[blk] & 8u)) tag = kQuarterMember | qr.bin;
                s.quarter_sigma[i] = qr.sigma;
                s.quarter_tag[i] = tag;
            }
            const uint32_t members = __ballot_sync(0xFFFFFFFFu, tag & kQuarterMember);
            if ((t & 31) == 0 && members) atomicAdd(&sh.quarter_n, static_cast<uint32_t>(__popc(members)));
            const uint32_t bin = tag & 0xFFu;
            const uint32_t peers = __match_any_sync(0xFFFFFFFFu, bin);
            if (bin < kCurveBins && (t & 31) == __ffs(peers) - 1)
                atomicAdd(&sh.bin_n[bin], static_cast<uint32_t>(__popc(peers)));
        }
        __threadfence_block();
        __syncthreads();
        const uint32_t qn = sh.quarter_n;
        if (qn > 0) {
            const uint32_t ranks[2] = {(qn - 1) / 2, qn / 2};
            select_ranks(s, kSetQuarter, 0, nq, ranks, 2, sh);
            quarter_median = median_from_pair(key_value(sh.result[0]), key_value(sh.result[1]));
        }
        // Queries 2b and 2b + 1 are bin b's lower and upper median.
        if (t < kBinQueries) {
            const uint32_t n = sh.bin_n[t / 2];
            sh.rank[t] = n == 0 ? 0 : ((t % 2) ? n / 2 : (n - 1) / 2);
        }
        radix_select(nq, kBinQueries, 2, sh, [&](int i, uint32_t& key, int& first) {
            const uint32_t tag = s.quarter_tag[i];
            const uint32_t bin = tag & 0xFFu;
            if (!(tag & kQuarterMember) || bin >= static_cast<uint32_t>(kCurveBins)) return false;
            key = order_key(s.quarter_sigma[i]);
            first = static_cast<int>(2 * bin);
            return true;
        });
        for (int b = 0; b < kCurveBins; ++b)
            bin_median[b] = sh.bin_n[b] ? median_from_pair(key_value(sh.result[2 * b]), key_value(sh.result[2 * b + 1]))
                                        : 0.0f;
    }

    if (t == 0) {
        auto channel_valid = [&](int c) { return c < C && sh.acc_n[c] >= min_accepted && sh.kept_n[c] > 0; };
        const bool valid0 = sh.rho_n > 0 && channel_valid(0);
        const float static_fraction = static_cast<float>(sh.acc_n[0]) / static_cast<float>(nb);
        for (int c = 0; c < kNoiseChannels; ++c) {
            const bool k = c == 0 ? valid0 : channel_valid(c);
            const float sigma = median_from_pair(kept[c][0], kept[c][1]);
            const float low = quartile_from_pair(kept[c][2], kept[c][3], c < C ? sh.kept_n[c] : 0u);
            reading[R_VALID + c] = k ? 1.0f : 0.0f;
            reading[R_SIGMA + c] = k ? sigma : 0.0f;
            reading[R_SIGMA_LOW + c] = k ? low : 0.0f;
        }
        reading[R_RHO] = valid0 ? median_from_pair(rho_pair[0], rho_pair[1]) : 0.0f;
        reading[R_STATIC] = valid0 ? static_fraction : 0.0f;
        reading[R_ACCEPTED] = static_cast<float>(sh.acc_n[0]);
        if (!curve) {
            for (int w = R_ACCEPTED + 1; w < kReadingWords; ++w) reading[w] = 0.0f;
        } else {
            // curve_bin_sigma (sample.rs:747-803): flat before the first and past the last populated
            // bin, linear between the nearest populated bin below and the nearest at or above.
            uint32_t populated = 0;
            int first_index = 0, last_index = 0;
            float first_sigma = 0.0f, last_sigma = 0.0f;
            for (int b = 0; b < kCurveBins; ++b) {
                if (sh.bin_n[b] < kMinBinQuarters) continue;
                if (populated == 0) {
                    first_index = b;
                    first_sigma = bin_median[b];
                }
                last_index = b;
                last_sigma = bin_median[b];
                ++populated;
            }
            const bool curve_valid =
                valid0 && sh.quarter_n > 0 && quarter_median > 0.0f && populated >= kMinPopulatedBins;
            const float divisor = curve_valid ? quarter_median : 1.0f;
            for (int bin = 0; bin < kCurveBins; ++bin) {
                int low_index = 0, high_index = 0;
                float low_sigma = 0.0f, high_sigma = 0.0f;
                bool has_high = false;
                for (int b = 0; b < kCurveBins; ++b) {
                    if (sh.bin_n[b] < kMinBinQuarters) continue;
                    if (b < bin) {
                        low_index = b;
                        low_sigma = bin_median[b];
                    }
                    if (b >= bin && !has_high) {
                        high_index = b;
                        high_sigma = bin_median[b];
                        has_high = true;
                    }
                }
                const int span_bins = high_index > low_index ? high_index - low_index : 1;
                const int offset_bins = bin - min(low_index, bin);
                const float fraction = static_cast<float>(offset_bins) / static_cast<float>(span_bins);
                const float between = low_sigma + (high_sigma - low_sigma) * fraction;
                const float sigma = bin <= first_index ? first_sigma : (bin >= last_index ? last_sigma : between);
                reading[R_RATIOS + bin] = curve_valid ? sigma / divisor : 0.0f;
            }
            reading[R_CURVE_VALID] = curve_valid ? 1.0f : 0.0f;
            reading[R_QUARTER_MEDIAN] = curve_valid ? quarter_median : 0.0f;
            reading[R_POPULATED] = static_cast<float>(populated);
        }
    }
}

// A reading without temporal stats: the Immerkaer words (already written) and zeros.
__global__ void spatial_reading_kernel(float* __restrict__ reading) {
    const int w = threadIdx.x + 2;
    if (w < kReadingWords) reading[w] = 0.0f;
}

// ---- the window fold --------------------------------------------------------------------------

__device__ float fold_correlation_factor(float rho, const float* settings) {
    const float r0 = 0.0f, r1 = 0.3f, r2 = 0.5f, r3 = 0.65f;
    const float a0 = 1.0f, a1 = 1.05f, a2 = 1.25f, a3 = 1.45f;
    const float x = fminf(fmaxf(rho, r0), r3);
    const float f0 = (x - r0) * settings[F_SEG];
    const float f1 = (x - r1) * settings[F_SEG + 1];
    const float f2 = (x - r2) * settings[F_SEG + 2];
    const float first = a0 + f0 * (a1 - a0);
    const float second = a1 + f1 * (a2 - a1);
    const float third = a2 + f2 * (a3 - a2);
    const float later = x <= r2 ? second : third;
    return x <= r1 ? first : later;
}

// exp and ln in double precision, rounded to float, as the oracle evaluates them.
__device__ float spatial_offset_factor(int dx, int dy, float rho) {
    const int sq = dx * dx + dy * dy;
    if (sq == 0) return 0.0f;
    if (rho <= 0.0f) return 1.0f;
    const float distance = sqrtf(static_cast<float>(sq));
    const float log_rho = static_cast<float>(log(static_cast<double>(rho)));
    const float shared = static_cast<float>(exp(static_cast<double>(distance * log_rho)));
    return 1.0f - shared;
}

__device__ float sorted_median(float* v, int n) {
    for (int i = 1; i < n; ++i) {
        const float key = v[i];
        int p = i;
        while (p > 0 && v[p - 1] > key) {
            v[p] = v[p - 1];
            --p;
        }
        v[p] = key;
    }
    return n > 0 ? (v[(n - 1) / 2] + v[n / 2]) * 0.5f : 0.0f;
}

__global__ void __launch_bounds__(256) noise_fold_kernel(const float* __restrict__ records,
                                                         const float* __restrict__ results, int capacity, int first,
                                                         int last, const float* __restrict__ settings, int channels,
                                                         int table_radius, float* __restrict__ state,
                                                         float* __restrict__ derived, float* __restrict__ spatial,
                                                         float* __restrict__ pilot) {
    __shared__ float medians[26];
    __shared__ float inputs[3];
    const int t = threadIdx.x;
    auto rec = [&](int frame) { return records + static_cast<int64_t>(frame % capacity) * kReadingWords; };
    auto has_sample = [&](int frame, int c) { return rec(frame)[R_VALID + c] != 0.0f; };
    auto has_curve = [&](int frame) { return rec(frame)[R_CURVE_VALID] != 0.0f; };
    if (t < 26) {
        float v[17];
        int n = 0;
        if (t < 8) {
            const int chain = t / 2, c = t % 2;
            float m = 0.0f;
            if (c < channels) {
                const float sigma_scale = settings[F_SIGMA_SCALE], imm_factor = settings[F_IMM];
                for (int f = first; f <= last; ++f) {
                    if (chain == 3 && !has_sample(f, c)) continue;
                    const float* r = rec(f);
                    const bool has = has_sample(f, c);
                    const float factor = fold_correlation_factor(r[R_RHO], settings);
                    const float immerkaer = imm_factor * results[static_cast<int64_t>(f % capacity) * 2 + c];
                    const float imm_low = r[c], sigma = r[R_SIGMA + c], sigma_low = r[R_SIGMA_LOW + c];
                    float x;
                    if (chain == 0) x = (has ? fmaxf(immerkaer, sigma * factor) : immerkaer) * sigma_scale;
                    else if (chain == 1) x = (has ? fmaxf(imm_low, sigma_low * factor) : imm_low) * sigma_scale;
                    else if (chain == 2) x = (has ? fmaxf(imm_low, sigma_low) : imm_low) * sigma_scale;
                    else x = sigma * sigma_scale;
                    v[n++] = x;
                }
                const float med = sorted_median(v, n);
                m = n > 0 ? fmaxf(med, kSigmaFloor) : 0.0f;
            }
            medians[t] = m;
        } else {
            const int word = t == 8 ? R_RHO : (t == 9 ? R_QUARTER_MEDIAN : R_RATIOS + t - 10);
            const bool curve_gate = t != 8;
            for (int f = first; f <= last; ++f)
                if (has_sample(f, 0) && (!curve_gate || has_curve(f))) v[n++] = rec(f)[word];
            medians[t] = sorted_median(v, n);
        }
    }
    __syncthreads();
    if (t == 0) {
        uint32_t sampled = 0, curved = 0;
        for (int f = first; f <= last; ++f) {
            sampled += has_sample(f, 0) ? 1u : 0u;
            curved += (has_sample(f, 0) && has_curve(f)) ? 1u : 0u;
        }
        const bool curve_present = sampled > 0 && 2 * curved >= sampled;
        uint32_t mask = sampled > 0 ? 1u : 0u;
        for (int c = 1; c < channels; ++c) {
            bool any = false;
            for (int f = first; f <= last; ++f) any = any || has_sample(f, c);
            if (any) mask |= 1u << c;
        }
        const bool rho_valid = mask & 1u, any_sampled = mask != 0;
        for (int c = 0; c < kNoiseChannels; ++c) {
            const bool sampled_c = mask & (1u << c);
            const float unb = medians[4 + c], temporal = medians[6 + c];
            state[S_MEDIAN + 1 + c] = medians[c];
            state[S_LOW + 1 + c] = medians[2 + c];
            state[S_LOW_UNB + 1 + c] = unb;
            state[S_TEMPORAL + 1 + c] = sampled_c ? temporal : (any_sampled ? unb : 0.0f);
            derived[D_SIGMA + c] = sampled_c ? temporal : unb;
        }
        float median_sum = 0.0f, low_sum = 0.0f;
        for (int c = 0; c < channels; ++c) {
            median_sum += medians[c] * medians[c];
            low_sum += medians[2 + c] * medians[2 + c];
        }
        const float rho = rho_valid ? medians[8] : 0.0f;
        state[S_MEDIAN] = 1.0f;
        state[S_LOW] = 1.0f;
        state[S_LOW_UNB] = 1.0f;
        state[S_TEMPORAL] = any_sampled ? 1.0f : 0.0f;
        state[S_RHO_VALID] = rho_valid ? 1.0f : 0.0f;
        state[S_RHO] = rho;
        state[S_CURVE] = curve_present ? 1.0f : 0.0f;
        state[S_QUARTER] = curve_present ? medians[9] : 0.0f;
        const bool curve_valid = curve_present && settings[F_CURVE_APPLIES] != 0.0f;
        for (int b = 0; b < 16; ++b) state[S_RATIOS + b] = curve_present ? medians[10 + b] : 0.0f;
        const float sigma0 = derived[D_SIGMA];
        const float g_max = settings[F_G_MAX], floor = settings[F_W_FLOOR];
        const float norm = sigma0 * sigma0 * g_max * g_max;
        const bool usable = isfinite(norm) && norm > floor;
        const float h2_measured = settings[F_H2_PIV] * static_cast<float>(channels) / median_sum;
        const float h2 = settings[F_H2_AUTO] != 0.0f ? h2_measured : settings[F_H2_FIXED];
        const float input_offset = settings[F_OFFSET_PV] * low_sum;
        const float noise_offset = settings[F_MAIN_OFFSET] != 0.0f ? input_offset : 0.0f;
        derived[D_WEIGHT] = usable ? norm : floor;
        derived[D_CURVE] = curve_valid ? 1.0f : 0.0f;
        derived[D_SAD] = settings[F_SAD] * medians[0];
        derived[D_CONF_SAD] = settings[F_CONF_SAD] * medians[0];
        derived[D_H2] = h2;
        derived[D_PILOT_H2] = h2 * settings[F_PILOT];
        derived[D_OFFSET] = noise_offset;
        derived[D_INPUT_OFFSET] = input_offset;
        derived[D_RHO] = rho;
        inputs[0] = noise_offset;
        inputs[1] = input_offset;
        inputs[2] = rho;
    }
    __syncthreads();
    if (table_radius > 0) {
        const int side = 2 * table_radius + 1;
        for (int i = t; i < side * side; i += blockDim.x) {
            const int dx = i % side - table_radius, dy = i / side - table_radius;
            spatial[i] = inputs[0] * spatial_offset_factor(dx, dy, inputs[2]);
            pilot[i] = inputs[1] * spatial_offset_factor(dx, dy, 0.0f);
        }
    }
}

}  // namespace

size_t noise_scratch_floats(int width, int height) {
    const size_t nb = static_cast<size_t>((width + kNB - 1) / kNB) * ((height + kNB - 1) / kNB);
    return nb * 18;  // sigma x2, texture x2, mean0, var0, mean_lag, pairs, rho, flags; 4 quarter sigmas, 4 tags
}

size_t noise_records_floats(int width, int height, int channels) {
    return static_cast<size_t>((width + kNB - 1) / kNB) * ((height + kNB - 1) / kNB) * record_len(channels);
}

cudaError_t launch_temporal_stats(const float* next, const float* prev, int channels, int width, int height,
                                  const int32_t* mv_field, int mv_blocks_x, int mv_blocks_y, int mv_step,
                                  bool luma_fields, float* records, cudaStream_t s) {
    if (channels < 1 || channels > 2 || width < 1 || height < 1) return cudaErrorInvalidValue;
    if (mv_field && (mv_blocks_x < 1 || mv_blocks_y < 1 || mv_step < 1)) return cudaErrorInvalidValue;
    dim3 grid((width + kNB - 1) / kNB, (height + kNB - 1) / kNB);
    if (!prev)  // the first frame of a stream has no previous frame: its records are zero
        return cudaMemsetAsync(records, 0, noise_records_floats(width, height, channels) * sizeof(float), s);
    const StatsMotion m{mv_field, mv_blocks_x, mv_blocks_y, mv_step};
    auto run = [&](auto kernel) { kernel<<<grid, 256, 0, s>>>(next, prev, width, height, m, records); };
    const int variant = (channels - 1) * 4 + (mv_field ? 2 : 0) + (luma_fields ? 1 : 0);
    switch (variant) {
        case 0: run(temporal_stats_kernel<1, false, false>); break;
        case 1: run(temporal_stats_kernel<1, false, true>); break;
        case 2: run(temporal_stats_kernel<1, true, false>); break;
        case 3: run(temporal_stats_kernel<1, true, true>); break;
        case 4: run(temporal_stats_kernel<2, false, false>); break;
        case 5: run(temporal_stats_kernel<2, false, true>); break;
        case 6: run(temporal_stats_kernel<2, true, false>); break;
        default: run(temporal_stats_kernel<2, true, true>); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_noise_reading(const float* records, int channels, int width, int height, float* scratch,
                                 uint32_t min_accepted, bool curve, float* reading, cudaStream_t s) {
    if (channels < 1 || channels > 2 || width < 1 || height < 1) return cudaErrorInvalidValue;
    if (!records) {
        spatial_reading_kernel<<<1, 32, 0, s>>>(reading);
        return cudaGetLastError();
    }
    const size_t nb = static_cast<size_t>((width + kNB - 1) / kNB) * ((height + kNB - 1) / kNB);
    BlockScratch b{};
    b.sigma[0] = scratch;
    b.sigma[1] = scratch + nb;
    b.texture[0] = scratch + 2 * nb;
    b.texture[1] = scratch + 3 * nb;
    b.mean0 = scratch + 4 * nb;
    b.var0 = scratch + 5 * nb;
    b.mean_lag = scratch + 6 * nb;
    b.pairs = scratch + 7 * nb;
    b.rho = scratch + 8 * nb;
    b.flags = reinterpret_cast<uint32_t*>(scratch + 9 * nb);
    b.quarter_sigma = scratch + 10 * nb;
    b.quarter_tag = reinterpret_cast<uint32_t*>(scratch + 14 * nb);
    if (channels == 1)
        noise_reading_kernel<1><<<1, kReadingThreads, 0, s>>>(records, width, height, b, min_accepted, curve, reading);
    else
        noise_reading_kernel<2><<<1, kReadingThreads, 0, s>>>(records, width, height, b, min_accepted, curve, reading);
    return cudaGetLastError();
}

cudaError_t launch_noise_fold(const float* records, const float* results, int capacity, int first, int last,
                              const float* settings, int channels, int table_radius, float* state, float* derived,
                              float* spatial, float* pilot, cudaStream_t s) {
    if (last < first || last - first + 1 > 17 || last - first + 1 > capacity || channels < 1 || channels > 2)
        return cudaErrorInvalidValue;
    noise_fold_kernel<<<1, 256, 0, s>>>(records, results, capacity, first, last, settings, channels, table_radius,
                                        state, derived, spatial, pilot);
    return cudaGetLastError();
}

}  // namespace avd
