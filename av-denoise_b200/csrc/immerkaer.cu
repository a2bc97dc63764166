// Immerkær spatial noise estimate on sm_100a: per-block partial sums of the absolute 3x3 noise
// mask response, the frame totals, and each channel's lower quartile of the per-block sigmas.
//
// Reference behaviour (av-denoise-core/src/noise):
//   kernels/stats.rs:24-94     each interior pixel's response 4c - 2(l + r + u + d) + (diagonals);
//                              a 32x8 block sums |response| per channel, thread 0..255 in order.
//   kernels/stats.rs:96-137    the frame totals: 256 strided partial sums, then summed in order.
//   kernels/sample.rs:181-203  a block's sigma = sqrt(pi/2) * sum / (6 * interior area of the block),
//                              blocks without interior excluded.
//   kernels/sample.rs:108-114, noise/select.rs:78-88
//                              the lower quartile from the elements of rank (n-1)/4 and (n+2)/4,
//                              interpolated by ((n-1) mod 4) / 4 (the host `lower_quartile`).
//
// Design: the partial kernel is one CTA per 32x8 block (a coalesced 32-wide row per warp); the
// quartile kernel is one CTA per channel running an exact 4-pass radix select (8 bits per pass)
// over the blocks' sigma bit patterns (non-negative floats order like their bits), recomputing
// each sigma from the partials on every pass, so no scratch beyond the partials is needed.

#include <cstdint>

#include "kernels.h"

namespace avd {
namespace {

constexpr int kBlockX = 32, kBlockY = 8, kLanes = 2;
constexpr int kSelectThreads = 1024;

template <int C>
__global__ void __launch_bounds__(kBlockX* kBlockY) immerkaer_partial_kernel(const float* __restrict__ frame,
                                                                          float* __restrict__ partials, int width,
                                                                          int height) {
    __shared__ float scratch[kBlockX * kBlockY * kLanes];
    const int x = blockIdx.x * kBlockX + threadIdx.x;
    const int y = blockIdx.y * kBlockY + threadIdx.y;
    const int t = threadIdx.y * kBlockX + threadIdx.x;
    const bool interior = x >= 1 && x < width - 1 && y >= 1 && y < height - 1;
#pragma unroll
    for (int c = 0; c < kLanes; ++c) {
        float r = 0.0f;
        if (c < C && interior) {
            auto at = [&](int dx, int dy) { return frame[(static_cast<int64_t>(y + dy) * width + x + dx) * C + c]; };
            const float cross = __fadd_rn(__fadd_rn(__fadd_rn(at(-1, 0), at(1, 0)), at(0, -1)), at(0, 1));
            const float diag = __fadd_rn(__fadd_rn(__fadd_rn(at(-1, -1), at(1, -1)), at(-1, 1)), at(1, 1));
            r = __fadd_rn(__fsub_rn(__fmul_rn(at(0, 0), 4.0f), __fmul_rn(cross, 2.0f)), diag);
        }
        scratch[t * kLanes + c] = fabsf(r);
    }
    __syncthreads();
    if (t < kLanes) {
        float sum = 0.0f;
        for (int i = 0; i < kBlockX * kBlockY; ++i) sum = __fadd_rn(sum, scratch[i * kLanes + t]);
        partials[(static_cast<int64_t>(blockIdx.y) * gridDim.x + blockIdx.x) * kLanes + t] = sum;
    }
}

__global__ void __launch_bounds__(256) immerkaer_reduce_kernel(const float* __restrict__ partials, int blocks,
                                                            float* __restrict__ results) {
    __shared__ float scratch[256 * kLanes];
    const int t = threadIdx.x;
    float s0 = 0.0f, s1 = 0.0f;
    for (int i = t; i < blocks; i += 256) {
        s0 = __fadd_rn(s0, partials[i * kLanes]);
        s1 = __fadd_rn(s1, partials[i * kLanes + 1]);
    }
    scratch[t * kLanes] = s0;
    scratch[t * kLanes + 1] = s1;
    __syncthreads();
    if (t < kLanes) {
        float total = 0.0f;
        for (int i = 0; i < 256; ++i) total = __fadd_rn(total, scratch[i * kLanes + t]);
        results[t] = total;
    }
}

// The sigma bit pattern of block `i` of channel `c`, or 0xFFFFFFFF for a block with no interior.
__device__ __forceinline__ uint32_t block_key(const float* partials, int i, int c, int cubes_x, int width, int height,
                                              float scale) {
    const int cx = i % cubes_x, cy = i / cubes_x;
    const int x0 = max(cx * kBlockX, 1), y0 = max(cy * kBlockY, 1);
    const int x1 = min(min((cx + 1) * kBlockX, width), width - 1);
    const int y1 = min(min((cy + 1) * kBlockY, height), height - 1);
    if (x1 <= x0 || y1 <= y0) return 0xFFFFFFFFu;
    const float area = static_cast<float>((x1 - x0) * (y1 - y0));
    const float sigma = __fdiv_rn(__fmul_rn(scale, partials[i * kLanes + c]), __fmul_rn(6.0f, area));
    return __float_as_uint(sigma);
}

// The elements of ranks rank[0] and rank[1] (0-based) among the blocks' keys, by one exact radix
// select of two queries: 8-bit digits from the top, one histogram per query, lanes of a warp that
// add to the same histogram word adding once by their count, one warp scanning each histogram.
__device__ void select_two(const float* partials, int blocks, int c, int cubes_x, int width, int height, float scale,
                           uint32_t* rank, uint32_t (*hist)[256], uint32_t* prefix) {
    const int t = threadIdx.x, warp = t / 32, lane = t % 32;
    if (t < 2) prefix[t] = 0;
    uint32_t mask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int b = t; b < 512; b += blockDim.x) (&hist[0][0])[b] = 0;
        __syncthreads();
        for (int base = 0; base < blocks; base += blockDim.x) {
            const int i = base + t;
            const uint32_t key = i < blocks ? block_key(partials, i, c, cubes_x, width, height, scale) : 0xFFFFFFFFu;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const bool hit = key != 0xFFFFFFFFu && (key & mask) == prefix[q];
                const uint32_t word = hit ? static_cast<uint32_t>(q) * 256u + ((key >> shift) & 0xFFu) : 0xFFFFFFFFu;
                const uint32_t peers = __match_any_sync(0xFFFFFFFFu, word);
                if (hit && lane == __ffs(peers) - 1) atomicAdd(&hist[0][0] + word, static_cast<uint32_t>(__popc(peers)));
            }
        }
        __syncthreads();
        if (warp < 2) {
            const uint32_t* h = hist[warp];
            uint32_t mine = 0;
            for (int b = 0; b < 8; ++b) mine += h[lane * 8 + b];
            uint32_t incl = mine;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                if (lane >= o) incl += v;
            }
            const uint32_t below = incl - mine, r = rank[warp];
            if (r >= below && r < incl) {
                uint32_t seen = below, b = 0;
                for (; b < 8; ++b) {
                    if (r < seen + h[lane * 8 + b]) break;
                    seen += h[lane * 8 + b];
                }
                prefix[warp] |= static_cast<uint32_t>(lane * 8 + b) << shift;
                rank[warp] = r - seen;
            }
        }
        mask |= 0xFFu << shift;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kSelectThreads) immerkaer_quartile_kernel(const float* __restrict__ partials,
                                                                         int cubes_x, int cubes_y, int width,
                                                                         int height, int channels, float scale,
                                                                         float* __restrict__ sigma_low) {
    __shared__ uint32_t hist[2][256];
    __shared__ uint32_t prefix[2], rank[2];
    __shared__ uint32_t count_s;
    const int c = blockIdx.x;
    const int blocks = cubes_x * cubes_y;
    if (c >= channels) {
        if (threadIdx.x == 0) sigma_low[c] = 0.0f;
        return;
    }
    if (threadIdx.x == 0) count_s = 0;
    __syncthreads();
    uint32_t mine = 0;
    for (int i = threadIdx.x; i < blocks; i += blockDim.x)
        mine += block_key(partials, i, c, cubes_x, width, height, scale) != 0xFFFFFFFFu ? 1u : 0u;
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xFFFFFFFFu, mine, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&count_s, mine);
    __syncthreads();
    const uint32_t n = count_s;
    if (n == 0) {
        if (threadIdx.x == 0) sigma_low[c] = 0.0f;
        return;
    }
    if (threadIdx.x == 0) {
        rank[0] = (n - 1) / 4;
        rank[1] = (n + 2) / 4;
    }
    __syncthreads();
    select_two(partials, blocks, c, cubes_x, width, height, scale, rank, hist, prefix);
    if (threadIdx.x == 0) {
        const float low = __uint_as_float(prefix[0]), high = __uint_as_float(prefix[1]);
        const float fraction = __fmul_rn(static_cast<float>((n - 1) % 4), 0.25f);
        sigma_low[c] = __fadd_rn(low, __fmul_rn(fraction, __fsub_rn(high, low)));
    }
}

}  // namespace

size_t immerkaer_partials_len(int width, int height) {
    return static_cast<size_t>((width + kBlockX - 1) / kBlockX) * ((height + kBlockY - 1) / kBlockY) * kLanes;
}

cudaError_t launch_immerkaer(const float* frame, int channels, int width, int height, float scale, float* partials,
                             float* results, float* sigma_low, cudaStream_t s) {
    if (channels < 1 || channels > 2 || width < 1 || height < 1) return cudaErrorInvalidValue;
    const int cubes_x = (width + kBlockX - 1) / kBlockX, cubes_y = (height + kBlockY - 1) / kBlockY;
    dim3 grid(cubes_x, cubes_y), block(kBlockX, kBlockY);
    if (channels == 1)
        immerkaer_partial_kernel<1><<<grid, block, 0, s>>>(frame, partials, width, height);
    else
        immerkaer_partial_kernel<2><<<grid, block, 0, s>>>(frame, partials, width, height);
    if (results) immerkaer_reduce_kernel<<<1, 256, 0, s>>>(partials, cubes_x * cubes_y, results);
    if (sigma_low)
        immerkaer_quartile_kernel<<<kLanes, kSelectThreads, 0, s>>>(partials, cubes_x, cubes_y, width, height,
                                                                   channels, scale, sigma_low);
    return cudaGetLastError();
}

}  // namespace avd
