// Frame ingest and egress between caller planes and the engine's f32 ring.
//
// HBM-bound byte work: each thread owns one 32-bit word of the caller plane (4 u8 or 2 u16
// samples), so loads and stores are coalesced 32-bit accesses and no two threads share a word.

#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.h"

namespace avd {

namespace {

constexpr int kBlock = 256;

int grid_for(int64_t items) {
    int64_t g = (items + kBlock - 1) / kBlock;
    // Grid-stride loops cover the rest; 148 SMs x 16 resident 256-thread blocks.
    return static_cast<int>(g < 148 * 16 ? (g > 0 ? g : 1) : 148 * 16);
}

// av-denoise-core/src/engine/kernels.rs:25-63: `ring = f32(code) / max`, a correctly rounded
// division (not a reciprocal multiply).
template <int SPW, int C>
__global__ void ingest_words_kernel(const uint32_t* __restrict__ p0, const uint32_t* __restrict__ p1,
                                    float* __restrict__ slot, int64_t pixels, float max_value) {
    constexpr uint32_t kBits = 32 / SPW;
    constexpr uint32_t kMask = (1u << kBits) - 1u;
    const int64_t words = (pixels + SPW - 1) / SPW;
    for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < words; w += (int64_t)gridDim.x * blockDim.x) {
        uint32_t w0 = __ldg(p0 + w);
        uint32_t w1 = C > 1 ? __ldg(p1 + w) : 0u;
#pragma unroll
        for (int lane = 0; lane < SPW; ++lane) {
            int64_t p = w * SPW + lane;
            if (p >= pixels) break;
            uint32_t c0 = (w0 >> (lane * kBits)) & kMask;
            slot[p * C] = __fdiv_rn(static_cast<float>(c0), max_value);
            if (C > 1) {
                uint32_t c1 = (w1 >> (lane * kBits)) & kMask;
                slot[p * C + 1] = __fdiv_rn(static_cast<float>(c1), max_value);
            }
        }
    }
}

// Many frames of mixed depth and size in one launch (no counterpart in the reference, which ingests
// one frame per launch): each thread takes global words, finds its frame by a binary search of the
// word prefix, and converts as ingest_words_kernel does, the same correctly rounded division.
__global__ void batch_ingest_kernel(const BatchIngestItem* __restrict__ items, const int64_t* __restrict__ prefix,
                                    int n, int64_t total) {
    for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < total; w += (int64_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = n - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(prefix + mid) <= w) lo = mid;
            else hi = mid - 1;
        }
        const BatchIngestItem& it = items[lo];
        const int64_t local = w - __ldg(prefix + lo);
        const int spw = it.samples_per_word, bits = 32 / spw;
        const uint32_t mask = (1u << bits) - 1u;
        const uint32_t w0 = __ldg(it.plane0 + local);
        const uint32_t w1 = it.channels > 1 ? __ldg(it.plane1 + local) : 0u;
        for (int lane = 0; lane < spw; ++lane) {
            const int64_t p = local * spw + lane;
            if (p >= it.pixels) break;
            it.dst[p * it.channels] = __fdiv_rn(static_cast<float>((w0 >> (lane * bits)) & mask), it.max_value);
            if (it.channels > 1)
                it.dst[p * 2 + 1] = __fdiv_rn(static_cast<float>((w1 >> (lane * bits)) & mask), it.max_value);
        }
    }
}

// av-denoise-core/src/engine/kernels.rs:64-90.
template <int C>
__global__ void ingest_f32_kernel(const float* __restrict__ p0, const float* __restrict__ p1, float* __restrict__ slot,
                                  int64_t pixels, float bias) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < pixels; p += (int64_t)gridDim.x * blockDim.x) {
        slot[p * C] = __fadd_rn(p0[p], bias);
        if (C > 1) slot[p * C + 1] = __fadd_rn(p1[p], bias);
    }
}

// av-denoise-core/src/engine/kernels.rs:103-153: `u32(clamp(v, 0, 1) * max + 0.5)` with a
// truncating conversion; lanes past the last pixel pack as zero.
__device__ __forceinline__ uint32_t quantise(float v, float max_value) {
    float c = fminf(fmaxf(v, 0.0f), 1.0f);
    return __float2uint_rz(__fadd_rn(__fmul_rn(c, max_value), 0.5f));
}

template <int SPW, int C>
__global__ void egress_words_kernel(const float* __restrict__ frame, uint32_t* __restrict__ p0,
                                    uint32_t* __restrict__ p1, int64_t pixels, float max_value) {
    constexpr uint32_t kBits = 32 / SPW;
    const int64_t words = (pixels + SPW - 1) / SPW;
    for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < words; w += (int64_t)gridDim.x * blockDim.x) {
        uint32_t packed0 = 0, packed1 = 0;
#pragma unroll
        for (int lane = 0; lane < SPW; ++lane) {
            int64_t p = w * SPW + lane;
            if (p < pixels) {
                packed0 |= quantise(frame[p * C], max_value) << (lane * kBits);
                if (C > 1) packed1 |= quantise(frame[p * C + 1], max_value) << (lane * kBits);
            }
        }
        p0[w] = packed0;
        if (C > 1) p1[w] = packed1;
    }
}

template <int C>
__global__ void egress_f32_kernel(const float* __restrict__ frame, float* __restrict__ p0, float* __restrict__ p1,
                                  int64_t pixels, float bias) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < pixels; p += (int64_t)gridDim.x * blockDim.x) {
        p0[p] = __fsub_rn(frame[p * C], bias);
        if (C > 1) p1[p] = __fsub_rn(frame[p * C + 1], bias);
    }
}

}  // namespace

cudaError_t launch_ingest(const void* plane0, const void* plane1, float* slot, int64_t pixels, int channels,
                          PlaneFormat fmt, float bias, cudaStream_t stream) {
    const auto* w0 = static_cast<const uint32_t*>(plane0);
    const auto* w1 = static_cast<const uint32_t*>(plane1);
    if (fmt.kind == 2) {
        int g = grid_for(pixels);
        const auto* f0 = static_cast<const float*>(plane0);
        const auto* f1 = static_cast<const float*>(plane1);
        if (channels == 1) ingest_f32_kernel<1><<<g, kBlock, 0, stream>>>(f0, f1, slot, pixels, bias);
        else ingest_f32_kernel<2><<<g, kBlock, 0, stream>>>(f0, f1, slot, pixels, bias);
        return cudaGetLastError();
    }
    int64_t words = (pixels + fmt.samples_per_word - 1) / fmt.samples_per_word;
    int g = grid_for(words);
    if (fmt.samples_per_word == 4) {
        if (channels == 1) ingest_words_kernel<4, 1><<<g, kBlock, 0, stream>>>(w0, w1, slot, pixels, fmt.max_value);
        else ingest_words_kernel<4, 2><<<g, kBlock, 0, stream>>>(w0, w1, slot, pixels, fmt.max_value);
    } else {
        if (channels == 1) ingest_words_kernel<2, 1><<<g, kBlock, 0, stream>>>(w0, w1, slot, pixels, fmt.max_value);
        else ingest_words_kernel<2, 2><<<g, kBlock, 0, stream>>>(w0, w1, slot, pixels, fmt.max_value);
    }
    return cudaGetLastError();
}

cudaError_t launch_batch_ingest(const BatchIngestItem* items, const int64_t* word_prefix, int n, int64_t total_words,
                                cudaStream_t stream) {
    if (n <= 0 || total_words <= 0) return cudaSuccess;
    batch_ingest_kernel<<<grid_for(total_words), kBlock, 0, stream>>>(items, word_prefix, n, total_words);
    return cudaGetLastError();
}

cudaError_t launch_egress(const float* frame, void* plane0, void* plane1, int64_t pixels, int channels,
                          PlaneFormat fmt, float bias, cudaStream_t stream) {
    auto* w0 = static_cast<uint32_t*>(plane0);
    auto* w1 = static_cast<uint32_t*>(plane1);
    if (fmt.kind == 2) {
        int g = grid_for(pixels);
        auto* f0 = static_cast<float*>(plane0);
        auto* f1 = static_cast<float*>(plane1);
        if (channels == 1) egress_f32_kernel<1><<<g, kBlock, 0, stream>>>(frame, f0, f1, pixels, bias);
        else egress_f32_kernel<2><<<g, kBlock, 0, stream>>>(frame, f0, f1, pixels, bias);
        return cudaGetLastError();
    }
    int64_t words = (pixels + fmt.samples_per_word - 1) / fmt.samples_per_word;
    int g = grid_for(words);
    if (fmt.samples_per_word == 4) {
        if (channels == 1) egress_words_kernel<4, 1><<<g, kBlock, 0, stream>>>(frame, w0, w1, pixels, fmt.max_value);
        else egress_words_kernel<4, 2><<<g, kBlock, 0, stream>>>(frame, w0, w1, pixels, fmt.max_value);
    } else {
        if (channels == 1) egress_words_kernel<2, 1><<<g, kBlock, 0, stream>>>(frame, w0, w1, pixels, fmt.max_value);
        else egress_words_kernel<2, 2><<<g, kBlock, 0, stream>>>(frame, w0, w1, pixels, fmt.max_value);
    }
    return cudaGetLastError();
}

namespace {
template <int C>
__global__ void collab_normalise_kernel(int32_t* __restrict__ accum, int32_t* __restrict__ wsum,
                                        float* __restrict__ out, int64_t pixels) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= pixels) return;
    const int32_t w = wsum[p];
#pragma unroll
    for (int c = 0; c < C; ++c) {
        const float acc = __int2float_rn(accum[p * C + c]);
        out[p * C + c] = w != 0 ? __fdiv_rn(__fmul_rn(acc, 5.0f), __int2float_rn(w)) : acc;
        accum[p * C + c] = 0;
    }
    wsum[p] = 0;
}
}  // namespace

cudaError_t launch_collab_normalise(int32_t* accum, int32_t* wsum, float* out, int64_t pixels, int channels,
                                    cudaStream_t stream) {
    const unsigned blocks = static_cast<unsigned>((pixels + 255) / 256);
    if (channels == 1)
        collab_normalise_kernel<1><<<blocks, 256, 0, stream>>>(accum, wsum, out, pixels);
    else
        collab_normalise_kernel<2><<<blocks, 256, 0, stream>>>(accum, wsum, out, pixels);
    return cudaGetLastError();
}

}  // namespace avd
