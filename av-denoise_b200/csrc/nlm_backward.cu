// Adjoint of the windowed NLMeans frame on sm_100a: dL/d(window frames) and dL/d(strength) for an
// upstream gradient dL/d(output), recomputing every weight instead of storing the
// (2d+1)(2a+1)^2 x pixels weight tensor.
//
// The forward being differentiated (av-denoise-core/src/nlmeans/kernels/fused.rs:138-530,
// accumulate.rs:152-202, helpers.rs:34-73), per output pixel p and channel c:
//   D_o(p) = scale * sum_{delta in patch} sum_c (I(clamp(p+delta)) - F_o(clamp(p+q_o+delta)))^2
//   w_o    = exp(-max(D_o - off_o, 0) * h2),         h2 = 255^2 / (3 strength^2 (2s+1)^2)
//   A = sum_o w_o F_o(clamp(p+q_o)),  W = sum_o w_o,  M = max_o w_o
//   out    = (I(p) wref M + A) / (wref M + W)          (out = I(p) when the denominator <= 1e-30)
// over the offsets o in the forward's order: for each pair k (q_k = -d+k) and every q, the forward
// frame k at +q then the backward frame 2d-k at -q; then the centre frame at every q != 0. The max
// passes its gradient to the first offset reaching it; the clamps fold border terms onto the edge
// pixels, exactly as the forward reads them.
//
// Kernel 1 (one thread per pixel) recomputes W, A, M, its argmax and the output, writes the
// direct centre term and keeps 5 floats per pixel. Kernel 2 gives each CTA a 16x16 tile: every
// thread walks all offsets for its pixel, recomputes w_o, and scatters the A term and the patch
// terms into shared-memory gradient tiles, one per window frame with an (a+s) halo, which are
// added to global memory once per CTA. dL/dh2 is reduced per CTA and summed in a fixed order.

#include <cstdint>

#include "kernels.h"

namespace avd {
namespace {

constexpr int kTile = 16;
constexpr int kRecord = 5;  // out[0], out[1], 1/den (0 = passthrough), dL/dM, argmax offset id

__device__ __forceinline__ int clampi(int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }

struct Bwd {
    const float* window;
    const float* grad_out;
    float* grad_window;
    float* records;
    float* partials;
    int width, height, d, a, s;
    int64_t frame_elems;
    float h2, wref, pair_off, spatial_off;
};

template <int C>
__device__ __forceinline__ const float* at(const Bwd& b, int f, int x, int y) {
    return b.window + f * b.frame_elems + (static_cast<int64_t>(clampi(y, b.height)) * b.width + clampi(x, b.width)) * C;
}

template <int C>
__device__ __forceinline__ float distance(const Bwd& b, int f, int px, int py, int qx, int qy) {
    const float scale = C == 1 ? 3.0f : 1.5f;
    float sum = 0.0f;
    for (int oy = -b.s; oy <= b.s; ++oy)
        for (int ox = -b.s; ox <= b.s; ++ox) {
            const float* c = at<C>(b, b.d, px + ox, py + oy);
            const float* n = at<C>(b, f, px + ox + qx, py + oy + qy);
            float l = 0.0f;
#pragma unroll
            for (int ch = 0; ch < C; ++ch) {
                const float diff = c[ch] - n[ch];
                l += diff * diff;
            }
            sum += l * scale;
        }
    return sum;
}

__device__ __forceinline__ float welsch(float dist, float h2, float off) { return expf(-fmaxf(dist - off, 0.0f) * h2); }

// Visits every offset of the forward's order as (id, frame, qx, qy, offset).
template <typename F>
__device__ __forceinline__ void for_offsets(const Bwd& b, F&& fn) {
    int id = 0;
    for (int k = 0; k < b.d; ++k)
        for (int qy = -b.a; qy <= b.a; ++qy)
            for (int qx = -b.a; qx <= b.a; ++qx) {
                fn(id++, k, qx, qy, b.pair_off);
                fn(id++, 2 * b.d - k, -qx, -qy, b.pair_off);
            }
    for (int qy = -b.a; qy <= b.a; ++qy)
        for (int qx = -b.a; qx <= b.a; ++qx) {
            if (qx == 0 && qy == 0) continue;
            fn(id++, b.d, qx, qy, b.spatial_off);
        }
}

template <int C>
__global__ void __launch_bounds__(256) bwd_pixel_kernel(Bwd b) {
    const int px = blockIdx.x * kTile + threadIdx.x % kTile;
    const int py = blockIdx.y * kTile + threadIdx.x / kTile;
    if (px >= b.width || py >= b.height) return;
    float acc[C] = {};
    float W = 0.0f, M = 0.0f;
    int argmax = -1;
    for_offsets(b, [&](int id, int f, int qx, int qy, float off) {
        const float w = welsch(distance<C>(b, f, px, py, qx, qy), b.h2, off);
        const float* n = at<C>(b, f, px + qx, py + qy);
#pragma unroll
        for (int ch = 0; ch < C; ++ch) acc[ch] += w * n[ch];
        W += w;
        if (w > M) {
            M = w;
            argmax = id;
        }
    });
    const int64_t p = static_cast<int64_t>(py) * b.width + px;
    const float* I = at<C>(b, b.d, px, py);
    const float* g = b.grad_out + p * C;
    float* gc = b.grad_window + b.d * b.frame_elems + p * C;
    float* rec = b.records + p * kRecord;
    const float den = b.wref * M + W;
    if (!(den > 1e-30f)) {
#pragma unroll
        for (int ch = 0; ch < C; ++ch) {
            gc[ch] = g[ch];
            rec[ch] = I[ch];
        }
        rec[2] = 0.0f;
        rec[3] = 0.0f;
        rec[4] = __int_as_float(-1);
        return;
    }
    const float inv = 1.0f / den;
    float gm = 0.0f;
    float out[2] = {0.0f, 0.0f};
#pragma unroll
    for (int ch = 0; ch < C; ++ch) {
        out[ch] = (I[ch] * b.wref * M + acc[ch]) * inv;
        gc[ch] = g[ch] * b.wref * M * inv;
        gm += g[ch] * b.wref * (I[ch] - out[ch]) * inv;
    }
    rec[0] = out[0];
    rec[1] = out[1];
    rec[2] = inv;
    rec[3] = gm;
    rec[4] = __int_as_float(argmax);
}

template <int C>
__global__ void __launch_bounds__(256) bwd_scatter_kernel(Bwd b) {
    extern __shared__ float tiles[];
    __shared__ float red[8];
    const int H = b.a + b.s;
    const int T = kTile + 2 * H;
    const int frames = 2 * b.d + 1;
    const int x0 = blockIdx.x * kTile - H, y0 = blockIdx.y * kTile - H;
    for (int i = threadIdx.x; i < frames * T * T * C; i += blockDim.x) tiles[i] = 0.0f;
    __syncthreads();
    const int px = blockIdx.x * kTile + threadIdx.x % kTile;
    const int py = blockIdx.y * kTile + threadIdx.x / kTile;
    float gh2 = 0.0f;
    if (px < b.width && py < b.height) {
        const int64_t p = static_cast<int64_t>(py) * b.width + px;
        const float* rec = b.records + p * kRecord;
        const float inv = rec[2];
        if (inv != 0.0f) {
            const float gm = rec[3];
            const int argmax = __float_as_int(rec[4]);
            float g[C], out[C];
#pragma unroll
            for (int ch = 0; ch < C; ++ch) {
                g[ch] = b.grad_out[p * C + ch];
                out[ch] = rec[ch];
            }
            const float scale2 = C == 1 ? 6.0f : 3.0f;  // 2 * channel scale
            auto slot = [&](int f, int x, int y) {
                return tiles + ((static_cast<int64_t>(f) * T + (clampi(y, b.height) - y0)) * T +
                                (clampi(x, b.width) - x0)) * C;
            };
            for_offsets(b, [&](int id, int f, int qx, int qy, float off) {
                const float dist = distance<C>(b, f, px, py, qx, qy);
                const float w = welsch(dist, b.h2, off);
                const float* n = at<C>(b, f, px + qx, py + qy);
                float gw = id == argmax ? gm : 0.0f;
                float* an = slot(f, px + qx, py + qy);
#pragma unroll
                for (int ch = 0; ch < C; ++ch) {
                    gw += g[ch] * (n[ch] - out[ch]) * inv;
                    atomicAdd(an + ch, g[ch] * w * inv);
                }
                const float excess = dist - off;
                if (excess > 0.0f && w > 0.0f) {
                    gh2 -= gw * excess * w;
                    const float gd = -gw * b.h2 * w * scale2;
                    for (int oy = -b.s; oy <= b.s; ++oy)
                        for (int ox = -b.s; ox <= b.s; ++ox) {
                            const float* c = at<C>(b, b.d, px + ox, py + oy);
                            const float* m = at<C>(b, f, px + ox + qx, py + oy + qy);
                            float* sc = slot(b.d, px + ox, py + oy);
                            float* sm = slot(f, px + ox + qx, py + oy + qy);
#pragma unroll
                            for (int ch = 0; ch < C; ++ch) {
                                const float t = gd * (c[ch] - m[ch]);
                                atomicAdd(sc + ch, t);
                                atomicAdd(sm + ch, -t);
                            }
                        }
                }
            });
        }
    }
    // dL/dh2 of the CTA, reduced in a fixed order.
    for (int o = 16; o > 0; o >>= 1) gh2 += __shfl_xor_sync(0xffffffffu, gh2, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = gh2;
    __syncthreads();
    if (threadIdx.x == 0) {
        float total = 0.0f;
        for (int i = 0; i < 8; ++i) total += red[i];
        b.partials[blockIdx.y * gridDim.x + blockIdx.x] = total;
    }
    // Flush the tiles (only positions inside the frame were written).
    for (int i = threadIdx.x; i < frames * T * T; i += blockDim.x) {
        const int f = i / (T * T), r = i % (T * T);
        const int gx = x0 + r % T, gy = y0 + r / T;
        if (gx < 0 || gy < 0 || gx >= b.width || gy >= b.height) continue;
        float* dst = b.grad_window + f * b.frame_elems + (static_cast<int64_t>(gy) * b.width + gx) * C;
#pragma unroll
        for (int ch = 0; ch < C; ++ch) {
            const float v = tiles[static_cast<int64_t>(i) * C + ch];
            if (v != 0.0f) atomicAdd(dst + ch, v);
        }
    }
}

__global__ void bwd_strength_kernel(const float* partials, int n, float h2, float strength, float* grad_strength) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float total = 0.0f;
    for (int i = 0; i < n; ++i) total += partials[i];
    // h2 = K / strength^2, so dh2/dstrength = -2 h2 / strength.
    *grad_strength = total * (-2.0f * h2 / strength);
}

}  // namespace

size_t nlm_backward_scratch_floats(int width, int height) {
    const size_t tiles = static_cast<size_t>((width + kTile - 1) / kTile) * ((height + kTile - 1) / kTile);
    return static_cast<size_t>(width) * height * kRecord + tiles;
}

size_t nlm_backward_smem_bytes(int channels, int temporal_radius, int search_radius, int patch_radius) {
    const size_t T = kTile + 2 * (search_radius + patch_radius);
    return static_cast<size_t>(2 * temporal_radius + 1) * T * T * channels * sizeof(float);
}

cudaError_t launch_nlm_backward(const NlmBackwardLaunch& l, cudaStream_t s) {
    Bwd b{};
    b.window = l.window;
    b.grad_out = l.grad_out;
    b.grad_window = l.grad_window;
    b.records = l.scratch;
    b.width = l.width;
    b.height = l.height;
    b.d = l.temporal_radius;
    b.a = l.search_radius;
    b.s = l.patch_radius;
    b.frame_elems = static_cast<int64_t>(l.width) * l.height * l.channels;
    b.partials = l.scratch + static_cast<size_t>(l.width) * l.height * kRecord;
    b.h2 = l.h2;
    b.wref = l.wref;
    b.pair_off = l.pair_offset;
    b.spatial_off = l.spatial_offset;
    const size_t frames_elems = static_cast<size_t>(2 * b.d + 1) * b.frame_elems;
    cudaError_t e = cudaMemsetAsync(l.grad_window, 0, frames_elems * sizeof(float), s);
    if (e != cudaSuccess) return e;
    dim3 grid((l.width + kTile - 1) / kTile, (l.height + kTile - 1) / kTile);
    const size_t smem = nlm_backward_smem_bytes(l.channels, b.d, b.a, b.s);
    if (l.channels == 1) {
        bwd_pixel_kernel<1><<<grid, 256, 0, s>>>(b);
        if (smem > 48 * 1024) cudaFuncSetAttribute(bwd_scatter_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   static_cast<int>(smem));
        bwd_scatter_kernel<1><<<grid, 256, smem, s>>>(b);
    } else {
        bwd_pixel_kernel<2><<<grid, 256, 0, s>>>(b);
        if (smem > 48 * 1024) cudaFuncSetAttribute(bwd_scatter_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   static_cast<int>(smem));
        bwd_scatter_kernel<2><<<grid, 256, smem, s>>>(b);
    }
    bwd_strength_kernel<<<1, 32, 0, s>>>(b.partials, static_cast<int>(grid.x * grid.y), l.h2, l.strength,
                                         l.grad_strength);
    return cudaGetLastError();
}

}  // namespace avd
