// NLMeans prefilters for sm_100a: the bilateral blur that builds a reference ring slot, and the
// windowed tile in its reference-ring form, which compares patches on the reference ring while it
// averages the input ring's values.
//
// Bilateral (av-denoise-core/src/nlmeans/kernels/bilateral.rs:16-107): for every pixel p,
//   w(o) = exp(-((dx^2 + dy^2) * inv_two_sigma_s_sq + |I(p+o) - I(p)|^2 * inv_two_sigma_r_sq))
// over the (2r+1)^2 offsets o = (dx, dy) in row-major order, coordinates clamped to the frame, and
//   out(p) = (sum w(o) I(p+o)) * (1 / sum w(o)).
// A 32 x 8 CTA stages its (32+2r) x (8+2r) window once in shared memory, one thread per output
// pixel. The sums are formed in the reference's order with every multiply and add rounded on its
// own (no fused multiply-add) and the exponential is exp_mirror.cuh's, so the reference slot equals
// the CPU restatement's bit for bit.
//
// The reference-ring NLM tile is the nlm.cu tile with two more shared tiles per pass for the input
// values (nlm_tile.cuh, REF): the reference form of fused.rs:532-900.

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "exp_mirror.cuh"
#include "kernels.h"
#include "nlm_tile.cuh"

namespace avd {

namespace {

using namespace nlm_tile_detail;

constexpr int kBx = 32, kBy = 8;

template <int C>
__global__ void __launch_bounds__(kBx * kBy) bilateral_kernel(const float* __restrict__ in, float* __restrict__ out,
                                                              int W, int H, int R, float inv_s, float inv_r) {
    extern __shared__ __align__(16) float tile[];
    const int tw = kBx + 2 * R;
    const int th = kBy + 2 * R;
    const int x0 = blockIdx.x * kBx - R;
    const int y0 = blockIdx.y * kBy - R;
    const int tid = threadIdx.y * kBx + threadIdx.x;
    for (int i = tid; i < tw * th; i += kBx * kBy) {
        const int r = i / tw;
        const int c = i - r * tw;
        const int gx = clampi(x0 + c, 0, W - 1);
        const int gy = clampi(y0 + r, 0, H - 1);
        const float* src = in + ((int64_t)gy * W + gx) * C;
#pragma unroll
        for (int ch = 0; ch < C; ++ch) tile[i * C + ch] = __ldg(src + ch);
    }
    __syncthreads();
    const int gx = blockIdx.x * kBx + threadIdx.x;
    const int gy = blockIdx.y * kBy + threadIdx.y;
    if (gx >= W || gy >= H) return;

    const float* ctr = tile + ((threadIdx.y + R) * tw + threadIdx.x + R) * C;
    float cv[C];
#pragma unroll
    for (int ch = 0; ch < C; ++ch) cv[ch] = ctr[ch];
    float wsum = 0.0f;
    float acc[C];
#pragma unroll
    for (int ch = 0; ch < C; ++ch) acc[ch] = 0.0f;
    for (int oy = 0; oy <= 2 * R; ++oy) {
        const int dy = oy - R;
        const float* row = tile + ((threadIdx.y + oy) * tw + threadIdx.x) * C;
        for (int ox = 0; ox <= 2 * R; ++ox) {
            const int dx = ox - R;
            const float* nb = row + ox * C;
            float range_sq = 0.0f;
#pragma unroll
            for (int ch = 0; ch < C; ++ch) {
                const float lane = __fsub_rn(nb[ch], cv[ch]);
                range_sq = __fadd_rn(range_sq, __fmul_rn(lane, lane));
            }
            const float spatial = __fmul_rn(static_cast<float>(dx * dx + dy * dy), inv_s);
            const float w = exp_mirror(-__fadd_rn(spatial, __fmul_rn(range_sq, inv_r)));
#pragma unroll
            for (int ch = 0; ch < C; ++ch) acc[ch] = __fadd_rn(acc[ch], __fmul_rn(nb[ch], w));
            wsum = __fadd_rn(wsum, w);
        }
    }
    const float inv = __frcp_rn(wsum);
    float* dst = out + ((int64_t)gy * W + gx) * C;
#pragma unroll
    for (int ch = 0; ch < C; ++ch) dst[ch] = __fmul_rn(acc[ch], inv);
}

template <int C, int S, bool FAST>
__global__ void __launch_bounds__(kThreads, C == 1 ? 4 : 3) nlm_ref_window_kernel(NlmLaunch a) {
    nlm_tile<C, S, FAST, false, true>(a, blockIdx.x, blockIdx.y);
}

template <int C, int S, bool FAST>
cudaError_t launch_ref_csf(const NlmLaunch& a, cudaStream_t stream) {
    using K = Cfg<C, S>;
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [] {
        attr_err = cudaFuncSetAttribute(nlm_ref_window_kernel<C, S, FAST>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    });
    if (attr_err != cudaSuccess) return attr_err;
    dim3 grid((a.width + kTX - 1) / kTX, (a.height + K::TY - 1) / K::TY);
    const size_t smem = nlm_smem_bytes<C, S>(a.search_radius, a.pairs, true);
    if (smem > 220 * 1024) return cudaErrorInvalidValue;
    nlm_ref_window_kernel<C, S, FAST><<<grid, kThreads, smem, stream>>>(a);
    return cudaGetLastError();
}

template <int C, int S>
cudaError_t dispatch_ref_s(const NlmLaunch& a, cudaStream_t stream) {
    if (a.patch_radius == S)
        return a.fast ? launch_ref_csf<C, S, true>(a, stream) : launch_ref_csf<C, S, false>(a, stream);
    if constexpr (S < 16) {
        return dispatch_ref_s<C, S + 1>(a, stream);
    } else {
        return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t launch_nlm_ref(const NlmLaunch& a, cudaStream_t stream) {
    if (!a.ref_ring || a.pairs < 0 || a.pairs > kMaxPairs || a.search_radius < 0 || a.search_radius > 8 ||
        a.patch_radius < 0 || a.patch_radius > 16)
        return cudaErrorInvalidValue;
    if (a.channels == 1) return dispatch_ref_s<1, 0>(a, stream);
    if (a.channels == 2) return dispatch_ref_s<2, 0>(a, stream);
    return cudaErrorInvalidValue;
}

cudaError_t launch_bilateral(const float* in, float* out, int width, int height, int channels, int radius,
                             float inv_two_sigma_s_sq, float inv_two_sigma_r_sq, cudaStream_t stream) {
    if (!in || !out || width < 1 || height < 1 || radius < 1 || radius > 22 || channels < 1 || channels > 2)
        return cudaErrorInvalidValue;
    const size_t smem = (size_t)(kBx + 2 * radius) * (kBy + 2 * radius) * channels * sizeof(float);
    dim3 grid((width + kBx - 1) / kBx, (height + kBy - 1) / kBy);
    dim3 block(kBx, kBy);
    if (channels == 1)
        bilateral_kernel<1><<<grid, block, smem, stream>>>(in, out, width, height, radius, inv_two_sigma_s_sq,
                                                           inv_two_sigma_r_sq);
    else
        bilateral_kernel<2><<<grid, block, smem, stream>>>(in, out, width, height, radius, inv_two_sigma_s_sq,
                                                           inv_two_sigma_r_sq);
    return cudaGetLastError();
}

}  // namespace avd
