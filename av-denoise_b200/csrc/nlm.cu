// NLMeans / NLMeans-HQ windowed denoise for sm_100a: one launch per output frame and plane group.
//
// What it computes (av-denoise-core/src/nlmeans/kernels/fused.rs:138-530, accumulate.rs:152-202,
// launch order dispatch/mod.rs:665-679): for every pixel p, every temporal pair pass k (q_k = -d+k,
// forward frame centre+q_k read at p+q, backward frame centre-q_k read at p-q, all q in the
// (2a+1)^2 window), then the single-frame pass (all q != 0), the patch distance
//   D(p, q) = scale * sum over the (2s+1)^2 patch of sum_c (centre - neighbour)^2
// gives the Welsch weight w = exp(-max(D - offset, 0) * h2), optionally times a per-block
// confidence; the passes accumulate sum w*I(neighbour), sum w and max w, and the finish is
//   out = (I * wref * max_w + sum wI) / (wref * max_w + sum w)   (I if the denominator <= 1e-30).
//
// How (B200 layout). A CTA owns a 32 x TY output tile and keeps every running sum in registers,
// so accumulators never leave the SM; each frame tile is read from HBM once per pass. The work
// is walked in two-lane steps: lane 0 and lane 1 are two (neighbour tile, offset) pairs that run
// side by side in packed f32x2 arithmetic (Blackwell's FADD2/FMUL2/FFMA2 issue two fp32 ops per
// slot). A temporal pass pairs the forward frame at +q with the backward frame at -q; the
// single-frame pass pairs two consecutive offsets. Per step:
//   phase 1 - row runs: each thread owns 8 consecutive pixels of one tile row plus the 2s halo
//             (its centre values stay in registers for the whole kernel), forms the squared
//             differences of both lanes and their 8 horizontal box sums with running sums, and
//             stores the lane pairs to a double-buffered row-sum tile;
//   phase 2 - column strips: each thread owns V pixels of one column, forms the vertical box
//             sums of both lanes, two MUFU ex2 give the weights, one FFMA2 accumulates w*I and
//             one FADD2 the weight sums.
// One barrier per step. The max weight is tracked as the minimum distance (exp is monotonic, so
// this is exact) when every lane shares one strength and no offset or confidence applies.
//
// The box sums run in a different order from the reference's direct row-major patch sum and
// the two lanes are summed at the end, so results can differ from the reference in the last
// bits; the parity tests bound the effect on the quantised output.

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "kernels.h"
#include "nlm_tile.cuh"

namespace avd {

namespace {

using namespace nlm_tile_detail;

template <int C, int S, bool FAST>
__global__ void __launch_bounds__(kThreads, C == 1 && FAST ? 5 : 4) nlm_window_kernel(NlmLaunch a) {
    nlm_tile<C, S, FAST>(a, blockIdx.x, blockIdx.y);
}

// The tuner's variants of the window kernel (patch radius up to kVariantMaxS): the same tile built
// for MINB resident CTAs per SM. The baseline's MINB is 5 for luma without offsets and 4 otherwise;
// variant 1 holds one CTA fewer (more registers), variant 2 one more.
constexpr int kVariantMaxS = 4;
template <int C, bool FAST>
constexpr int baseline_minb() {
    return C == 1 && FAST ? 5 : 4;
}
template <int C, int S, bool FAST, int MINB>
__global__ void __launch_bounds__(kThreads, MINB) nlm_window_variant_kernel(NlmLaunch a) {
    nlm_tile<C, S, FAST>(a, blockIdx.x, blockIdx.y);
}

template <int C, int S, bool FAST, int MINB>
cudaError_t launch_variant(const NlmLaunch& a, dim3 grid, size_t smem, cudaStream_t stream) {
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [] {
        attr_err = cudaFuncSetAttribute(nlm_window_variant_kernel<C, S, FAST, MINB>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    });
    if (attr_err != cudaSuccess) return attr_err;
    nlm_window_variant_kernel<C, S, FAST, MINB><<<grid, kThreads, smem, stream>>>(a);
    return cudaGetLastError();
}

// Persistent batch: every CTA takes tiles from one counter until the batch's tiles run out. Tile t
// belongs to the job j with prefix[j] <= t < prefix[j + 1]; jobs are whole launch descriptions.
template <int C, int S, bool FAST>
__global__ void __launch_bounds__(kThreads, C == 1 && FAST ? 5 : 4)
    nlm_batch_kernel(const NlmLaunch* __restrict__ jobs, const int* __restrict__ prefix, int njobs, int* counter) {
    using K = Cfg<C, S>;
    __shared__ int tile_s;
    const int total = prefix[njobs];
    for (;;) {
        __syncthreads();  // the previous tile is done with shared memory and `tile_s`
        if (threadIdx.x == 0) tile_s = atomicAdd(counter, 1);
        __syncthreads();
        const int t = tile_s;
        if (t >= total) return;
        int lo = 0, hi = njobs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (prefix[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        const NlmLaunch& a = jobs[lo];
        const int local = t - prefix[lo];
        const int tiles_x = (a.width + kTX - 1) / kTX;
        nlm_tile<C, S, FAST>(a, local % tiles_x, local / tiles_x);
    }
}

template <int C, int S, bool FAST>
cudaError_t launch_csf(const NlmLaunch& a, cudaStream_t stream) {
    using K = Cfg<C, S>;
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [] {
        attr_err = cudaFuncSetAttribute(nlm_window_kernel<C, S, FAST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        200 * 1024);
    });
    if (attr_err != cudaSuccess) return attr_err;
    dim3 grid((a.width + kTX - 1) / kTX, (a.height + K::TY - 1) / K::TY);
    size_t smem = nlm_smem_bytes<C, S>(a.search_radius, a.pairs, false);
    if constexpr (S <= kVariantMaxS) {
        constexpr int base = baseline_minb<C, FAST>();
        if (a.variant == 1) return launch_variant<C, S, FAST, base - 1>(a, grid, smem, stream);
        if (a.variant == 2) return launch_variant<C, S, FAST, base + 1>(a, grid, smem, stream);
    }
    nlm_window_kernel<C, S, FAST><<<grid, kThreads, smem, stream>>>(a);
    return cudaGetLastError();
}

template <int C, int S>
cudaError_t dispatch_s(const NlmLaunch& a, cudaStream_t stream) {
    if (a.patch_radius == S) return a.fast ? launch_csf<C, S, true>(a, stream) : launch_csf<C, S, false>(a, stream);
    if constexpr (S < 16) {
        return dispatch_s<C, S + 1>(a, stream);
    } else {
        return cudaErrorInvalidValue;
    }
}

template <int C, int S, bool FAST>
cudaError_t batch_csf(const NlmLaunch* jobs, const int* prefix, int njobs, int* counter, int max_a, int max_pairs,
                      cudaStream_t stream) {
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [] {
        attr_err = cudaFuncSetAttribute(nlm_batch_kernel<C, S, FAST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        200 * 1024);
    });
    if (attr_err != cudaSuccess) return attr_err;
    const size_t smem = nlm_smem_bytes<C, S>(max_a, max_pairs, false);
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, nlm_batch_kernel<C, S, FAST>, kThreads, smem);
    if (e != cudaSuccess) return e;
    nlm_batch_kernel<C, S, FAST><<<sms * (per_sm > 0 ? per_sm : 1), kThreads, smem, stream>>>(jobs, prefix, njobs,
                                                                                              counter);
    return cudaGetLastError();
}

template <int C, int S>
cudaError_t batch_s(int s, bool fast, const NlmLaunch* jobs, const int* prefix, int njobs, int* counter, int max_a,
                    int max_pairs, cudaStream_t stream) {
    if (s == S)
        return fast ? batch_csf<C, S, true>(jobs, prefix, njobs, counter, max_a, max_pairs, stream)
                    : batch_csf<C, S, false>(jobs, prefix, njobs, counter, max_a, max_pairs, stream);
    if constexpr (S < 16) {
        return batch_s<C, S + 1>(s, fast, jobs, prefix, njobs, counter, max_a, max_pairs, stream);
    } else {
        return cudaErrorInvalidValue;
    }
}

}  // namespace

// Cfg<C, S>::TY: the tile height depends on the patch radius alone.
int nlm_tile_rows(int /*channels*/, int patch_radius) {
    const int v = (32 - 2 * patch_radius) / 4;
    return 4 * (v >= 1 ? v : 1);
}

int nlm_tile_cols() { return kTX; }

int nlm_window_variants(int /*channels*/, int patch_radius, bool /*fast*/) {
    return patch_radius <= kVariantMaxS ? 3 : 1;
}

cudaError_t launch_nlm_batch(const NlmLaunch* jobs, const int* prefix, int njobs, int* counter, int channels,
                             int patch_radius, bool fast, int max_search_radius, int max_pairs, cudaStream_t stream) {
    if (channels == 1)
        return batch_s<1, 0>(patch_radius, fast, jobs, prefix, njobs, counter, max_search_radius, max_pairs, stream);
    if (channels == 2)
        return batch_s<2, 0>(patch_radius, fast, jobs, prefix, njobs, counter, max_search_radius, max_pairs, stream);
    return cudaErrorInvalidValue;
}

cudaError_t launch_nlm(const NlmLaunch& a, cudaStream_t stream) {
    if (a.pairs < 0 || a.pairs > kMaxPairs || a.search_radius < 0 || a.search_radius > 8 || a.patch_radius < 0 ||
        a.patch_radius > 16)
        return cudaErrorInvalidValue;
    if (a.ref_ring) return launch_nlm_ref(a, stream);
    if (a.channels == 1) return dispatch_s<1, 0>(a, stream);
    if (a.channels == 2) return dispatch_s<2, 0>(a, stream);
    return cudaErrorInvalidValue;
}

}  // namespace avd
