// NLMeans / NLMeans-HQ windowed denoise for sm_100a: one launch per output frame and plane group.
//
// What it computes (av-denoise-core/src/nlmeans/kernels/fused.rs:138-530, accumulate.rs:152-202,
// launch order dispatch/mod.rs:665-679): for every pixel p, every temporal pair pass k (q_k = -d+k,
// forward frame centre+q_k read at p+q, backward frame centre-q_k read at p-q, all q in the
// (2a+1)^2 window), then the single-frame pass (all q != 0), the patch distance
//   D(p, q) = scale * sum over the (2s+1)^2 patch of sum_c (centre - neighbour)^2
// gives the Welsch weight w = exp(-max(D - offset, 0) * h2), optionally times a per-block
// confidence; the pass accumulates sum w*I(neighbour), sum w and max w, and the finish is
//   out = (I * wref * max_w + sum wI) / (wref * max_w + sum w)   (I if the denominator <= 1e-30).
//
// How (B200 layout): a CTA owns a 32 x TY output tile and walks every pass and offset with the
// running sums in registers, so the accumulators never leave the SM. Per offset:
//   phase 1 - row runs: each task owns 8 consecutive pixels of one tile row (plus the 2s halo),
//             computes the squared differences against the neighbour frame staged in shared
//             memory, and forms the 8 horizontal box sums with a running sum; one 16-byte store
//             pair writes them to a double-buffered row-sum tile;
//   phase 2 - column strips: each thread owns V pixels of one column, forms the vertical box
//             sums with a running sum, then the weight (one MUFU ex2) and the accumulation.
// One barrier per offset (the row-sum tile is double buffered). The per-offset cost is ~15
// issue slots per output pixel against one MUFU op, which is why the kernel is bound by issue
// and the SFU, not by HBM: every frame tile is read from HBM once per pass.
//
// The box sums run in a different order from the reference's direct row-major patch sum, so
// D can differ in the last bits; the weights feed a normalised average, and the parity tests
// bound the effect on the quantised output.

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "kernels.h"

namespace avd {

namespace {

constexpr int kTX = 32;       // tile columns
constexpr int kThreads = 128;  // 4 warps: 32 columns x 4 strips
constexpr int kRun = 8;        // phase-1 run length
constexpr int kRuns = kTX / kRun;
constexpr float kLog2e = 1.4426950408889634f;

__host__ __device__ constexpr int round_up4(int v) { return (v + 3) & ~3; }

template <int C, int S>
struct Cfg {
    static constexpr int V = (32 - 2 * S) / 4 >= 1 ? (32 - 2 * S) / 4 : 1;  // outputs per column strip
    static constexpr int TY = 4 * V;                                       // tile rows
    static constexpr int HR = TY + 2 * S;                                  // row-sum rows
    static constexpr int TASKS = HR * kRuns;                               // phase-1 tasks
    static constexpr int CW = kTX + 2 * S;                                 // centre tile columns
    static constexpr int CSTRIDE = round_up4(CW * C);                      // floats per centre row
    static constexpr int CROWS = TY + 2 * S;
    static constexpr int RUNW = kRun + 2 * S;  // pixels one run reads
    static constexpr int RUNF4 = (RUNW * C + 3) / 4;
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// The Welsch weight from an unscaled box sum `d` (sum of squared differences):
// w = exp(-max(d * scale - off, 0) * h2) = 2^(max(...) * (-h2 * log2 e)).
__device__ __forceinline__ float welsch(float d, float scale, float off, float neg_h2_log2e) {
    float excess = fmaxf(fmaf(d, scale, -off), 0.0f);
#ifdef AVD_NLM_ACCURATE_EXP
    return expf(excess * (neg_h2_log2e / kLog2e));
#else
    return ex2_approx(excess * neg_h2_log2e);
#endif
}

// Stages frame `slot` over the tile's window into shared memory, coordinates clamped to the image
// as the reference's `read_clamped_line` does (helpers.rs:20-32).
template <int C>
__device__ void load_tile(float* tile, int stride, int rows, int cols, const float* __restrict__ frame, int x0, int y0,
                          int W, int H) {
    const int n = rows * cols;
    for (int idx = threadIdx.x; idx < n; idx += kThreads) {
        int r = idx / cols;
        int c = idx - r * cols;
        int gx = clampi(x0 + c, 0, W - 1);
        int gy = clampi(y0 + r, 0, H - 1);
        const float* src = frame + ((int64_t)gy * W + gx) * C;
        float* dst = tile + r * stride + c * C;
        if (C == 1) {
            dst[0] = __ldg(src);
        } else {
            float2 v = __ldg(reinterpret_cast<const float2*>(src));
            *reinterpret_cast<float2*>(dst) = v;
        }
    }
}

// Phase 1 of one offset for one direction: 8 horizontal box sums of one tile row.
template <int C, int S>
__device__ __forceinline__ void row_run(const float* __restrict__ ctr_row, const float* __restrict__ nbr_row,
                                        float* __restrict__ hs_out) {
    using K = Cfg<C, S>;
    float cv[K::RUNF4 * 4];
#pragma unroll
    for (int i = 0; i < K::RUNF4; ++i) {
        float4 v = *reinterpret_cast<const float4*>(ctr_row + 4 * i);
        cv[4 * i] = v.x;
        cv[4 * i + 1] = v.y;
        cv[4 * i + 2] = v.z;
        cv[4 * i + 3] = v.w;
    }
    float d[K::RUNW];
#pragma unroll
    for (int i = 0; i < K::RUNW; ++i) {
        if (C == 1) {
            float diff = cv[i] - nbr_row[i];
            d[i] = diff * diff;
        } else {
            float2 n = *reinterpret_cast<const float2*>(nbr_row + 2 * i);
            float du = cv[2 * i] - n.x;
            float dv = cv[2 * i + 1] - n.y;
            d[i] = fmaf(dv, dv, du * du);
        }
    }
    float h[kRun];
    float run = d[0];
#pragma unroll
    for (int i = 1; i <= 2 * S; ++i) run += d[i];
    h[0] = run;
#pragma unroll
    for (int j = 1; j < kRun; ++j) {
        run = run + d[j + 2 * S] - d[j - 1];
        h[j] = run;
    }
    *reinterpret_cast<float4*>(hs_out) = make_float4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<float4*>(hs_out + 4) = make_float4(h[4], h[5], h[6], h[7]);
}

template <int C, int S>
struct Smem {
    float* ctr;
    float* nbr[2];
    float* hs;  // [2 buffers][2 directions][HR][kTX]
    int nstride;
    int nrows, ncols;
};

// One pass (a temporal pair when PAIR, else the single-frame pass) over the whole window.
template <int C, int S, bool PAIR, bool CONF>
__device__ __forceinline__ void run_pass(const Smem<C, S>& sm, int A, float scale, float off_pair,
                                         const float* __restrict__ lut, float neg_h2_log2e, const float* cf,
                                         const float* cb, int& buf, float (&acc_tot)[Cfg<C, S>::V][C],
                                         float (&ws_tot)[Cfg<C, S>::V], float (&wm)[Cfg<C, S>::V]) {
    using K = Cfg<C, S>;
    constexpr int V = K::V;
    const int tid = threadIdx.x;
    const int col = tid & 31;
    const int y0 = (tid >> 5) * V;
    const int side = 2 * A + 1;
    const int hs_plane = K::HR * kTX;

    float acc[V][C];
    float ws[V];
#pragma unroll
    for (int k = 0; k < V; ++k) {
        ws[k] = 0.0f;
#pragma unroll
        for (int c = 0; c < C; ++c) acc[k][c] = 0.0f;
    }

    for (int qyi = 0; qyi < side; ++qyi) {
        const int qy = qyi - A;
        for (int qxi = 0; qxi < side; ++qxi) {
            const int qx = qxi - A;
            if (!PAIR && qx == 0 && qy == 0) continue;
            float* hs = sm.hs + buf * 2 * hs_plane;

            // Phase 1: row runs.
            for (int task = tid; task < K::TASKS; task += kThreads) {
                const int r = task / kRuns;
                const int x0 = (task - r * kRuns) * kRun;
                const float* crow = sm.ctr + r * K::CSTRIDE + x0 * C;
                const float* nrow = sm.nbr[0] + (r + qy + A) * sm.nstride + (x0 + qx + A) * C;
                row_run<C, S>(crow, nrow, hs + r * kTX + x0);
                if (PAIR) {
                    const float* brow = sm.nbr[1] + (r - qy + A) * sm.nstride + (x0 - qx + A) * C;
                    row_run<C, S>(crow, brow, hs + hs_plane + r * kTX + x0);
                }
            }
            __syncthreads();

            // Phase 2: column strips.
            const float off = PAIR ? off_pair : (lut ? __ldg(lut + qyi * side + qxi) : 0.0f);
            float hv[V + 2 * S];
#pragma unroll
            for (int i = 0; i < V + 2 * S; ++i) hv[i] = hs[(y0 + i) * kTX + col];
            float hb[PAIR ? V + 2 * S : 1];
            if (PAIR) {
#pragma unroll
                for (int i = 0; i < V + 2 * S; ++i) hb[i] = hs[hs_plane + (y0 + i) * kTX + col];
            }
            float run = hv[0];
#pragma unroll
            for (int i = 1; i <= 2 * S; ++i) run += hv[i];
            float runb = 0.0f;
            if (PAIR) {
                runb = hb[0];
#pragma unroll
                for (int i = 1; i <= 2 * S; ++i) runb += hb[i];
            }
            const float* nf = sm.nbr[0] + (y0 + S + qy + A) * sm.nstride + (col + S + qx + A) * C;
            const float* nb = PAIR ? sm.nbr[1] + (y0 + S - qy + A) * sm.nstride + (col + S - qx + A) * C : nullptr;
#pragma unroll
            for (int k = 0; k < V; ++k) {
                if (k > 0) {
                    run = run + hv[k + 2 * S] - hv[k - 1];
                    if (PAIR) runb = runb + hb[k + 2 * S] - hb[k - 1];
                }
                float w = welsch(run, scale, off, neg_h2_log2e);
                if (CONF) w *= cf[k];
                const float* pf = nf + k * sm.nstride;
                if (!PAIR) {
#pragma unroll
                    for (int c = 0; c < C; ++c) acc[k][c] = fmaf(pf[c], w, acc[k][c]);
                    ws[k] += w;
                    wm[k] = fmaxf(wm[k], w);
                } else {
                    float wb = welsch(runb, scale, off, neg_h2_log2e);
                    if (CONF) wb *= cb[k];
                    const float* pb = nb + k * sm.nstride;
#pragma unroll
                    for (int c = 0; c < C; ++c) acc[k][c] = fmaf(pb[c], wb, fmaf(pf[c], w, acc[k][c]));
                    ws[k] += w + wb;
                    wm[k] = fmaxf(wm[k], fmaxf(w, wb));
                }
            }
            buf ^= 1;
        }
    }

    // The pass adds its register sums to the frame sums once, as each reference launch does.
#pragma unroll
    for (int k = 0; k < V; ++k) {
        ws_tot[k] += ws[k];
#pragma unroll
        for (int c = 0; c < C; ++c) acc_tot[k][c] += acc[k][c];
    }
}

template <int C, int S>
__global__ void __launch_bounds__(kThreads) nlm_window_kernel(NlmLaunch a) {
    using K = Cfg<C, S>;
    constexpr int V = K::V;
    extern __shared__ __align__(16) float smem_raw[];

    const int A = a.search_radius;
    const int W = a.width, H = a.height;
    const int X0 = blockIdx.x * kTX;
    const int Y0 = blockIdx.y * K::TY;
    const int tid = threadIdx.x;
    const int col = tid & 31;
    const int y0 = (tid >> 5) * V;

    Smem<C, S> sm;
    sm.nrows = K::TY + 2 * S + 2 * A;
    sm.ncols = kTX + 2 * S + 2 * A;
    sm.nstride = round_up4(sm.ncols * C);
    sm.ctr = smem_raw;
    sm.nbr[0] = sm.ctr + K::CROWS * K::CSTRIDE;
    sm.nbr[1] = sm.nbr[0] + sm.nrows * sm.nstride;
    sm.hs = sm.nbr[1] + (a.pairs > 0 ? sm.nrows * sm.nstride : 0);

    const float h2 = __ldg(a.derived + a.h2_word);
    const float off_pair = __ldg(a.derived + a.offset_word);
    const float neg_h2_log2e = -h2 * kLog2e;
    const float scale = C == 1 ? 3.0f : 1.5f;

    const float* centre = a.ring + a.slot_centre * a.frame_elems;
    load_tile<C>(sm.ctr, K::CSTRIDE, K::CROWS, K::CW, centre, X0 - S, Y0 - S, W, H);

    float acc[V][C];
    float ws[V];
    float wm[V];
#pragma unroll
    for (int k = 0; k < V; ++k) {
        ws[k] = 0.0f;
        wm[k] = 0.0f;
#pragma unroll
        for (int c = 0; c < C; ++c) acc[k][c] = 0.0f;
    }

    int buf = 0;
    float cf[V], cb[V];
    for (int p = 0; p < a.pairs; ++p) {
        __syncthreads();  // every thread is done with the previous pass's tiles
        load_tile<C>(sm.nbr[0], sm.nstride, sm.nrows, sm.ncols, a.ring + a.slot_fwd[p] * a.frame_elems, X0 - S - A,
                     Y0 - S - A, W, H);
        load_tile<C>(sm.nbr[1], sm.nstride, sm.nrows, sm.ncols, a.ring + a.slot_bwd[p] * a.frame_elems, X0 - S - A,
                     Y0 - S - A, W, H);
        __syncthreads();
        if (a.conf) {
#pragma unroll
            for (int k = 0; k < V; ++k) {
                int gx = min(X0 + col, W - 1), gy = min(Y0 + y0 + k, H - 1);
                int bc = min(gx / a.conf_step, a.blocks_x - 1);
                int br = min(gy / a.conf_step, a.blocks_y - 1);
                cf[k] = __ldg(a.conf + a.conf_fwd_off[p] + br * a.blocks_x + bc);
                cb[k] = __ldg(a.conf + a.conf_bwd_off[p] + br * a.blocks_x + bc);
            }
            run_pass<C, S, true, true>(sm, A, scale, off_pair, nullptr, neg_h2_log2e, cf, cb, buf, acc, ws, wm);
        } else {
            run_pass<C, S, true, false>(sm, A, scale, off_pair, nullptr, neg_h2_log2e, cf, cb, buf, acc, ws, wm);
        }
    }

    __syncthreads();
    load_tile<C>(sm.nbr[0], sm.nstride, sm.nrows, sm.ncols, centre, X0 - S - A, Y0 - S - A, W, H);
    __syncthreads();
    run_pass<C, S, false, false>(sm, A, scale, 0.0f, a.spatial_lut, neg_h2_log2e, cf, cb, buf, acc, ws, wm);

    // Finish (accumulate.rs:175-201), written straight to the output frame.
    const int gx = X0 + col;
#pragma unroll
    for (int k = 0; k < V; ++k) {
        const int gy = Y0 + y0 + k;
        if (gx >= W || gy >= H) continue;
        const float* orig = sm.ctr + (y0 + k + S) * K::CSTRIDE + (col + S) * C;
        const float self_weight = __fmul_rn(a.wref, wm[k]);
        const float denom = __fadd_rn(self_weight, ws[k]);
        float* dst = a.out + ((int64_t)gy * W + gx) * C;
        if (denom > 1e-30f) {
            const float inv = __frcp_rn(denom);
#pragma unroll
            for (int c = 0; c < C; ++c) dst[c] = __fmul_rn(__fadd_rn(__fmul_rn(orig[c], self_weight), acc[k][c]), inv);
        } else {
#pragma unroll
            for (int c = 0; c < C; ++c) dst[c] = orig[c];
        }
    }
}

template <int C, int S>
size_t smem_bytes(int A, int pairs) {
    using K = Cfg<C, S>;
    int nrows = K::TY + 2 * S + 2 * A;
    int ncols = kTX + 2 * S + 2 * A;
    int nstride = round_up4(ncols * C);
    size_t floats = (size_t)K::CROWS * K::CSTRIDE + (size_t)(pairs > 0 ? 2 : 1) * nrows * nstride +
                    (size_t)2 * 2 * K::HR * kTX;
    return floats * sizeof(float);
}

template <int C, int S>
cudaError_t launch_cs(const NlmLaunch& a, cudaStream_t stream) {
    using K = Cfg<C, S>;
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [] {
        attr_err = cudaFuncSetAttribute(nlm_window_kernel<C, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        200 * 1024);
    });
    if (attr_err != cudaSuccess) return attr_err;
    dim3 grid((a.width + kTX - 1) / kTX, (a.height + K::TY - 1) / K::TY);
    size_t smem = smem_bytes<C, S>(a.search_radius, a.pairs);
    nlm_window_kernel<C, S><<<grid, kThreads, smem, stream>>>(a);
    return cudaGetLastError();
}

template <int C, int S>
cudaError_t dispatch_s(const NlmLaunch& a, cudaStream_t stream) {
    if (a.patch_radius == S) return launch_cs<C, S>(a, stream);
    if constexpr (S < 16) {
        return dispatch_s<C, S + 1>(a, stream);
    } else {
        return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t launch_nlm(const NlmLaunch& a, cudaStream_t stream) {
    if (a.pairs < 0 || a.pairs > kMaxPairs || a.search_radius < 0 || a.search_radius > 8 || a.patch_radius < 0 ||
        a.patch_radius > 16)
        return cudaErrorInvalidValue;
    if (a.channels == 1) return dispatch_s<1, 0>(a, stream);
    if (a.channels == 2) return dispatch_s<2, 0>(a, stream);
    return cudaErrorInvalidValue;
}

}  // namespace avd
