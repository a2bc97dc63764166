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
// Both kernels run on the forward's tile (nlm_tile.cuh): a CTA of 128 threads owns a 32 x TY tile,
// the frames are staged in shared memory once per pass, and each step takes two offsets (lanes) in
// packed f32x2 arithmetic with the forward's row-run / column-strip box sums.
//  - The record kernel is the forward tile with the max weight's first offset tracked: it writes
//    per pixel out, 1/den, dL/dM and that offset, and the centre pixel's direct term.
//  - The gradient kernel recomputes each step's distances and weights (phases 1-2, as the forward),
//    turns each pixel's weight gradient into dL/dD and scatters the weighted-sum term into the
//    neighbour frame's shared gradient tile, then box-sums dL/dD back over the patch window on the
//    tile plus its s halo (phase 3 vertical, phase 4 horizontal) and adds the distance terms: the
//    centre frame's into registers each thread owns for the whole kernel, the neighbour frame's into
//    its shared tile. A pass's tiles are added to global memory once, at the clamped pixels.
// dL/dh2 is reduced per CTA and summed in a fixed order.

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <type_traits>

#include "kernels.h"
#include "nlm_tile.cuh"

namespace avd {
namespace {

using namespace nlm_tile_detail;


template <int C, int S>
size_t record_smem_bytes(int A, int pairs) {
    using K = Cfg<C, S>;
    const int nrows = K::TY + 2 * S + 2 * A, ncols = kTX + 2 * S + 2 * A;
    const int nstride = nbr_stride(ncols, C);
    const size_t floats = (size_t)round_up4(K::CROWS * K::CSTRIDE) +
                          (size_t)round_up4((pairs > 0 ? 2 : 1) * nrows * nstride) + (size_t)2 * K::HS_BUF;
    return floats * sizeof(float);
}

template <int C, int S>
size_t grad_smem_bytes(int A) {
    using K = Cfg<C, S>;
    const int nrows = K::TY + 2 * S + 2 * A, ncols = kTX + 2 * S + 2 * A;
    const int nstride = nbr_stride(ncols, C);
    const size_t tile = (size_t)round_up4(nrows * nstride);
    constexpr int RPS = (K::TY + 2 * S + 3) / 4;  // extended rows per column strip
    const size_t floats = (size_t)round_up4(K::CROWS * K::CSTRIDE) + 4 * tile + (size_t)K::HR * kHsStride +
                          (size_t)2 * (2 * S + 1 + 4 * RPS) * kTX + (size_t)2 * 4 * RPS * (kTX + 4 * S);
    return floats * sizeof(float);
}

template <int C, int S, bool FAST>
__global__ void __launch_bounds__(kThreads) nlm_record_kernel(NlmLaunch a, RecordOut r) {
    nlm_tile<C, S, FAST, true>(a, blockIdx.x, blockIdx.y, &r);
}

struct GradArgs {
    NlmLaunch a;  // the window as a ring: centre slot d, pair k's frames k and 2d - k
    const float* grad_out;
    const float* records;
    float* grad_window;
    float* partials;  // one per tile
    float h2;
};

// Per-pixel values of the outputs a thread owns, from the records.
template <int C, int V>
struct PixelGrad {
    float gamma[C][V];  // dL/dout_c / den
    float out[C][V];
    float gm[V];        // dL/dM
    int arg[V];         // the max weight's first offset id
    bool active[V];
};

// dL/dM reaches the offset that set the max weight.
template <int C, int V>
__device__ __forceinline__ float ln_gm(const PixelGrad<C, V>& pg, int k, int id) {
    return id == pg.arg[k] ? pg.gm[k] : 0.0f;
}

// Adds a pass's gradient tile into a frame's gradient, at the clamped pixels the tile was staged
// from (border duplicates fold onto the edge pixels).
template <int C>
__device__ void flush_tile(const float* tile, int stride, int rows, int cols, float* grad_frame, int x0, int y0, int W,
                           int H) {
    for (int i = threadIdx.x; i < rows * cols; i += kThreads) {
        const int r = i / cols, c = i - r * cols;
        const int gx = clampi(x0 + c, 0, W - 1), gy = clampi(y0 + r, 0, H - 1);
        float* dst = grad_frame + ((int64_t)gy * W + gx) * C;
#pragma unroll
        for (int ch = 0; ch < C; ++ch) {
            const float v = tile[r * stride + c * C + ch];
            if (v != 0.0f) atomicAdd(dst + ch, v);
        }
    }
}

template <bool ATOMIC>
__device__ __forceinline__ void add_to(float* p, float v) {
    if constexpr (ATOMIC)
        atomicAdd(p, v);
    else
        *p += v;
}

template <int C, int S, bool FAST>
__global__ void __launch_bounds__(kThreads) nlm_grad_kernel(GradArgs g) {
    using K = Cfg<C, S>;
    constexpr int V = K::V;
    constexpr int EH = K::TY + 2 * S;  // extended rows: the tile plus its s halo
    constexpr int RPS = (EH + 3) / 4;  // extended rows per column strip
    // The 2s halo columns right of the tile's 32 (ex = 32 + m) are spread over all 128 threads:
    // cell e = tid + 128 i is (ey = e / 2s, ex = 32 + e % 2s).
    constexpr int kHaloCells = 2 * S * EH;
    constexpr int NX = (kHaloCells + kThreads - 1) / kThreads;

    const NlmLaunch& a = g.a;
    const int A = a.search_radius;
    const int W = a.width, H = a.height;
    const int X0 = blockIdx.x * kTX, Y0 = blockIdx.y * K::TY;
    const int tid = threadIdx.x, col = tid & 31, strip = tid >> 5;
    const int y0 = strip * V;
    const int side = 2 * A + 1;

    const int nrows = K::TY + 2 * S + 2 * A, ncols = kTX + 2 * S + 2 * A;
    const int nstride = nbr_stride(ncols, C);
    const int tile_floats = round_up4(nrows * nstride);
    float* ctr = smem_raw;
    float* nbr0 = ctr + round_up4(K::CROWS * K::CSTRIDE);
    float* nbr1 = nbr0 + tile_floats;
    float* gt0 = nbr1 + tile_floats;
    float* gt1 = gt0 + tile_floats;
    float* hs = gt1 + tile_floats;                              // HR x kHsStride
    // dL/dD * 2 scale per tile row and lane pair, rows -ETOP..-1 and TY..4 RPS - 1 held at zero so the
    // vertical box reads them unguarded; then its vertical box on the extended rows, each row padded
    // with 2s zero lane pairs on both sides so the horizontal box reads them unguarded.
    constexpr int ETOP = 2 * S + 1;
    constexpr int GVW = kTX + 4 * S;
    float2* et_raw = reinterpret_cast<float2*>(hs + K::HR * kHsStride);
    float2* et = et_raw + ETOP * kTX;
    float2* gv = et_raw + (ETOP + 4 * RPS) * kTX;
    for (int i = tid; i < (ETOP + 4 * RPS) * kTX + 4 * RPS * GVW; i += kThreads) et_raw[i] = f2(0.0f, 0.0f);

    const float h2 = g.h2;
    const float off_pair = __ldg(a.derived + a.offset_word);
    const float scale = C == 1 ? 3.0f : 1.5f;
    const float neg_h2_log2e = -h2 * kLog2e;
    const float2 kk = FAST ? f2(scale * neg_h2_log2e, scale * neg_h2_log2e) : f2(neg_h2_log2e, neg_h2_log2e);
    const float2 scale2 = f2(scale, scale);
    const float e_scale = -h2 * 2.0f * scale;

    const float* centre = a.ring + a.slot_centre * a.frame_elems;
    load_tile<C>(ctr, K::CSTRIDE, K::CROWS, K::CW, centre, X0 - S, Y0 - S, W, H);

    PixelGrad<C, V> pg;
#pragma unroll
    for (int k = 0; k < V; ++k) {
        const int gx = X0 + col, gy = Y0 + y0 + k;
        pg.active[k] = false;
        pg.gm[k] = 0.0f;
        pg.arg[k] = -1;
#pragma unroll
        for (int c = 0; c < C; ++c) {
            pg.gamma[c][k] = 0.0f;
            pg.out[c][k] = 0.0f;
        }
        if (gx < W && gy < H) {
            const int64_t px = (int64_t)gy * W + gx;
            const float* r = g.records + px * kRecordWords;
            const float inv = r[2];
            pg.active[k] = inv != 0.0f;
            pg.gm[k] = r[3];
            pg.arg[k] = __float_as_int(r[4]);
#pragma unroll
            for (int c = 0; c < C; ++c) {
                pg.gamma[c][k] = g.grad_out[px * C + c] * inv;
                pg.out[c][k] = r[c];
            }
        }
    }
    // The centre frame's distance gradient on the extended cells this thread owns: column col of
    // rows RPS strip .. RPS strip + RPS - 1, and its halo cells.
    float gcen[RPS][C];
    float gext[NX > 0 ? NX : 1][C];
#pragma unroll
    for (int i = 0; i < RPS; ++i)
#pragma unroll
        for (int c = 0; c < C; ++c) gcen[i][c] = 0.0f;
#pragma unroll
    for (int i = 0; i < (NX > 0 ? NX : 1); ++i)
#pragma unroll
        for (int c = 0; c < C; ++c) gext[i][c] = 0.0f;
    float gh2 = 0.0f;
    __syncthreads();

    CentreRun<C, S> crun;
    if (K::CTR_REG) {
        const int r = ((tid >> 5) << 3) + (tid & 7);
        const int x0 = ((tid >> 3) & 3) * kRun;
        crun.load(ctr + min(r, K::CROWS - 1) * K::CSTRIDE + x0 * C);
    }

    // One step: two offsets (lanes) against the staged tiles t0 / t1, their gradient tiles g0 / g1.
    // `atomic_tag` (std::true_type or std::false_type): whether the two lanes may scatter into the
    // same gradient tile (the single-frame pass) and so add with shared atomics.
    auto grad_step = [&](auto atomic_tag, const float* t0, const float* t1, float* g0, float* g1, int dx0, int dy0,
                         int dx1, int dy1, int id0, int id1, float2 negoff) {
        constexpr bool kAtomic = decltype(atomic_tag)::value;
        // Phase 1: the row box sums of both lanes' squared differences (the forward's).
        for (int slot = tid; slot < K::TASK_SLOTS; slot += kThreads) {
            const int r = ((slot >> 5) << 3) + (slot & 7);
            if (r >= K::HR) continue;
            const int x0 = ((slot >> 3) & 3) * kRun;
            const float* n0 = t0 + (r + dy0 + A) * nstride + (x0 + dx0 + A) * C;
            const float* n1 = t1 + (r + dy1 + A) * nstride + (x0 + dx1 + A) * C;
            if (K::CTR_REG) {
                row_run<C, S>(crun, n0, n1, hs + r * kHsStride + 2 * x0);
            } else {
                CentreRun<C, S> c;
                c.load(ctr + r * K::CSTRIDE + x0 * C);
                row_run<C, S>(c, n0, n1, hs + r * kHsStride + 2 * x0);
            }
        }
        __syncthreads();
        // Phase 2: distances, weights, dL/dw, the weighted-sum term, dL/dD.
        {
            float2 hv[V + 2 * S];
#pragma unroll
            for (int i = 0; i < V + 2 * S; ++i) hv[i] = *reinterpret_cast<const float2*>(hs + (y0 + i) * kHsStride + 2 * col);
            float2 dist = hv[0];
#pragma unroll
            for (int i = 1; i <= 2 * S; ++i) dist = add2(dist, hv[i]);
            const int c0 = (y0 + S + dy0 + A) * nstride + (col + S + dx0 + A) * C;
            const int c1 = (y0 + S + dy1 + A) * nstride + (col + S + dx1 + A) * C;
#pragma unroll
            for (int k = 0; k < V; ++k) {
                if (k > 0) dist = sub2(add2(dist, hv[k + 2 * S]), hv[k - 1]);
                float2 x, w;
                if (FAST) {
                    x = mul2(dist, scale2);
                    const float2 e = mul2(dist, kk);
                    w = f2(ex2_approx(e.x), ex2_approx(e.y));
                } else {
                    x = fma2(dist, scale2, negoff);
                    const float2 e = mul2(f2(fmaxf(x.x, 0.0f), fmaxf(x.y, 0.0f)), kk);
                    w = f2(ex2_approx(e.x), ex2_approx(e.y));
                }
                float2 E = f2(0.0f, 0.0f);
                if (pg.active[k]) {
                    const int i0 = c0 + k * nstride, i1 = c1 + k * nstride;
                    float gw0 = ln_gm(pg, k, id0), gw1 = ln_gm(pg, k, id1);
#pragma unroll
                    for (int c = 0; c < C; ++c) {
                        gw0 += pg.gamma[c][k] * (t0[i0 + c] - pg.out[c][k]);
                        gw1 += pg.gamma[c][k] * (t1[i1 + c] - pg.out[c][k]);
                        add_to<kAtomic>(g0 + i0 + c, pg.gamma[c][k] * w.x);
                        add_to<kAtomic>(g1 + i1 + c, pg.gamma[c][k] * w.y);
                    }
                    if (x.x > 0.0f && w.x > 0.0f) {
                        E.x = gw0 * w.x * e_scale;
                        gh2 -= gw0 * x.x * w.x;
                    }
                    if (x.y > 0.0f && w.y > 0.0f) {
                        E.y = gw1 * w.y * e_scale;
                        gh2 -= gw1 * x.y * w.y;
                    }
                }
                et[(y0 + k) * kTX + col] = E;
            }
        }
        __syncthreads();
        // Phase 3: the vertical box of dL/dD onto this strip's extended rows.
        {
            const int e0 = strip * RPS;
            const float2* ec = et + e0 * kTX + col;
            float2 sum = ec[-2 * S * kTX];
#pragma unroll
            for (int r = 1 - 2 * S; r <= 0; ++r) sum = add2(sum, ec[r * kTX]);
            float2* gc = gv + e0 * GVW + 2 * S + col;
#pragma unroll
            for (int i = 0; i < RPS; ++i) {
                if (e0 + i >= EH) break;
                if (i > 0) sum = sub2(add2(sum, ec[i * kTX]), ec[(i - 2 * S - 1) * kTX]);
                gc[i * GVW] = sum;
            }
        }
        __syncthreads();
        // Phase 4: the horizontal box, then the distance terms of both lanes at one extended cell.
        auto cell = [&](int ey, int ex, float* acc) {
            const float2* gr = gv + ey * GVW + ex;  // padded columns ex .. ex + 2s hold lane pairs ex - 2s .. ex
            float2 G = gr[2 * S];
#pragma unroll
            for (int u = 2 * S - 1; u >= 0; --u) G = add2(G, gr[u]);
            if (G.x == 0.0f && G.y == 0.0f) return;
            const float* cc = ctr + ey * K::CSTRIDE + ex * C;
            const int i0 = (ey + dy0 + A) * nstride + (ex + dx0 + A) * C;
            const int i1 = (ey + dy1 + A) * nstride + (ex + dx1 + A) * C;
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const float term0 = G.x * (cc[c] - t0[i0 + c]);
                const float term1 = G.y * (cc[c] - t1[i1 + c]);
                acc[c] += term0 + term1;
                add_to<kAtomic>(g0 + i0 + c, -term0);
                add_to<kAtomic>(g1 + i1 + c, -term1);
            }
        };
#pragma unroll
        for (int i = 0; i < RPS; ++i) {
            const int ey = strip * RPS + i;
            if (ey < EH) cell(ey, col, gcen[i]);
        }
        if constexpr (S > 0) {
#pragma unroll
            for (int i = 0; i < NX; ++i) {
                const int e = tid + i * kThreads;
                if (e < kHaloCells) cell(e / (2 * S), kTX + e % (2 * S), gext[i]);
            }
        }
    };

    const int nelem = nrows * nstride;
    for (int p = 0; p < a.pairs; ++p) {
        __syncthreads();  // every thread is done with the previous pass's tiles
        load_tile<C>(nbr0, nstride, nrows, ncols, a.ring + a.slot_fwd[p] * a.frame_elems, X0 - S - A, Y0 - S - A, W, H);
        load_tile<C>(nbr1, nstride, nrows, ncols, a.ring + a.slot_bwd[p] * a.frame_elems, X0 - S - A, Y0 - S - A, W, H);
        for (int i = tid; i < nelem; i += kThreads) {
            gt0[i] = 0.0f;
            gt1[i] = 0.0f;
        }
        __syncthreads();
        const float2 negoff = f2(-off_pair, -off_pair);
        for (int qy = -A; qy <= A; ++qy)
            for (int qx = -A; qx <= A; ++qx) {
                const int id0 = 2 * ((p * side + qy + A) * side + qx + A);
                // Each lane scatters into its own frame's tile, one cell per pixel: no atomics.
                grad_step(std::false_type{}, nbr0, nbr1, gt0, gt1, qx, qy, -qx, -qy, id0, id0 + 1, negoff);
            }
        __syncthreads();
        flush_tile<C>(gt0, nstride, nrows, ncols, g.grad_window + a.slot_fwd[p] * a.frame_elems, X0 - S - A,
                      Y0 - S - A, W, H);
        flush_tile<C>(gt1, nstride, nrows, ncols, g.grad_window + a.slot_bwd[p] * a.frame_elems, X0 - S - A,
                      Y0 - S - A, W, H);
    }

    // The single-frame pass: both lanes read and scatter into the centre frame's tile.
    __syncthreads();
    load_tile<C>(nbr0, nstride, nrows, ncols, centre, X0 - S - A, Y0 - S - A, W, H);
    for (int i = tid; i < nelem; i += kThreads) gt0[i] = 0.0f;
    __syncthreads();
    {
        const int n = side * side - 1;
        const int mid = A * side + A;
        const int spatial_base = 2 * a.pairs * side * side;
        for (int i = 0; i < n; i += 2) {
            const int l0 = i < mid ? i : i + 1;
            const int l1 = i + 1 < mid ? i + 1 : i + 2;
            float2 negoff = f2(0.0f, 0.0f);
            if (!FAST && a.spatial_lut) negoff = f2(-__ldg(a.spatial_lut + l0), -__ldg(a.spatial_lut + l1));
            grad_step(std::true_type{}, nbr0, nbr0, gt0, gt0, l0 % side - A, l0 / side - A, l1 % side - A, l1 / side - A,
                      spatial_base + i, spatial_base + i + 1, negoff);
        }
    }
    __syncthreads();
    float* grad_centre = g.grad_window + a.slot_centre * a.frame_elems;
    flush_tile<C>(gt0, nstride, nrows, ncols, grad_centre, X0 - S - A, Y0 - S - A, W, H);
    // The owned centre cells, at their clamped pixels.
    auto flush_cell = [&](int ey, int ex, const float* acc) {
        const int gx = clampi(X0 - S + ex, 0, W - 1), gy = clampi(Y0 - S + ey, 0, H - 1);
        float* dst = grad_centre + ((int64_t)gy * W + gx) * C;
#pragma unroll
        for (int c = 0; c < C; ++c)
            if (acc[c] != 0.0f) atomicAdd(dst + c, acc[c]);
    };
#pragma unroll
    for (int i = 0; i < RPS; ++i) {
        const int ey = strip * RPS + i;
        if (ey < EH) flush_cell(ey, col, gcen[i]);
    }
    if constexpr (S > 0) {
#pragma unroll
        for (int i = 0; i < NX; ++i) {
            const int e = tid + i * kThreads;
            if (e < kHaloCells) flush_cell(e / (2 * S), kTX + e % (2 * S), gext[i]);
        }
    }
    // dL/dh2 of the tile, summed in a fixed order.
    __shared__ float red[kThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) gh2 += __shfl_xor_sync(0xffffffffu, gh2, o);
    if ((tid & 31) == 0) red[tid >> 5] = gh2;
    __syncthreads();
    if (tid == 0) {
        float total = 0.0f;
        for (int i = 0; i < kThreads / 32; ++i) total += red[i];
        g.partials[blockIdx.y * gridDim.x + blockIdx.x] = total;
    }
}

__global__ void strength_kernel(const float* partials, int n, float h2, float strength, float* grad_strength) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float total = 0.0f;
    for (int i = 0; i < n; ++i) total += partials[i];
    // h2 = K / strength^2, so dh2/dstrength = -2 h2 / strength.
    *grad_strength = total * (-2.0f * h2 / strength);
}

__global__ void window_words_kernel(float* words, float h2, float pair_offset, float spatial_offset, int a) {
    const int side = 2 * a + 1;
    for (int i = threadIdx.x; i < side * side; i += blockDim.x)
        words[8 + i] = i == a * side + a ? 0.0f : spatial_offset;
    if (threadIdx.x == 0) {
        words[0] = h2;
        words[1] = pair_offset;
    }
}

constexpr int kWordFloats = 8 + 17 * 17;

int tiles_for(int width, int height, int patch_radius) {
    const int v = (32 - 2 * patch_radius) / 4;
    const int ty = 4 * (v >= 1 ? v : 1);
    return ((width + kTX - 1) / kTX) * ((height + ty - 1) / ty);
}

template <int C, int S>
cudaError_t launch_adjoint_s(const NlmLaunch& a, const RecordOut& rec, const GradArgs& g, cudaStream_t s) {
    using K = Cfg<C, S>;
    const dim3 grid((a.width + kTX - 1) / kTX, (a.height + K::TY - 1) / K::TY);
    const size_t rbytes = record_smem_bytes<C, S>(a.search_radius, a.pairs);
    const size_t gbytes = grad_smem_bytes<C, S>(a.search_radius);
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        for (auto f : {nlm_record_kernel<C, S, true>, nlm_record_kernel<C, S, false>})
            if (attr == cudaSuccess)
                attr = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        for (auto f : {nlm_grad_kernel<C, S, true>, nlm_grad_kernel<C, S, false>})
            if (attr == cudaSuccess)
                attr = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 226 * 1024);
    });
    if (attr != cudaSuccess) return attr;
    if (a.fast) {
        nlm_record_kernel<C, S, true><<<grid, kThreads, rbytes, s>>>(a, rec);
        nlm_grad_kernel<C, S, true><<<grid, kThreads, gbytes, s>>>(g);
    } else {
        nlm_record_kernel<C, S, false><<<grid, kThreads, rbytes, s>>>(a, rec);
        nlm_grad_kernel<C, S, false><<<grid, kThreads, gbytes, s>>>(g);
    }
    return cudaGetLastError();
}

template <int C, int S = 0>
cudaError_t dispatch_adjoint(const NlmLaunch& a, const RecordOut& rec, const GradArgs& g, cudaStream_t s) {
    if constexpr (S <= 16) {
        if (a.patch_radius == S) return launch_adjoint_s<C, S>(a, rec, g, s);
        return dispatch_adjoint<C, S + 1>(a, rec, g, s);
    } else {
        return cudaErrorInvalidValue;
    }
}

}  // namespace

size_t nlm_backward_scratch_floats(int width, int height) {
    // Records, the words, and one dL/dh2 partial per tile of the smallest tile height.
    return static_cast<size_t>(width) * height * kRecordWords + kWordFloats + tiles_for(width, height, 16);
}

size_t nlm_backward_smem_bytes(int channels, int /*temporal_radius*/, int search_radius, int patch_radius) {
    // The gradient kernel's staging (the record kernel's is smaller).
    const int v = (32 - 2 * patch_radius) / 4;
    const int ty = 4 * (v >= 1 ? v : 1);
    const int nrows = ty + 2 * patch_radius + 2 * search_radius;
    const int ncols = kTX + 2 * patch_radius + 2 * search_radius;
    const int nstride = nbr_stride(ncols, channels);
    const int cw = kTX + 2 * patch_radius, crows = ty + 2 * patch_radius;
    const int rps = (ty + 2 * patch_radius + 3) / 4;
    const size_t floats = (size_t)round_up4(crows * nbr_stride(cw, channels)) + 4 * (size_t)round_up4(nrows * nstride) +
                          (size_t)(ty + 2 * patch_radius) * kHsStride +
                          (size_t)2 * (2 * patch_radius + 1 + 4 * rps) * kTX +
                          (size_t)2 * 4 * rps * (kTX + 4 * patch_radius);
    return floats * sizeof(float);
}

cudaError_t launch_nlm_backward(const NlmBackwardLaunch& l, cudaStream_t s) {
    if (l.temporal_radius < 0 || l.temporal_radius > kMaxPairs || l.search_radius < 0 || l.search_radius > 8 ||
        l.patch_radius < 0 || l.patch_radius > 16 || l.channels < 1 || l.channels > 2)
        return cudaErrorInvalidValue;
    const int d = l.temporal_radius;
    const int64_t frame_elems = static_cast<int64_t>(l.width) * l.height * l.channels;
    float* records = l.scratch;
    float* words = records + static_cast<size_t>(l.width) * l.height * kRecordWords;
    float* partials = words + kWordFloats;
    cudaError_t e = cudaMemsetAsync(l.grad_window, 0, static_cast<size_t>(2 * d + 1) * frame_elems * sizeof(float), s);
    if (e != cudaSuccess) return e;
    window_words_kernel<<<1, 128, 0, s>>>(words, l.h2, l.pair_offset, l.spatial_offset, l.search_radius);
    NlmLaunch a{};
    a.ring = l.window;
    a.width = l.width;
    a.height = l.height;
    a.channels = l.channels;
    a.frame_elems = frame_elems;
    a.slot_centre = d;
    a.pairs = d;
    for (int k = 0; k < d; ++k) {
        a.slot_fwd[k] = k;
        a.slot_bwd[k] = 2 * d - k;
    }
    a.patch_radius = l.patch_radius;
    a.search_radius = l.search_radius;
    a.derived = words;
    a.h2_word = 0;
    a.offset_word = 1;
    a.spatial_lut = words + 8;
    a.conf = nullptr;
    a.wref = l.wref;
    a.fast = (l.pair_offset == 0.0f && l.spatial_offset == 0.0f) ? 1 : 0;
    a.out = nullptr;
    RecordOut rec{l.grad_out, records, l.grad_window + d * frame_elems};
    GradArgs g{a, l.grad_out, records, l.grad_window, partials, l.h2};
    e = l.channels == 1 ? dispatch_adjoint<1>(a, rec, g, s) : dispatch_adjoint<2>(a, rec, g, s);
    if (e != cudaSuccess) return e;
    strength_kernel<<<1, 32, 0, s>>>(partials, tiles_for(l.width, l.height, l.patch_radius), l.h2, l.strength,
                                     l.grad_strength);
    return cudaGetLastError();
}

cudaError_t launch_window_words(float* words, float h2, float pair_offset, float spatial_offset, int a,
                                cudaStream_t s) {
    window_words_kernel<<<1, 128, 0, s>>>(words, h2, pair_offset, spatial_offset, a);
    return cudaGetLastError();
}

}  // namespace avd
