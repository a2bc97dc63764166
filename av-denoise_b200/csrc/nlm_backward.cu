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
// Both kernels give a CTA a 32x8 tile and walk the offsets in the forward's order with the frames
// staged once in shared memory. Per offset, the squared differences over the tile plus an s halo
// are box-summed into the tile's patch distances (as the forward's separable path does). Kernel 1
// recomputes W, A, M, its argmax and the output, writes the direct centre term and keeps 5 floats
// per pixel. Kernel 2 turns each pixel's weight gradient into dL/dD, box-sums it back over the
// patch window (the adjoint of the box sum), and adds the distance terms and the weighted-sum
// term into shared-memory gradient tiles, one per window frame, which each CTA adds to global
// memory once, at the clamped pixels. dL/dh2 is reduced per CTA and summed in a fixed order.

#include <cstdint>

#include "kernels.h"

namespace avd {
namespace {

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

// Tile geometry: a CTA owns TX x TY output pixels. For every offset it stages nothing new: the
// 2d+1 frames are staged once with an (a+s) halo (clamped reads, so the inner loops never clamp),
// the squared differences are formed over the tile plus an s halo, box-summed into the patch
// distances, and (backward) the distance gradients are box-summed back over the same window.
constexpr int TX = 32, TY = 8;

struct TileGeo {
    int H, WT, HT;  // halo, staged tile width and height
    int EW, EH;     // extended (tile + s halo) width and height
};

__device__ __forceinline__ TileGeo tile_geo(const Bwd& b) {
    TileGeo g;
    g.H = b.a + b.s;
    g.WT = TX + 2 * g.H;
    g.HT = TY + 2 * g.H;
    g.EW = TX + 2 * b.s;
    g.EH = TY + 2 * b.s;
    return g;
}

size_t tile_floats(int channels, int d, int a, int s, bool backward) {
    const size_t H = a + s, WT = TX + 2 * H, HT = TY + 2 * H;
    const size_t EW = TX + 2 * s, EH = TY + 2 * s;
    const size_t frames = static_cast<size_t>(2 * d + 1) * WT * HT * channels;
    size_t n = frames + EW * EH + EH * TX;  // staged frames, squared differences, row sums
    if (backward) n += frames + TY * TX + TY * EW;  // gradient tiles, dL/dD, its row sums
    return n;
}

// PHASE 0 recomputes the forward's sums per pixel and writes the records and the direct centre
// term; PHASE 1 scatters the weight and distance gradients.
template <int C, int PHASE, int S>
__global__ void __launch_bounds__(TX* TY) bwd_tile_kernel(Bwd b) {
    extern __shared__ float sm[];
    __shared__ float red[TX * TY / 32];
    TileGeo G = tile_geo(b);
    constexpr int EW = TX + 2 * S, EH = TY + 2 * S;
    G.EW = EW;
    G.EH = EH;
    const int frames = 2 * b.d + 1;
    const int fstride = G.WT * G.HT * C;
    float* fs = sm;                                   // staged frames
    float* sq = fs + frames * fstride;                // EH x EW
    float* hs = sq + G.EH * G.EW;                     // EH x TX
    float* gs = hs + G.EH * TX;                       // gradient tiles (PHASE 1)
    float* gd = gs + (PHASE == 1 ? frames * fstride : 0);  // TY x TX
    float* bh = gd + TY * TX;                         // TY x EW
    const int t = threadIdx.x;
    const int tx = t % TX, ty = t / TX;
    const int x0 = blockIdx.x * TX - G.H, y0 = blockIdx.y * TY - G.H;  // staged tile origin
    for (int i = t; i < frames * G.WT * G.HT; i += blockDim.x) {
        const int f = i / (G.WT * G.HT), r = i % (G.WT * G.HT);
        const float* src = at<C>(b, f, x0 + r % G.WT, y0 + r / G.WT);
#pragma unroll
        for (int c = 0; c < C; ++c) {
            fs[static_cast<int64_t>(i) * C + c] = src[c];
            if (PHASE == 1) gs[static_cast<int64_t>(i) * C + c] = 0.0f;
        }
    }
    const int px = blockIdx.x * TX + tx, py = blockIdx.y * TY + ty;
    const bool inside = px < b.width && py < b.height;
    const int64_t p = static_cast<int64_t>(inside ? py : 0) * b.width + (inside ? px : 0);
    const float scale = C == 1 ? 3.0f : 1.5f;
    auto F = [&](int f, int lx, int ly) { return fs + ((static_cast<int64_t>(f) * G.HT + ly) * G.WT + lx) * C; };
    auto Gt = [&](int f, int lx, int ly) { return gs + ((static_cast<int64_t>(f) * G.HT + ly) * G.WT + lx) * C; };
    // Local coordinates of pixel p in the staged tile.
    const int plx = tx + G.H, ply = ty + G.H;

    float acc[C] = {};
    float W = 0.0f, M = 0.0f, g[C] = {}, out[C] = {}, inv = 0.0f, gm = 0.0f, gh2 = 0.0f;
    int argmax = -1;
    if (PHASE == 1 && inside) {
        const float* rec = b.records + p * kRecord;
        inv = rec[2];
        gm = rec[3];
        argmax = __float_as_int(rec[4]);
#pragma unroll
        for (int c = 0; c < C; ++c) {
            g[c] = b.grad_out[p * C + c];
            out[c] = rec[c];
        }
    }
    const bool active = inside && (PHASE == 0 || inv != 0.0f);
    // The centre-frame gradient of the extended-grid cells this thread owns (ey = ty + j TY,
    // ex = tx + i TX), kept in registers across the offsets.
    constexpr int kOwnRows = (EH + TY - 1) / TY, kOwnCols = (EW + TX - 1) / TX;
    float gcen[kOwnRows * kOwnCols][C];
#pragma unroll
    for (int i = 0; i < kOwnRows * kOwnCols; ++i)
#pragma unroll
        for (int c = 0; c < C; ++c) gcen[i][c] = 0.0f;
    __syncthreads();

    for_offsets(b, [&](int id, int f, int qx, int qy, float off) {
        // (a) squared differences over the tile plus an s halo (virtual positions).
#pragma unroll
        for (int ey = ty; ey < EH; ey += TY)
#pragma unroll
            for (int ex = tx; ex < EW; ex += TX) {
                const int lx = ex - S + G.H, ly = ey - S + G.H;
                const float* cc = F(b.d, lx, ly);
                const float* nn = F(f, lx + qx, ly + qy);
                float l = 0.0f;
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    const float diff = cc[c] - nn[c];
                    l += diff * diff;
                }
                sq[ey * EW + ex] = l * scale;
            }
        __syncthreads();
        // (b) horizontal patch sums.
#pragma unroll
        for (int ey = ty; ey < EH; ey += TY) {
            float r = 0.0f;
#pragma unroll
            for (int k = 0; k <= 2 * S; ++k) r += sq[ey * EW + tx + k];
            hs[ey * TX + tx] = r;
        }
        __syncthreads();
        // (c) the distance and weight of this thread's pixel.
        float dist = 0.0f;
#pragma unroll
        for (int k = 0; k <= 2 * S; ++k) dist += hs[(ty + k) * TX + tx];
        const float w = welsch(dist, b.h2, off);
        const float* nq = F(f, plx + qx, ply + qy);
        if (PHASE == 0) {
            if (active) {
#pragma unroll
                for (int c = 0; c < C; ++c) acc[c] += w * nq[c];
                W += w;
                if (w > M) {
                    M = w;
                    argmax = id;
                }
            }
            return;  // the next offset's (a) writes `sq` only after its own barrier below
        }
        float gdd = 0.0f;
        if (active) {
            float gw = id == argmax ? gm : 0.0f;
            float* an = Gt(f, plx + qx, ply + qy);
#pragma unroll
            for (int c = 0; c < C; ++c) {
                gw += g[c] * (nq[c] - out[c]) * inv;
                an[c] += g[c] * w * inv;  // p -> p + q is one-to-one: one writer per cell
            }
            const float excess = dist - off;
            if (excess > 0.0f && w > 0.0f) {
                gh2 -= gw * excess * w;
                gdd = -gw * b.h2 * w * 2.0f * scale;
            }
        }
        gd[ty * TX + tx] = gdd;
        __syncthreads();
        // (d) horizontal box of dL/dD onto the extended grid: v sees every owned p within s.
#pragma unroll
        for (int ex = tx; ex < EW; ex += TX) {
            float v = 0.0f;
#pragma unroll
            for (int k = 0; k <= 2 * S; ++k) {
                const int cx = ex - k;
                if (cx >= 0 && cx < TX) v += gd[ty * TX + cx];
            }
            bh[ty * EW + ex] = v;
        }
        __syncthreads();
        // (e) vertical box, then the distance terms into both frames' gradient tiles.
#pragma unroll
        for (int ey = ty; ey < EH; ey += TY)
#pragma unroll
            for (int ex = tx; ex < EW; ex += TX) {
            float B = 0.0f;
#pragma unroll
            for (int k = 0; k <= 2 * S; ++k) {
                const int r = ey - k;
                if (r >= 0 && r < TY) B += bh[r * EW + ex];
            }
            if (B == 0.0f) continue;
            const int lx = ex - S + G.H, ly = ey - S + G.H;
            const float* cc = F(b.d, lx, ly);
            const float* nn = F(f, lx + qx, ly + qy);
            // One writer per cell and offset: the centre term stays in this thread's registers,
            // and v -> v + q is one-to-one on the virtual grid.
            float* gn = Gt(f, lx + qx, ly + qy);
            const int slot = ((ey - ty) / TY) * ((EW + TX - 1) / TX) + (ex - tx) / TX;
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const float term = B * (cc[c] - nn[c]);
                gcen[slot][c] += term;
                gn[c] -= term;
            }
        }
        __syncthreads();
    });
    if (PHASE == 0) {
        if (!inside) return;
        const float* I = F(b.d, plx, ply);
        const float* gp = b.grad_out + p * C;
        float* gc = b.grad_window + b.d * b.frame_elems + p * C;
        float* rec = b.records + p * kRecord;
        const float den = b.wref * M + W;
        if (!(den > 1e-30f)) {
#pragma unroll
            for (int c = 0; c < C; ++c) {
                gc[c] = gp[c];
                rec[c] = I[c];
            }
            rec[2] = 0.0f;
            rec[3] = 0.0f;
            rec[4] = __int_as_float(-1);
            return;
        }
        const float iv = 1.0f / den;
        float g_m = 0.0f, o[2] = {0.0f, 0.0f};
#pragma unroll
        for (int c = 0; c < C; ++c) {
            o[c] = (I[c] * b.wref * M + acc[c]) * iv;
            gc[c] = gp[c] * b.wref * M * iv;
            g_m += gp[c] * b.wref * (I[c] - o[c]) * iv;
        }
        rec[0] = o[0];
        rec[1] = o[1];
        rec[2] = iv;
        rec[3] = g_m;
        rec[4] = __int_as_float(argmax);
        return;
    }
    // The owned centre-frame cells join the tile (every offset's barrier has passed).
#pragma unroll
    for (int j = 0; j < kOwnRows; ++j)
#pragma unroll
        for (int i = 0; i < kOwnCols; ++i) {
            const int ey = ty + j * TY, ex = tx + i * TX;
            if (ey >= EH || ex >= EW) continue;
            float* gc = Gt(b.d, ex - S + G.H, ey - S + G.H);
#pragma unroll
            for (int c = 0; c < C; ++c) gc[c] += gcen[j * kOwnCols + i][c];
        }
    __syncthreads();
    for (int o = 16; o > 0; o >>= 1) gh2 += __shfl_xor_sync(0xffffffffu, gh2, o);
    if ((t & 31) == 0) red[t >> 5] = gh2;
    __syncthreads();
    if (t == 0) {
        float total = 0.0f;
        for (int i = 0; i < TX * TY / 32; ++i) total += red[i];
        b.partials[blockIdx.y * gridDim.x + blockIdx.x] = total;
    }
    // Flush: each staged position adds into its clamped pixel (border duplicates fold there).
    for (int i = t; i < frames * G.WT * G.HT; i += blockDim.x) {
        const int f = i / (G.WT * G.HT), r = i % (G.WT * G.HT);
        const int gx = clampi(x0 + r % G.WT, b.width), gy = clampi(y0 + r / G.WT, b.height);
        float* dst = b.grad_window + f * b.frame_elems + (static_cast<int64_t>(gy) * b.width + gx) * C;
#pragma unroll
        for (int c = 0; c < C; ++c) {
            const float v = gs[static_cast<int64_t>(i) * C + c];
            if (v != 0.0f) atomicAdd(dst + c, v);
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
    const size_t tiles = static_cast<size_t>((width + TX - 1) / TX) * ((height + TY - 1) / TY);
    return static_cast<size_t>(width) * height * kRecord + tiles;
}

size_t nlm_backward_smem_bytes(int channels, int temporal_radius, int search_radius, int patch_radius) {
    return tile_floats(channels, temporal_radius, search_radius, patch_radius, true) * sizeof(float);
}

template <int C, int S>
cudaError_t launch_tiles_s(const Bwd& b, dim3 grid, cudaStream_t s) {
    const size_t fwd = tile_floats(C, b.d, b.a, b.s, false) * sizeof(float);
    const size_t bwd = tile_floats(C, b.d, b.a, b.s, true) * sizeof(float);
    cudaFuncSetAttribute(bwd_tile_kernel<C, 0, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(fwd));
    cudaFuncSetAttribute(bwd_tile_kernel<C, 1, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bwd));
    bwd_tile_kernel<C, 0, S><<<grid, TX * TY, fwd, s>>>(b);
    bwd_tile_kernel<C, 1, S><<<grid, TX * TY, bwd, s>>>(b);
    return cudaGetLastError();
}

template <int C, int S = 0>
cudaError_t launch_tiles(const Bwd& b, dim3 grid, cudaStream_t s) {
    if constexpr (S <= 16) {
        if (b.s == S) return launch_tiles_s<C, S>(b, grid, s);
        return launch_tiles<C, S + 1>(b, grid, s);
    } else {
        return cudaErrorInvalidValue;
    }
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
    dim3 grid((l.width + TX - 1) / TX, (l.height + TY - 1) / TY);
    e = l.channels == 1 ? launch_tiles<1>(b, grid, s) : launch_tiles<2>(b, grid, s);
    if (e != cudaSuccess) return e;
    bwd_strength_kernel<<<1, 32, 0, s>>>(b.partials, static_cast<int>(grid.x * grid.y), l.h2, l.strength,
                                         l.grad_strength);
    return cudaGetLastError();
}

namespace {
__global__ void window_words_kernel(float* words, float h2, float pair_offset, float spatial_offset, int a) {
    const int side = 2 * a + 1;
    for (int i = threadIdx.x; i < side * side; i += blockDim.x)
        words[8 + i] = i == a * side + a ? 0.0f : spatial_offset;
    if (threadIdx.x == 0) {
        words[0] = h2;
        words[1] = pair_offset;
    }
}
}  // namespace

cudaError_t launch_window_words(float* words, float h2, float pair_offset, float spatial_offset, int a,
                                cudaStream_t s) {
    window_words_kernel<<<1, 128, 0, s>>>(words, h2, pair_offset, spatial_offset, a);
    return cudaGetLastError();
}

}  // namespace avd
