// The NLMeans window tile shared by the forward (nlm.cu) and its adjoint (nlm_adjoint.cu): tile
// geometry, shared-memory staging, the two-lane row-run / column-strip step and the whole tile
// (see nlm.cu for what it computes and how it maps to the SM).

#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.h"

namespace avd {
namespace nlm_tile_detail {

constexpr int kTX = 32;        // tile columns
constexpr int kThreads = 128;  // 4 warps: 32 columns x 4 strips
constexpr int kRun = 8;        // phase-1 run length
constexpr float kLog2e = 1.4426950408889634f;

// Shared-memory strides are chosen so no phase reads or writes conflict in the banks:
//  - phase 1 gives lane l the row (l & 7) and the run (l >> 3) of its warp's 8-row group, so a
//    scalar (or float2, for two channels) read of a neighbour tile hits 32 distinct banks when
//    the neighbour row stride, in pixels, is odd;
//  - the row-sum tile is written as float4 by 8 rows at a time and read as float2 along a row,
//    which is conflict free when its row stride is 4 x an odd number of floats.
__host__ __device__ constexpr int round_up4(int v) { return (v + 3) & ~3; }
__host__ __device__ constexpr int stride_4odd(int v) {
    return (round_up4(v) / 4) % 2 ? round_up4(v) : round_up4(v) + 4;
}
__host__ __device__ constexpr int nbr_stride(int cols, int c) { return c * (cols | 1); }

constexpr int kHsStride = stride_4odd(2 * kTX);  // 68 floats: 32 lane pairs per row-sum row

template <int C, int S>
struct Cfg {
    static constexpr int V = (32 - 2 * S) / 4 >= 1 ? (32 - 2 * S) / 4 : 1;  // outputs per column strip
    static constexpr int TY = 4 * V;                                       // tile rows
    static constexpr int HR = TY + 2 * S;                                  // row-sum rows
    static constexpr int TASK_SLOTS = (HR + 7) / 8 * 32;                   // phase-1 tasks (8-row groups)
    static constexpr bool CTR_REG = C == 1 && TASK_SLOTS <= kThreads;      // centre run kept in registers
    static constexpr int CW = kTX + 2 * S;                                 // centre tile columns
    static constexpr int CSTRIDE = nbr_stride(CW, C);                      // floats per centre row
    static constexpr int CROWS = TY + 2 * S;
    static constexpr int RUNW = kRun + 2 * S;  // pixels one run reads
    static constexpr int HS_BUF = HR * kHsStride;
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float min3(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

__device__ __forceinline__ float max3(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// a - b as one FFMA2: b * (-1) + a.
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, f2(-1.0f, -1.0f), a); }

// Stages a frame over the tile's window into shared memory, coordinates clamped to the image as
// the reference's `read_clamped_line` does (helpers.rs:20-32).
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

// The centre values of one phase-1 run, each duplicated into both lanes of a pair: u (and v).
template <int C, int S>
struct CentreRun {
    float2 u[Cfg<C, S>::RUNW];
    float2 v[C == 2 ? Cfg<C, S>::RUNW : 1];

    __device__ __forceinline__ void load(const float* ctr_row) {
#pragma unroll
        for (int i = 0; i < Cfg<C, S>::RUNW; ++i) {
            if (C == 1) {
                u[i] = f2(ctr_row[i], ctr_row[i]);
            } else {
                float2 c = *reinterpret_cast<const float2*>(ctr_row + 2 * i);
                u[i] = f2(c.x, c.x);
                v[i] = f2(c.y, c.y);
            }
        }
    }
};

// Phase 1 of one step: the 8 horizontal box sums of one tile row for both lanes, stored as lane
// pairs. `n0` and `n1` point at the run's first halo pixel in each lane's neighbour tile.
template <int C, int S>
__device__ __forceinline__ void row_run(const CentreRun<C, S>& c, const float* __restrict__ n0,
                                        const float* __restrict__ n1, float* __restrict__ hs_out) {
    constexpr int RUNW = Cfg<C, S>::RUNW;
    float2 d[RUNW];
#pragma unroll
    for (int i = 0; i < RUNW; ++i) {
        if (C == 1) {
            float2 diff = sub2(c.u[i], f2(n0[i], n1[i]));
            d[i] = mul2(diff, diff);
        } else {
            float2 a = *reinterpret_cast<const float2*>(n0 + 2 * i);
            float2 b = *reinterpret_cast<const float2*>(n1 + 2 * i);
            float2 du = sub2(c.u[i], f2(a.x, b.x));
            float2 dv = sub2(c.v[i], f2(a.y, b.y));
            d[i] = fma2(dv, dv, mul2(du, du));
        }
    }
    float2 h[kRun];
    float2 run = d[0];
#pragma unroll
    for (int i = 1; i <= 2 * S; ++i) run = add2(run, d[i]);
    h[0] = run;
#pragma unroll
    for (int j = 1; j < kRun; ++j) {
        run = sub2(add2(run, d[j + 2 * S]), d[j - 1]);
        h[j] = run;
    }
#pragma unroll
    for (int m = 0; m < kRun / 2; ++m)
        *reinterpret_cast<float4*>(hs_out + 4 * m) = make_float4(h[2 * m].x, h[2 * m].y, h[2 * m + 1].x, h[2 * m + 1].y);
}

// Shared-memory layout of one CTA. With a reference ring (a prefilter), `ctr` and `nbr` hold the
// reference frames the distances compare and `val` the input frames whose values are averaged;
// without one, `val` is unused and the values come from `nbr`.
struct Smem {
    float* ctr;     // centre frame, s halo, rows of CSTRIDE floats
    float* nbr[2];  // neighbour tiles, s + a halo, rows of `nstride` floats
    float* val[2];  // input neighbour tiles beside reference `nbr` tiles, same geometry
    float* hs;      // [2 buffers][HR][kTX lane pairs], rows of kHsStride floats
    int nstride, nrows, ncols;
};

// Whether a tile CTA stages its centre tile in the row-sum buffers: with the centre runs kept in
// registers (CTR_REG) the staged tile is read once, before the first step writes a row sum, and the
// finish reads the centre values from the frame, so the tile needs no space of its own. That keeps a
// luma tile at s=2, a=5 and two pairs under 38 KB, six CTAs to an SM. Not in the adjoint's record
// tiles, whose finish reads the staged tile.
template <int C, int S, bool REC>
__host__ __device__ constexpr bool centre_in_row_sums() {
    return Cfg<C, S>::CTR_REG && !REC && round_up4(Cfg<C, S>::CROWS * Cfg<C, S>::CSTRIDE) <= 2 * Cfg<C, S>::HS_BUF;
}

// Dynamic shared memory of one tile CTA for search radius A, `pairs` temporal pair passes and,
// with `ref`, the input value tiles beside the reference tiles (forward tiles, not the records).
template <int C, int S>
inline size_t nlm_smem_bytes(int A, int pairs, bool ref) {
    using K = Cfg<C, S>;
    const int nrows = K::TY + 2 * S + 2 * A;
    const int ncols = kTX + 2 * S + 2 * A;
    const int nstride = nbr_stride(ncols, C);
    const size_t tiles = (size_t)round_up4((pairs > 0 ? 2 : 1) * nrows * nstride);
    const size_t ctr = centre_in_row_sums<C, S, false>() ? 0 : (size_t)round_up4(K::CROWS * K::CSTRIDE);
    const size_t floats = ctr + (ref ? 2 : 1) * tiles + (size_t)2 * K::HS_BUF;
    return floats * sizeof(float);
}

// Per-thread accumulators: lane pairs, summed at the finish.
template <int C, int V>
struct Acc {
    float2 a[C][V];  // sum w * I per channel
    float2 ws[V];    // sum w
    float m[V];      // min distance (FAST) or max weight (HQ)
    int id[V];       // with tracking: the first offset (in the forward's order) reaching m
};

// The lanes of one step: neighbour tiles and offsets (the neighbour of pixel p is p + (dx, dy)),
// and each lane's offset id in the forward's order (fused.rs: for each pair pass k and q, the
// forward frame then the backward frame; then the single-frame pass's q != 0, row-major). With a
// reference ring, v0 and v1 are the input tiles whose values the lanes average.
struct Lanes {
    const float* t0;
    const float* t1;
    int dx0, dy0, dx1, dy1;
    int id0, id1;
    const float* v0;
    const float* v1;
};

// One two-lane step: phase 1, barrier, phase 2. FAST: one strength, no offsets, no confidence.
// TRACK: keep the id of the first offset reaching the max weight (the adjoint's records); lane 0's
// id is below lane 1's and steps run in id order, so strict comparisons keep the first.
// REF: distances on the reference tiles t0/t1, values from the input tiles v0/v1.
template <int C, int S, bool FAST, bool CONF, bool TRACK = false, bool REF = false>
__device__ __forceinline__ void step(const Smem& sm, int A, const Lanes& ln, int& buf, const CentreRun<C, S>& crun,
                                     float2 kk, float2 scale2, float2 negoff, const float2* conf,
                                     Acc<C, Cfg<C, S>::V>& acc) {
    using K = Cfg<C, S>;
    constexpr int V = K::V;
    const int tid = threadIdx.x;
    float* hs = sm.hs + buf * K::HS_BUF;

    for (int slot = tid; slot < K::TASK_SLOTS; slot += kThreads) {
        const int r = ((slot >> 5) << 3) + (slot & 7);
        if (r >= K::HR) continue;
        const int x0 = ((slot >> 3) & 3) * kRun;
        const float* n0 = ln.t0 + (r + ln.dy0 + A) * sm.nstride + (x0 + ln.dx0 + A) * C;
        const float* n1 = ln.t1 + (r + ln.dy1 + A) * sm.nstride + (x0 + ln.dx1 + A) * C;
        if (K::CTR_REG) {
            row_run<C, S>(crun, n0, n1, hs + r * kHsStride + 2 * x0);
        } else {
            CentreRun<C, S> c;
            c.load(sm.ctr + r * K::CSTRIDE + x0 * C);
            row_run<C, S>(c, n0, n1, hs + r * kHsStride + 2 * x0);
        }
    }
    __syncthreads();

    const int col = tid & 31;
    const int y0 = (tid >> 5) * V;
    float2 hv[V + 2 * S];
#pragma unroll
    for (int i = 0; i < V + 2 * S; ++i) hv[i] = *reinterpret_cast<const float2*>(hs + (y0 + i) * kHsStride + 2 * col);
    float2 dist = hv[0];
#pragma unroll
    for (int i = 1; i <= 2 * S; ++i) dist = add2(dist, hv[i]);
    const float* p0 = (REF ? ln.v0 : ln.t0) + (y0 + S + ln.dy0 + A) * sm.nstride + (col + S + ln.dx0 + A) * C;
    const float* p1 = (REF ? ln.v1 : ln.t1) + (y0 + S + ln.dy1 + A) * sm.nstride + (col + S + ln.dx1 + A) * C;
#pragma unroll
    for (int k = 0; k < V; ++k) {
        if (k > 0) dist = sub2(add2(dist, hv[k + 2 * S]), hv[k - 1]);
        float2 w;
        if (FAST) {
            float2 e = mul2(dist, kk);
            w = f2(ex2_approx(e.x), ex2_approx(e.y));
            if (TRACK) {
                if (dist.x < acc.m[k]) {
                    acc.m[k] = dist.x;
                    acc.id[k] = ln.id0;
                }
                if (dist.y < acc.m[k]) {
                    acc.m[k] = dist.y;
                    acc.id[k] = ln.id1;
                }
            } else {
                acc.m[k] = min3(acc.m[k], dist.x, dist.y);
            }
        } else {
            float2 x = fma2(dist, scale2, negoff);
            x = f2(fmaxf(x.x, 0.0f), fmaxf(x.y, 0.0f));
            float2 e = mul2(x, kk);
            w = f2(ex2_approx(e.x), ex2_approx(e.y));
            if (CONF) w = mul2(w, conf[k]);
            if (TRACK) {
                if (w.x > acc.m[k]) {
                    acc.m[k] = w.x;
                    acc.id[k] = ln.id0;
                }
                if (w.y > acc.m[k]) {
                    acc.m[k] = w.y;
                    acc.id[k] = ln.id1;
                }
            } else {
                acc.m[k] = max3(acc.m[k], w.x, w.y);
            }
        }
        const float* q0 = p0 + k * sm.nstride;
        const float* q1 = p1 + k * sm.nstride;
        if (C == 1) {
            acc.a[0][k] = fma2(f2(q0[0], q1[0]), w, acc.a[0][k]);
        } else {
            float2 a = *reinterpret_cast<const float2*>(q0);
            float2 b = *reinterpret_cast<const float2*>(q1);
            acc.a[0][k] = fma2(f2(a.x, b.x), w, acc.a[0][k]);
            acc.a[C - 1][k] = fma2(f2(a.y, b.y), w, acc.a[C - 1][k]);
        }
        acc.ws[k] = add2(acc.ws[k], w);
    }
    buf ^= 1;
}

extern __shared__ __align__(16) float smem_raw[];

// Whether `v`, quantised as the egress does (engine/kernels.rs:103-153: clamped to [0, 1], times
// the largest code, plus 0.5, truncated), lies within `band` codes of a change of code.
__device__ __forceinline__ bool near_code_boundary(float v, float code_max, float band) {
    const float t = fminf(fmaxf(v, 0.0f), 1.0f) * code_max + 0.5f;
    const float f = t - floorf(t);
    return f < band || f > 1.0f - band;
}

// Appends `pixel` to `list` where `near` holds: one atomic per warp. Every lane of the warp calls it.
__device__ __forceinline__ void note_fix(bool near, int64_t pixel, int* list, int* count) {
    const unsigned m = __ballot_sync(0xffffffffu, near);
    if (m == 0) return;
    const int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == __ffs(m) - 1) base = atomicAdd(count, __popc(m));
    base = __shfl_sync(0xffffffffu, base, __ffs(m) - 1);
    if (near) list[base + __popc(m & ((1u << lane) - 1u))] = static_cast<int>(pixel);
}

// Where a record tile writes instead of the output: per pixel out[2], 1/den (0 when the pixel
// passes through), dL/dM and the argmax id, for upstream gradient `grad_out`; and the direct
// centre-frame term dL/dout * wref M / den into `grad_centre`.
struct RecordOut {
    const float* grad_out;
    float* records;
    float* grad_centre;
};
constexpr int kRecordWords = 5;

// One output tile (tile_x, tile_y) of the launch `a`; the whole CTA calls it. REC: the adjoint's
// records instead of the output (the max weight tracked with its first offset id). REF: the
// distances compare the reference ring `a.ref_ring` (the `_ref` kernels of fused.rs:532-900) while
// the averaged values and the finish's centre value come from the input ring `a.ring`.
template <int C, int S, bool FAST, bool REC = false, bool REF = false>
__device__ __forceinline__ void nlm_tile(const NlmLaunch& a, int tile_x, int tile_y, const RecordOut* rec = nullptr) {
    using K = Cfg<C, S>;
    constexpr int V = K::V;
    static_assert(!(REC && REF), "the adjoint records have no reference-ring form");

    const int A = a.search_radius;
    const int W = a.width, H = a.height;
    const int X0 = tile_x * kTX;
    const int Y0 = tile_y * K::TY;
    const int tid = threadIdx.x;
    const int col = tid & 31;
    const int y0 = (tid >> 5) * V;
    const int side = 2 * A + 1;

    constexpr bool kCtrAlias = centre_in_row_sums<C, S, REC>();
    Smem sm;
    sm.nrows = K::TY + 2 * S + 2 * A;
    sm.ncols = kTX + 2 * S + 2 * A;
    sm.nstride = nbr_stride(sm.ncols, C);
    const int tile_floats = round_up4((a.pairs > 0 ? 2 : 1) * sm.nrows * sm.nstride);
    if (kCtrAlias) {
        sm.hs = smem_raw;
        sm.ctr = smem_raw;  // read by the centre runs before the first step writes a row sum
        sm.nbr[0] = smem_raw + 2 * K::HS_BUF;
    } else {
        sm.ctr = smem_raw;
        sm.nbr[0] = sm.ctr + round_up4(K::CROWS * K::CSTRIDE);
    }
    sm.nbr[1] = sm.nbr[0] + sm.nrows * sm.nstride;
    sm.val[0] = sm.nbr[0] + tile_floats;
    sm.val[1] = sm.val[0] + sm.nrows * sm.nstride;
    if (!kCtrAlias) sm.hs = sm.nbr[0] + (REF ? 2 : 1) * tile_floats;

    const float h2 = __ldg(a.derived + a.h2_word);
    const float off_pair = __ldg(a.derived + a.offset_word);
    const float scale = C == 1 ? 3.0f : 1.5f;
    const float neg_h2_log2e = -h2 * kLog2e;
    const float2 kk = FAST ? f2(scale * neg_h2_log2e, scale * neg_h2_log2e) : f2(neg_h2_log2e, neg_h2_log2e);
    const float2 scale2 = f2(scale, scale);

    const float* centre = a.ring + a.slot_centre * a.frame_elems;
    const float* dist_ring = REF ? a.ref_ring : a.ring;
    const float* dist_centre = dist_ring + a.slot_centre * a.frame_elems;
    load_tile<C>(sm.ctr, K::CSTRIDE, K::CROWS, K::CW, dist_centre, X0 - S, Y0 - S, W, H);
    __syncthreads();

    CentreRun<C, S> crun;
    if (K::CTR_REG) {
        const int r = ((tid >> 5) << 3) + (tid & 7);
        const int x0 = ((tid >> 3) & 3) * kRun;
        crun.load(sm.ctr + min(r, K::CROWS - 1) * K::CSTRIDE + x0 * C);
    }

    Acc<C, V> acc;
#pragma unroll
    for (int k = 0; k < V; ++k) {
        acc.ws[k] = f2(0.0f, 0.0f);
        acc.m[k] = FAST ? __int_as_float(0x7f800000) : 0.0f;  // +inf min distance / 0 max weight
        acc.id[k] = -1;
#pragma unroll
        for (int c = 0; c < C; ++c) acc.a[c][k] = f2(0.0f, 0.0f);
    }

    int buf = 0;
    float2 conf[V];
    for (int p = 0; p < a.pairs; ++p) {
        __syncthreads();  // every thread is done with the previous pass's tiles
        load_tile<C>(sm.nbr[0], sm.nstride, sm.nrows, sm.ncols, dist_ring + a.slot_fwd[p] * a.frame_elems,
                     X0 - S - A, Y0 - S - A, W, H);
        load_tile<C>(sm.nbr[1], sm.nstride, sm.nrows, sm.ncols, dist_ring + a.slot_bwd[p] * a.frame_elems,
                     X0 - S - A, Y0 - S - A, W, H);
        if (REF) {
            load_tile<C>(sm.val[0], sm.nstride, sm.nrows, sm.ncols, a.ring + a.slot_fwd[p] * a.frame_elems,
                         X0 - S - A, Y0 - S - A, W, H);
            load_tile<C>(sm.val[1], sm.nstride, sm.nrows, sm.ncols, a.ring + a.slot_bwd[p] * a.frame_elems,
                         X0 - S - A, Y0 - S - A, W, H);
        }
        const bool use_conf = !FAST && a.conf != nullptr;
#pragma unroll
        for (int k = 0; k < V; ++k) {
            conf[k] = f2(1.0f, 1.0f);
            if (use_conf) {
                int gx = min(X0 + col, W - 1), gy = min(Y0 + y0 + k, H - 1);
                int bc = min(gx / a.conf_step, a.blocks_x - 1);
                int br = min(gy / a.conf_step, a.blocks_y - 1);
                conf[k] = f2(__ldg(a.conf + a.conf_fwd_off[p] + br * a.blocks_x + bc),
                             __ldg(a.conf + a.conf_bwd_off[p] + br * a.blocks_x + bc));
            }
        }
        __syncthreads();
        Lanes ln{sm.nbr[0], sm.nbr[1], 0, 0, 0, 0, 0, 0, sm.val[0], sm.val[1]};
        const float2 negoff = f2(-off_pair, -off_pair);
        for (int qy = -A; qy <= A; ++qy) {
            for (int qx = -A; qx <= A; ++qx) {
                ln.dx0 = qx;
                ln.dy0 = qy;
                ln.dx1 = -qx;
                ln.dy1 = -qy;
                ln.id0 = 2 * ((p * side + qy + A) * side + qx + A);
                ln.id1 = ln.id0 + 1;
                if (use_conf)
                    step<C, S, FAST, true, REC, REF>(sm, A, ln, buf, crun, kk, scale2, negoff, conf, acc);
                else
                    step<C, S, FAST, false, REC, REF>(sm, A, ln, buf, crun, kk, scale2, negoff, conf, acc);
            }
        }
    }

    // The single-frame pass: the window without its centre, two consecutive offsets per step.
    __syncthreads();
    load_tile<C>(sm.nbr[0], sm.nstride, sm.nrows, sm.ncols, dist_centre, X0 - S - A, Y0 - S - A, W, H);
    if (REF) load_tile<C>(sm.val[0], sm.nstride, sm.nrows, sm.ncols, centre, X0 - S - A, Y0 - S - A, W, H);
    __syncthreads();
    {
        Lanes ln{sm.nbr[0], sm.nbr[0], 0, 0, 0, 0, 0, 0, sm.val[0], sm.val[0]};
        const int n = side * side - 1;
        const int mid = A * side + A;
        const int spatial_base = 2 * a.pairs * side * side;
        for (int i = 0; i < n; i += 2) {
            ln.id0 = spatial_base + i;
            ln.id1 = spatial_base + i + 1;
            const int l0 = i < mid ? i : i + 1;
            const int l1 = i + 1 < mid ? i + 1 : i + 2;
            ln.dx0 = l0 % side - A;
            ln.dy0 = l0 / side - A;
            ln.dx1 = l1 % side - A;
            ln.dy1 = l1 / side - A;
            float2 negoff = f2(0.0f, 0.0f);
            if (!FAST && a.spatial_lut) negoff = f2(-__ldg(a.spatial_lut + l0), -__ldg(a.spatial_lut + l1));
            step<C, S, FAST, false, REC, REF>(sm, A, ln, buf, crun, kk, scale2, negoff, conf, acc);
        }
    }

    if (REC) {
        // accumulate.rs:175-201 differentiated at this pixel: with den = wref M + W, out =
        // (I wref M + A) / den, dL/dM = sum_c g_c wref (I_c - out_c) / den, and the direct term of
        // the centre pixel's own value dL/dI = g wref M / den (I when den <= 1e-30 passes through).
        const int gx = X0 + col;
#pragma unroll
        for (int k = 0; k < V; ++k) {
            const int gy = Y0 + y0 + k;
            if (gx >= W || gy >= H) continue;
            const int64_t px = (int64_t)gy * W + gx;
            const float max_w = FAST ? ex2_approx(acc.m[k] * kk.x) : acc.m[k];
            const float wsum = acc.ws[k].x + acc.ws[k].y;
            const float* orig = sm.ctr + (y0 + k + S) * K::CSTRIDE + (col + S) * C;
            const float* g = rec->grad_out + px * C;
            float* gc = rec->grad_centre + px * C;
            float* r = rec->records + px * kRecordWords;
            const float self_weight = a.wref * max_w;
            const float den = self_weight + wsum;
            if (!(den > 1e-30f)) {
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    gc[c] = g[c];
                    r[c] = orig[c];
                }
                if (C == 1) r[1] = 0.0f;
                r[2] = 0.0f;
                r[3] = 0.0f;
                r[4] = __int_as_float(-1);
                continue;
            }
            const float inv = 1.0f / den;
            float gm = 0.0f;
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const float o = (orig[c] * self_weight + acc.a[c][k].x + acc.a[c][k].y) * inv;
                gc[c] = g[c] * self_weight * inv;
                gm += g[c] * a.wref * (orig[c] - o) * inv;
                r[c] = o;
            }
            if (C == 1) r[1] = 0.0f;
            r[2] = inv;
            r[3] = gm;
            r[4] = __int_as_float(acc.id[k]);
        }
        return;
    }

    // Finish (accumulate.rs:175-201), written straight to the output frame.
    const int gx = X0 + col;
    const bool flags = a.fix_count != nullptr;
    const float band = a.code_max * (a.fix_band + kFixBandPerH2 * h2);
#pragma unroll
    for (int k = 0; k < V; ++k) {
        const int gy = Y0 + y0 + k;
        bool near = false;
        if (gx < W && gy < H) {
            const float max_w = FAST ? ex2_approx(acc.m[k] * kk.x) : acc.m[k];
            const float wsum = acc.ws[k].x + acc.ws[k].y;
            // The centre value: the input's own (accumulate.rs:175-201 reads the input ring), which
            // the reference-ring tile does not hold.
            const float* orig = (REF || kCtrAlias) ? centre + ((int64_t)gy * W + gx) * C
                                                   : sm.ctr + (y0 + k + S) * K::CSTRIDE + (col + S) * C;
            const float self_weight = __fmul_rn(a.wref, max_w);
            const float denom = __fadd_rn(self_weight, wsum);
            float* dst = a.out + ((int64_t)gy * W + gx) * C;
            if (denom > 1e-30f) {
                const float inv = __frcp_rn(denom);
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    const float sum_wi = acc.a[c][k].x + acc.a[c][k].y;
                    const float v = __fmul_rn(__fadd_rn(__fmul_rn(orig[c], self_weight), sum_wi), inv);
                    dst[c] = v;
                    if (flags) near |= near_code_boundary(v, a.code_max, band);
                }
            } else {
#pragma unroll
                for (int c = 0; c < C; ++c) dst[c] = orig[c];  // passes through exactly
            }
        }
        if (flags) note_fix(near, (int64_t)gy * W + gx, a.fix_list, a.fix_count);
    }
}


}  // namespace nlm_tile_detail
}  // namespace avd
