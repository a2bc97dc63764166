// The exact finish of NLMeans samples that sit near a rounding boundary, for sm_100a.
//
// Why. The window kernel (nlm.cu) sums each patch distance with running box sums and weighs it with
// the MUFU ex2 approximation, so its float result differs from the reference kernels' arithmetic in
// the last bits (a few 1e-6 at most). Quantised to codes that difference only matters where the
// result lies within it of a change of code, and there it decides the code: wherever one
// neighbour dominates, the self weight equals its weight and the exact result is the mean of two
// integer codes, a half code. So the window kernel flags every pixel whose result lies within
// `fix_band` codes of a boundary, and this kernel recomputes exactly those pixels in the
// operation order of the reference kernels as the FP32 mirror restates them
// (av-denoise-core/src/nlmeans/kernels/fused.rs:138-530 and accumulate.rs:152-202, launch order
// dispatch/mod.rs:665-679):
//   - each patch distance is the row-major sum over the (2s+1)^2 patch of
//     line_sum_sq(centre - neighbour) * scale (helpers.rs:34-62, fused.rs:19-43), coordinates
//     clamped to the frame (helpers.rs:20-32);
//   - each weight is exp(-max(D - offset, 0) * h2) (helpers.rs:70-73) with the exponential of
//     exp_mirror.cuh, times the block's confidence where it applies;
//   - each pass folds its offsets in row-major order into its own sums
//     (acc = (acc + I_f w_f) + I_b w_b, ws = ws + (w_f + w_b), wm = max(wm, max(w_f, w_b)) for a
//     pair; acc = acc + I w, ws = ws + w, wm = max(wm, w) for the single frame), which are then
//     added to the frame's accumulators, pairs first;
//   - the finish is (I * wref*max_w + A) * (1 / (wref*max_w + W)), or I when the denominator is at
//     most 1e-30.
// Every multiply and add is rounded on its own (the file is also built with -fmad=false).
//
// How (B200 layout). One warp per flagged pixel, no block-wide barriers: many pixels are in
// flight on every SM, which hides the latency of the window staging and of the order-bound folds.
// For each pass the warp stages its pixel's search windows (the (2(a+s)+1)^2 neighbourhood of each
// frame the pass compares, coordinates clamped) in its own shared memory (a launch with only the
// single-frame pass double-buffers it: the next pixel's copies fly while this one is computed, and
// the averaged samples are read from the window too), then every lane forms
// distances two at a time as two independent chains (a pair's forward and backward offset, or two
// spatial offsets), reading the centre patch as a broadcast and the taps at immediate offsets when
// the patch radius is a template argument (0..3; a generic loop reading the frames covers larger
// radii). The weights and the products I*w land in the warp's shared memory in offset order. The
// passes are independent until they are added to the frame's accumulators, so the warp folds a
// batch of passes at once: lane (pass, accumulator) walks its pass's offsets in order for one of
// the C channel sums, the weight sum or the max weight; the pass results are then added to the
// frame's accumulators in pass order and lane 0 finishes the pixel.

#include <cuda_runtime.h>

#include <cstdint>

#include "exp_mirror.cuh"
#include "kernels.h"

namespace avd {

namespace {

constexpr int kWarps = 4;               // 128 threads, one pixel per warp
constexpr int kMaxTplS = 3;             // patch radii with a compile-time tap loop and staged windows
constexpr int kMaxItemFloats = 2048;    // per warp: the weights and products of one batch of passes

__device__ __forceinline__ int clampc(int v, int limit) { return v < 0 ? 0 : (v >= limit ? limit - 1 : v); }
__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }

// Floats of one warp's staged windows: two (2R+1)^2 windows and a (2s+1)^2 centre patch.
__host__ __device__ inline int window_floats(int C, int R, int s) {
    return C * (2 * (2 * R + 1) * (2 * R + 1) + (2 * s + 1) * (2 * s + 1));
}

__device__ __forceinline__ float welsch_mirror(float dist, float h2, float off) {
    const float excess = fmaxf(__fsub_rn(dist, off), 0.0f);
    return exp_mirror(__fmul_rn(-excess, h2));
}

// The mirror's line sum starts from 0, and 0 + x = x for the non-negative first square, so the sum
// starts from that square. One tap: line_sum_sq(centre - neighbour) * scale added to the running
// sum (helpers.rs:34-62), every operation rounded on its own.
template <int C>
__device__ __forceinline__ float tap(float sum, const float* c, float n0, float n1, float scale) {
    const float l0 = __fsub_rn(c[0], n0);
    float l = __fmul_rn(l0, l0);
    if (C == 2) {
        const float l1 = __fsub_rn(c[1], n1);
        l = __fadd_rn(l, __fmul_rn(l1, l1));
    }
    return __fadd_rn(sum, __fmul_rn(l, scale));
}

template <int C>
__device__ __forceinline__ const float* at(const float* frame, int x, int y, int W, int H) {
    return frame + ((int64_t)clampc(y, H) * W + clampc(x, W)) * C;
}

// Two patch distances in the mirror's order (fused.rs:19-43), tap by tap in row-major order, as two
// independent chains, all from shared memory: `c` is the centre patch (rows of `cstride` floats),
// `n0` and `n1` each lane's neighbour patch origin (rows of `nstride` floats).
template <int C, int S>
__device__ __forceinline__ float2 distances_staged(const float* c, int cstride, const float* n0, const float* n1,
                                                   int nstride, float scale) {
    float sum0 = 0.0f, sum1 = 0.0f;
#pragma unroll
    for (int ty = 0; ty <= 2 * S; ++ty) {
#pragma unroll
        for (int tx = 0; tx <= 2 * S; ++tx) {
            const float* cp = c + ty * cstride + tx * C;
            const float* a = n0 + ty * nstride + tx * C;
            const float* b = n1 + ty * nstride + tx * C;
            sum0 = tap<C>(sum0, cp, a[0], C == 2 ? a[1] : 0.0f, scale);
            sum1 = tap<C>(sum1, cp, b[0], C == 2 ? b[1] : 0.0f, scale);
        }
    }
    return f2(sum0, sum1);
}

// Any patch radius, straight from the frames (clamped reads).
template <int C>
__device__ __forceinline__ float2 distances_generic(const float* __restrict__ ctr, int px, int py, int s,
                                                    const float* __restrict__ f0, int x0, int y0,
                                                    const float* __restrict__ f1, int x1, int y1, int W, int H,
                                                    float scale) {
    float sum0 = 0.0f, sum1 = 0.0f;
    for (int ty = 0; ty <= 2 * s; ++ty)
        for (int tx = 0; tx <= 2 * s; ++tx) {
            const float* c = at<C>(ctr, px - s + tx, py - s + ty, W, H);
            const float cv[2] = {__ldg(c), C == 2 ? __ldg(c + 1) : 0.0f};
            const float* a = at<C>(f0, x0 + tx, y0 + ty, W, H);
            const float* b = at<C>(f1, x1 + tx, y1 + ty, W, H);
            sum0 = tap<C>(sum0, cv, __ldg(a), C == 2 ? __ldg(a + 1) : 0.0f, scale);
            sum1 = tap<C>(sum1, cv, __ldg(b), C == 2 ? __ldg(b + 1) : 0.0f, scale);
        }
    return f2(sum0, sum1);
}

// Item floats of one pass: a pair pass holds W_f, W_b and C rows each of I_f w_f and I_b w_b over
// its (2a+1)^2 offsets; the single-frame pass W and C rows of I w over its (2a+1)^2 - 1.
__host__ __device__ inline int pass_floats(int C, int side, bool pair) {
    return pair ? (2 + 2 * C) * side * side : (1 + C) * (side * side - 1);
}

// S in 0..kMaxTplS: compile-time patch radius, windows staged per warp; S < 0: any radius, read
// from the frames.
template <int C, int S>
__global__ void __launch_bounds__(kWarps * 32) nlm_exact_kernel(NlmLaunch a, int warp_floats) {
    extern __shared__ __align__(16) float exact_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int W = a.width, H = a.height;
    const int64_t count = a.fix_list ? static_cast<int64_t>(*a.fix_count) : static_cast<int64_t>(W) * H;
    const int A = a.search_radius, s = S >= 0 ? S : a.patch_radius, side = 2 * A + 1, nq = side * side;
    const float h2 = __ldg(a.derived + a.h2_word);
    const float off_pair = a.fast ? 0.0f : __ldg(a.derived + a.offset_word);
    const bool use_conf = !a.fast && a.conf != nullptr;
    const bool lut = a.spatial_lut && !a.fast;
    const float scale = C == 1 ? 3.0f : 1.5f;
    const float* dring = a.ref_ring ? a.ref_ring : a.ring;
    const float* ctr = a.ring + a.slot_centre * a.frame_elems;
    const float* rctr = dring + a.slot_centre * a.frame_elems;
    const int R = A + s;
    const int rs = 2 * R + 1;    // staged window side
    const int wstride = rs * C;  // floats per staged window row
    const int pside = 2 * s + 1;
    const int mid = A * side + A;
    const int npass = a.pairs + 1;  // pair passes k = 0..d-1, then the single-frame pass
    constexpr int kRoles = C + 2;   // channel sums, weight sum, max weight

    // (q mod side, q div side) of every window offset q, shared by the CTA's warps.
    int* qtab = reinterpret_cast<int*>(exact_smem + kWarps * warp_floats);
    for (int q = threadIdx.x; q < nq; q += kWarps * 32) {
        qtab[q] = q % side;
        qtab[q + nq] = q / side;
    }
    __syncthreads();
    float* mine = exact_smem + warp * warp_floats;
    float* win0 = mine;
    float* win1 = win0 + (S >= 0 ? rs * rs * C : 0);
    float* cpatch = win1 + (S >= 0 ? rs * rs * C : 0);
    float* items = cpatch + (S >= 0 ? pside * pside * C : 0);

    // Stages the (2r+1)^2 neighbourhood of (px, py) in `frame`, clamped, into `dst` with
    // asynchronous copies (one per pixel, all in flight together), then waits for them.
    auto stage = [&](float* dst, const float* frame, int px, int py, int r) {
        const int n = (2 * r + 1) * (2 * r + 1);
        for (int i = lane; i < n; i += 32) {
            const int ry = i / (2 * r + 1), rx = i - ry * (2 * r + 1);
            const float* src = at<C>(frame, px - r + rx, py - r + ry, W, H);
            const unsigned dst_s = static_cast<unsigned>(__cvta_generic_to_shared(dst + i * C));
            if (C == 1)
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst_s), "l"(src) : "memory");
            else
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst_s), "l"(src) : "memory");
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    };
    // A single-frame launch (no pair passes) stages one window per pixel, so its windows are
    // double-buffered in the two window slots: the next pixel's copies are in flight while this
    // pixel's distances are formed.
    const bool prefetch = S >= 0 && a.pairs == 0;
    auto issue = [&](float* dst, int64_t item) {
        const int pn = a.fix_list ? a.fix_list[item] : static_cast<int>(item);
        const int qx = pn % W, qy = pn / W, n = rs * rs;
        for (int k = lane; k < n; k += 32) {
            const int ry = k / rs, rx = k - ry * rs;
            const float* src = at<C>(rctr, qx - R + rx, qy - R + ry, W, H);
            const unsigned dst_s = static_cast<unsigned>(__cvta_generic_to_shared(dst + k * C));
            if (C == 1)
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst_s), "l"(src) : "memory");
            else
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst_s), "l"(src) : "memory");
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    // The single-frame pass's items of pixel (px, py) into `it` (rows: W, then per channel I w, over
    // q != 0), from the staged window `sw`; every lane calls it.
    auto single_items = [&](float* it, const float* sw, int px, int py) {
        // rows: W, then per channel I w, over q != 0; a lane forms items j and j + 32
        const int n = nq - 1;
        for (int j = lane; j < n; j += 64) {
            const bool two = j + 32 < n;
            const int l0 = j < mid ? j : j + 1;
            const int j1 = two ? j + 32 : j;
            const int l1 = j1 < mid ? j1 : j1 + 1;
            const int qx0 = qtab[l0] - A, qy0 = qtab[l0 + nq] - A;
            const int qx1 = qtab[l1] - A, qy1 = qtab[l1 + nq] - A;
            float2 d;
            if (S >= 0) {
                d = distances_staged<C, (S >= 0 ? S : 0)>(
                    sw + (R - s) * wstride + (R - s) * C, wstride,
                    sw + (R + qy0 - s) * wstride + (R + qx0 - s) * C,
                    sw + (R + qy1 - s) * wstride + (R + qx1 - s) * C, wstride, scale);
            } else {
                d = distances_generic<C>(rctr, px, py, s, rctr, px + qx0 - s, py + qy0 - s, rctr,
                                         px + qx1 - s, py + qy1 - s, W, H, scale);
            }
            const float w0 = welsch_mirror(d.x, h2, lut ? __ldg(a.spatial_lut + l0) : 0.0f);
            const float w1 = welsch_mirror(d.y, h2, lut ? __ldg(a.spatial_lut + l1) : 0.0f);
            float v0[C], v1[C];
            if (S >= 0 && !a.ref_ring) {
                // The staged centre window holds the same clamped samples.
                const float* n0 = sw + (R + qy0) * wstride + (R + qx0) * C;
                const float* n1 = sw + (R + qy1) * wstride + (R + qx1) * C;
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    v0[c] = n0[c];
                    v1[c] = n1[c];
                }
            } else {
                const float* n0 = at<C>(ctr, px + qx0, py + qy0, W, H);
                const float* n1 = at<C>(ctr, px + qx1, py + qy1, W, H);
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    v0[c] = __ldg(n0 + c);
                    v1[c] = __ldg(n1 + c);
                }
            }
            it[j] = w0;
#pragma unroll
            for (int c = 0; c < C; ++c) it[(1 + c) * n + j] = __fmul_rn(v0[c], w0);
            if (two) {
                it[j + 32] = w1;
#pragma unroll
                for (int c = 0; c < C; ++c) it[(1 + c) * n + j + 32] = __fmul_rn(v1[c], w1);
            }
        }
    };

    const int64_t first = (int64_t)blockIdx.x * kWarps + warp, stride = (int64_t)gridDim.x * kWarps;
    int cur = 0;
    if (prefetch && first < count) issue(win0, first);

    for (int64_t i = first; i < count; i += stride) {
        const int pix = a.fix_list ? a.fix_list[i] : static_cast<int>(i);
        const int px = pix % W, py = pix / W;
        float* sw = win0;  // the staged window of the single-frame pass
        if (prefetch) {
            sw = cur ? win1 : win0;
            if (i + stride < count) {
                issue(cur ? win0 : win1, i + stride);
                asm volatile("cp.async.wait_group 1;\n" ::: "memory");
            } else {
                asm volatile("cp.async.wait_group 0;\n" ::: "memory");
            }
            __syncwarp();
        }
        // lanes 0..kRoles-1: the frame's accumulators (sum I w per channel, sum w, max w)
        float acc = 0.0f;

        for (int b0 = 0; b0 < npass;) {
            // The batch: consecutive passes whose items fit in this warp's item space and whose fold
            // lanes fit in the warp.
            int b1 = b0, used = 0;
            while (b1 < npass && (b1 - b0 + 1) * kRoles <= 32) {
                const int f = pass_floats(C, side, b1 < a.pairs);
                if (b1 > b0 && used + f > kMaxItemFloats) break;
                used += f;
                ++b1;
            }
            // Form every item of the batch.
            int off = 0;
            for (int p = b0; p < b1; ++p) {
                float* it = items + off;
                if (p < a.pairs) {
                    const float* fwd = a.ring + a.slot_fwd[p] * a.frame_elems;
                    const float* bwd = a.ring + a.slot_bwd[p] * a.frame_elems;
                    const float* rfwd = dring + a.slot_fwd[p] * a.frame_elems;
                    const float* rbwd = dring + a.slot_bwd[p] * a.frame_elems;
                    if (S >= 0) {
                        __syncwarp();  // every lane is done with the previous windows
                        stage(win0, rfwd, px, py, R);
                        stage(win1, rbwd, px, py, R);
                        stage(cpatch, rctr, px, py, s);
                        __syncwarp();
                    }
                    float cf = 1.0f, cb = 1.0f;
                    if (use_conf) {
                        const int bc = min(px / a.conf_step, a.blocks_x - 1);
                        const int br = min(py / a.conf_step, a.blocks_y - 1);
                        cf = __ldg(a.conf + a.conf_fwd_off[p] + br * a.blocks_x + bc);
                        cb = __ldg(a.conf + a.conf_bwd_off[p] + br * a.blocks_x + bc);
                    }
                    // rows: W_f, W_b, then per channel I_f w_f and I_b w_b
                    for (int q = lane; q < nq; q += 32) {
                        const int qx = qtab[q] - A, qy = qtab[q + nq] - A;
                        float2 d;
                        if (S >= 0) {
                            d = distances_staged<C, (S >= 0 ? S : 0)>(
                                cpatch, pside * C, win0 + (R + qy - s) * wstride + (R + qx - s) * C,
                                win1 + (R - qy - s) * wstride + (R - qx - s) * C, wstride, scale);
                        } else {
                            d = distances_generic<C>(rctr, px, py, s, rfwd, px + qx - s, py + qy - s, rbwd,
                                                     px - qx - s, py - qy - s, W, H, scale);
                        }
                        float wf = welsch_mirror(d.x, h2, off_pair);
                        float wb = welsch_mirror(d.y, h2, off_pair);
                        if (use_conf) {
                            wf = __fmul_rn(wf, cf);
                            wb = __fmul_rn(wb, cb);
                        }
                        it[q] = wf;
                        it[nq + q] = wb;
                        if (S >= 0 && !a.ref_ring) {
                            // The averaged samples are the staged windows' own (same clamped pixels).
                            const float* fp = win0 + (R + qy) * wstride + (R + qx) * C;
                            const float* bp = win1 + (R - qy) * wstride + (R - qx) * C;
#pragma unroll
                            for (int c = 0; c < C; ++c) {
                                it[(2 + 2 * c) * nq + q] = __fmul_rn(fp[c], wf);
                                it[(3 + 2 * c) * nq + q] = __fmul_rn(bp[c], wb);
                            }
                        } else {
                            const float* fp = at<C>(fwd, px + qx, py + qy, W, H);
                            const float* bp = at<C>(bwd, px - qx, py - qy, W, H);
#pragma unroll
                            for (int c = 0; c < C; ++c) {
                                it[(2 + 2 * c) * nq + q] = __fmul_rn(__ldg(fp + c), wf);
                                it[(3 + 2 * c) * nq + q] = __fmul_rn(__ldg(bp + c), wb);
                            }
                        }
                    }
                } else {
                    if (S >= 0 && !prefetch) {
                        __syncwarp();
                        stage(win0, rctr, px, py, R);
                        __syncwarp();
                    }
                    single_items(it, sw, px, py);
                }
                off += pass_floats(C, side, p < a.pairs);
            }
            __syncwarp();

            // Fold: lane (pass p, role r) walks pass p's items in offset order (fused.rs:317-346 for a
            // pair: acc = (acc + I_f w_f) + I_b w_b, ws = ws + (w_f + w_b), wm = max(wm, max(w_f, w_b));
            // fused.rs:506-530 for the single frame: acc = acc + I w, ws = ws + w, wm = max(wm, w)).
            float pass = 0.0f;
            const int lp = b0 + lane / kRoles, role = lane % kRoles;
            if (lane < (b1 - b0) * kRoles) {
                int poff = 0;
                for (int p = b0; p < lp; ++p) poff += pass_floats(C, side, p < a.pairs);
                const float* it = items + poff;
                // Every fold lane runs the same instructions on its own rows (no divergence between
                // the accumulators): the channel sums take (p + x) + y, the weight sum p + (x + y), the
                // max weight max(p, max(x, y)); the single frame's rows have y = 0 and x alone.
                const bool pair = lp < a.pairs;
                const int len = pair ? nq : nq - 1;
                const float* x = pair ? (role < C ? it + (2 + 2 * role) * nq : it)
                                      : (role < C ? it + (1 + role) * (nq - 1) : it);
                const float* y = pair ? (role < C ? it + (3 + 2 * role) * nq : it + nq) : x;
                const bool is_sum = role < C, is_ws = role == C;
                if (pair) {
                    for (int q = 0; q < len; ++q) {
                        const float xv = x[q], yv = y[q];
                        const float s1 = __fadd_rn(__fadd_rn(pass, xv), yv);
                        const float s2 = __fadd_rn(pass, __fadd_rn(xv, yv));
                        const float m = fmaxf(pass, fmaxf(xv, yv));
                        pass = is_sum ? s1 : (is_ws ? s2 : m);
                    }
                } else {
                    for (int q = 0; q < len; ++q) {
                        const float xv = x[q];
                        const float s1 = __fadd_rn(pass, xv);
                        const float m = fmaxf(pass, xv);
                        pass = role <= C ? s1 : m;
                    }
                }
            }
            // The frame's accumulators take the batch's passes in order (accumulate.rs reads them
            // pair by pair, then the single frame).
            for (int p = b0; p < b1; ++p) {
                const float v = __shfl_sync(0xffffffffu, pass, (p - b0) * kRoles + (lane % kRoles));
                if (lane < kRoles) acc = lane == C + 1 ? fmaxf(acc, v) : __fadd_rn(acc, v);
            }
            __syncwarp();  // the items are read before the next batch overwrites them
            b0 = b1;
        }

        // ---- the finish (accumulate.rs:175-201), by lane 0 ----
        float fin[kRoles];
#pragma unroll
        for (int r = 0; r < kRoles; ++r) fin[r] = __shfl_sync(0xffffffffu, acc, r);
        if (lane == 0) {
            const float* orig = ctr + (int64_t)pix * C;
            const float self_weight = __fmul_rn(a.wref, fin[C + 1]);
            const float denom = __fadd_rn(self_weight, fin[C]);
            float* dst = a.out + (int64_t)pix * C;
#pragma unroll
            for (int c = 0; c < C; ++c) {
                if (denom > 1e-30f) {
                    const float inv = __frcp_rn(denom);
                    const float num = __fadd_rn(__fmul_rn(orig[c], self_weight), fin[c]);
                    dst[c] = __fmul_rn(num, inv);
                } else {
                    dst[c] = orig[c];
                }
            }
        }
        cur ^= 1;  // every lane is past this pixel's window reads (the fold's __syncwarp)
    }
}

__global__ void exp_mirror_kernel(const float* __restrict__ x, float* __restrict__ out, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = exp_mirror(x[i]);
}

template <int C, int S>
cudaError_t launch_cs(const NlmLaunch& a, int sms, cudaStream_t stream) {
    const int side = 2 * a.search_radius + 1;
    const int R = a.search_radius + a.patch_radius;
    // one batch must hold at least the largest single pass
    const int items = min(kMaxItemFloats, max(pass_floats(C, side, a.pairs > 0),
                                              (a.pairs) * pass_floats(C, side, true) + pass_floats(C, side, false)));
    const int warp_floats = (S >= 0 ? window_floats(C, R, a.patch_radius) : 0) + max(items, pass_floats(C, side, a.pairs > 0));
    const size_t smem = sizeof(float) * (kWarps * static_cast<size_t>(warp_floats) + 2 * side * side);
    cudaError_t e = cudaFuncSetAttribute(nlm_exact_kernel<C, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, nlm_exact_kernel<C, S>, kWarps * 32, smem);
    if (e != cudaSuccess) return e;
    // Persistent over the pixels: the count is only known on the device.
    const int64_t ctas_all = ((int64_t)a.width * a.height + kWarps - 1) / kWarps;
    const int64_t slots = static_cast<int64_t>(sms) * (per_sm > 0 ? per_sm : 1);
    const int grid = static_cast<int>(ctas_all < slots ? ctas_all : slots);
    nlm_exact_kernel<C, S><<<grid, kWarps * 32, smem, stream>>>(a, warp_floats);
    return cudaGetLastError();
}

template <int C>
cudaError_t launch_c(const NlmLaunch& a, int sms, cudaStream_t stream) {
    switch (a.patch_radius) {
        case 0: return launch_cs<C, 0>(a, sms, stream);
        case 1: return launch_cs<C, 1>(a, sms, stream);
        case 2: return launch_cs<C, 2>(a, sms, stream);
        case 3: return launch_cs<C, 3>(a, sms, stream);
        default: return launch_cs<C, -1>(a, sms, stream);
    }
}

}  // namespace

cudaError_t launch_nlm_exact(const NlmLaunch& a, cudaStream_t stream) {
    static_assert(kMaxTplS == 3, "launch_c dispatches radii 0..3 to the staged kernel");
    if (a.search_radius < 0 || a.search_radius > 8 || a.patch_radius < 0 || a.patch_radius > 16 || a.pairs < 0 ||
        a.pairs > kMaxPairs || (a.fix_list != nullptr) != (a.fix_count != nullptr))
        return cudaErrorInvalidValue;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    if (a.channels == 1) return launch_c<1>(a, sms, stream);
    if (a.channels == 2) return launch_c<2>(a, sms, stream);
    return cudaErrorInvalidValue;
}

cudaError_t launch_exp_mirror(const float* x, float* out, int64_t n, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    const int64_t blocks = (n + 255) / 256;
    exp_mirror_kernel<<<static_cast<int>(blocks < 4096 ? blocks : 4096), 256, 0, stream>>>(x, out, n);
    return cudaGetLastError();
}

}  // namespace avd
