// CPU ORACLE - test infrastructure only. Nothing in the product links or calls this file; only the
// tests, `__graft_entry__.smoke()` and the CPU-baseline leg of `bench.py` load it, as the checker.
//
// A C++17 restatement of av-denoise's NLMeans kernel arithmetic (the reference is CubeCL Rust and
// cannot be built here: no cargo, and its CubeCL git dependency is not vendored). Two modes:
//   - float: "FP32 mirror" - the same operations, the same order and the same clamping as the
//     reference kernels, compiled with -ffp-contract=off so no multiply-add is fused;
//   - double: an FP64 reference of the same maths.
// Each function names the reference lines it follows (paths inside the av-denoise project).
//
// Parity pin: the reference ships no numeric golden vectors for NLMeans (its parity fixture holds
// FNV hashes recorded on an AMD GPU), and the reference cannot be built here. The restatement is
// pinned by the reference's host-formula tests (Welsch weight, h2 normalisation) and its
// behavioural suites, which tests/ re-run here; beyond those, numeric NLMeans outputs are
// parity unpinned.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

// av-denoise-core/src/nlmeans/kernels/helpers.rs:6-15 (`clamp_coord`).
inline int clamp_coord(int v, int limit) { return v < 0 ? 0 : (v >= limit ? limit - 1 : v); }

// av-denoise-core/src/nlmeans/kernels/helpers.rs:50-62 (`channel_scale`).
template <typename T>
inline T channel_scale(int channels) { return channels == 1 ? T(3) : T(1.5); }

template <typename T>
struct Frame {
    const T* data;  // interleaved, `channels` values per pixel
    int width, height, channels;
    inline const T* at_clamped(int x, int y) const {
        int cx = clamp_coord(x, width), cy = clamp_coord(y, height);
        return data + ((size_t)cy * width + cx) * channels;
    }
};

// av-denoise-core/src/nlmeans/kernels/helpers.rs:34-46 (`line_sum_sq`): sequential, no FMA.
template <typename T>
inline T line_sum_sq(const T* a, const T* b, int channels) {
    T sum = T(0);
    for (int c = 0; c < channels; ++c) {
        T lane = a[c] - b[c];
        T sq = lane * lane;
        sum = sum + sq;
    }
    return sum;
}

// The FP32 mirror's exponential. The reference writes `f32::exp` (helpers.rs:70-73,
// bilateral.rs:72); its lowering to device code happens inside CubeCL (ChillFish8/cubecl@e3c9246,
// not vendored), so its last-bit rounding is unknown. The mirror fixes one evaluation, written from
// the mathematics so a CUDA kernel can repeat it operation for operation:
//   n = rint(x * log2(e)), r = x - n*ln2 by Cody and Waite's two-constant reduction (ln2 split
//   into a 16-bit head, so n*head is exact, and the float nearest the remainder), |r| <= ln2/2;
//   e^r by its degree-7 Taylor polynomial (coefficients 1/k!) in Horner form with fused
//   multiply-adds (truncation error below 0.1 ulp on the reduced range);
//   e^x = e^r * 2^n, the power built exactly.
// x below -87 gives 0 (e^x would be subnormal) as does NaN; x above 88 overflows to +inf where
// n reaches 128. Measured against the double-precision exponential: within 1 ulp
// (tests/test_oracle_nlm.py).
constexpr float kExpLog2e = 1.44269502162933349609375f;     // float(log2(e))
constexpr float kExpLn2Hi = 0.693145751953125f;             // ln2 to 16 bits
constexpr float kExpLn2Lo = 1.428606765330187045037746e-06f;  // float(ln2 - kExpLn2Hi)

inline float exp_mirror(float x) {
    if (!(x >= -87.0f)) return 0.0f;
    const float n = std::rint(x * kExpLog2e);
    float r = std::fma(n, -kExpLn2Hi, x);
    r = std::fma(n, -kExpLn2Lo, r);
    float p = 1.0f / 5040.0f;
    p = std::fma(p, r, 1.0f / 720.0f);
    p = std::fma(p, r, 1.0f / 120.0f);
    p = std::fma(p, r, 1.0f / 24.0f);
    p = std::fma(p, r, 1.0f / 6.0f);
    p = std::fma(p, r, 0.5f);
    p = std::fma(p, r, 1.0f);
    p = std::fma(p, r, 1.0f);
    const int e = static_cast<int>(n) + 127;
    uint32_t bits = e >= 255 ? 0x7f800000u : static_cast<uint32_t>(e) << 23;
    float scale;
    std::memcpy(&scale, &bits, sizeof(scale));
    return p * scale;
}

inline float exp_of(float x) { return exp_mirror(x); }
inline double exp_of(double x) { return std::exp(x); }

// av-denoise-core/src/nlmeans/kernels/helpers.rs:70-73 (`welsch_weight`).
template <typename T>
inline T welsch(T sum, T h2, T off) {
    T excess = std::max(sum - off, T(0));
    return exp_of(-excess * h2);
}

// The patch distance of the direct (deterministic baseline) form: the distance tile element at
// tile position (tx, ty) is `line_sum_sq(centre[t] - neighbour[t + q]) * scale`
// (fused.rs:243-268, 460-477), summed row by row over the (2s+1)^2 patch (fused.rs:19-43).
template <typename T>
inline T patch_distance(const Frame<T>& centre, const Frame<T>& nbr, int px, int py, int qx, int qy,
                        int s, T scale) {
    T sum = T(0);
    const int C = centre.channels;
    if (px - s >= 0 && py - s >= 0 && px + s < centre.width && py + s < centre.height && px + qx - s >= 0 &&
        py + qy - s >= 0 && px + qx + s < centre.width && py + qy + s < centre.height) {
        // Every tap inside the frame: the same sums in the same order, without the clamps.
        const size_t row = static_cast<size_t>(centre.width) * C;
        const T* c = centre.data + (static_cast<size_t>(py - s) * centre.width + (px - s)) * C;
        const T* n = nbr.data + (static_cast<size_t>(py + qy - s) * centre.width + (px + qx - s)) * C;
        for (int oy = 0; oy <= 2 * s; ++oy, c += row, n += row) {
            for (int ox = 0; ox <= 2 * s; ++ox) {
                T d = line_sum_sq(c + ox * C, n + ox * C, C) * scale;
                sum = sum + d;
            }
        }
        return sum;
    }
    for (int oy = -s; oy <= s; ++oy) {
        for (int ox = -s; ox <= s; ++ox) {
            int tx = px + ox, ty = py + oy;
            const T* c = centre.at_clamped(tx, ty);
            const T* n = nbr.at_clamped(tx + qx, ty + qy);
            T d = line_sum_sq(c, n, centre.channels) * scale;
            sum = sum + d;
        }
    }
    return sum;
}

struct Conf {
    const float* fwd;  // per motion block, or null
    const float* bwd;
    int step, blocks_x, blocks_y;
};

// One output pixel of the windowed path, mirroring the launch order of `run_windowed_kernels`
// (dispatch/mod.rs:665-679): zeroed accumulators, one pair launch per q_k in -d..-1
// (`nlm_fused_pair_accumulate_window`, fused.rs:138-347), then the single-frame launch
// (`nlm_fused_single_window`, fused.rs:364-530), then `nlm_finish` (accumulate.rs:152-202).
// Each launch keeps register sums and adds them to the buffers once at its end. `refs` is the
// window the distances compare: the window itself, or a prefilter's reference frames (the `_ref`
// launches, fused.rs:532-900, which average the input's values all the same).
template <typename T>
void nlm_pixel(const std::vector<Frame<T>>& window, const std::vector<Frame<T>>& refs, int d, int px, int py,
               int a, int s, T h2, T noise_offset, const T* lut, const std::vector<Conf>& conf, T wref, T* out) {
    const int C = window[d].channels;
    const Frame<T>& ctr = window[d];
    const Frame<T>& rctr = refs[d];
    const T scale = channel_scale<T>(C);
    T accum[2] = {T(0), T(0)};
    T weight_sum = T(0);
    T max_weight = T(0);

    for (int k = 0; k < d; ++k) {
        // q_k = -d + k: the forward frame is centre + q_k, the backward frame centre - q_k.
        const Frame<T>& fwd = window[k];
        const Frame<T>& bwd = window[2 * d - k];
        const Frame<T>& rfwd = refs[k];
        const Frame<T>& rbwd = refs[2 * d - k];
        const Conf* cf = conf.empty() ? nullptr : &conf[k];
        T acc[2] = {T(0), T(0)};
        T ws = T(0), wm = T(0);
        for (int qy = -a; qy <= a; ++qy) {
            for (int qx = -a; qx <= a; ++qx) {
                T sum_f = patch_distance(rctr, rfwd, px, py, qx, qy, s, scale);
                T sum_b = patch_distance(rctr, rbwd, px, py, -qx, -qy, s, scale);
                T w_f = welsch(sum_f, h2, noise_offset);
                T w_b = welsch(sum_b, h2, noise_offset);
                if (cf && cf->fwd) {
                    int bc = std::min(px / cf->step, cf->blocks_x - 1);
                    int br = std::min(py / cf->step, cf->blocks_y - 1);
                    w_f = w_f * T(cf->fwd[br * cf->blocks_x + bc]);
                    w_b = w_b * T(cf->bwd[br * cf->blocks_x + bc]);
                }
                const T* fp = fwd.at_clamped(px + qx, py + qy);
                const T* bp = bwd.at_clamped(px - qx, py - qy);
                for (int c = 0; c < C; ++c) {
                    T t0 = fp[c] * w_f;
                    T t1 = acc[c] + t0;
                    T t2 = bp[c] * w_b;
                    acc[c] = t1 + t2;
                }
                ws = ws + (w_f + w_b);
                wm = std::max(wm, std::max(w_f, w_b));
            }
        }
        for (int c = 0; c < C; ++c) accum[c] = accum[c] + acc[c];
        weight_sum = weight_sum + ws;
        max_weight = std::max(max_weight, wm);
    }

    {
        T acc[2] = {T(0), T(0)};
        T ws = T(0), wm = T(0);
        const int side = 2 * a + 1;
        for (int qy = -a; qy <= a; ++qy) {
            for (int qx = -a; qx <= a; ++qx) {
                if (qx == 0 && qy == 0) continue;
                T dist = patch_distance(rctr, rctr, px, py, qx, qy, s, scale);
                T off = lut ? lut[(qy + a) * side + (qx + a)] : T(0);
                T w = welsch(dist, h2, off);
                const T* np = ctr.at_clamped(px + qx, py + qy);
                for (int c = 0; c < C; ++c) {
                    T t0 = np[c] * w;
                    acc[c] = acc[c] + t0;
                }
                ws = ws + w;
                wm = std::max(wm, w);
            }
        }
        for (int c = 0; c < C; ++c) accum[c] = accum[c] + acc[c];
        weight_sum = weight_sum + ws;
        max_weight = std::max(max_weight, wm);
    }

    // accumulate.rs:175-201 (`nlm_finish`).
    const T* orig = ctr.at_clamped(px, py);
    T self_weight = wref * max_weight;
    T denom = self_weight + weight_sum;
    for (int c = 0; c < C; ++c) {
        if (denom > T(1e-30)) {
            T inv = T(1) / denom;
            T num = orig[c] * self_weight + accum[c];
            out[c] = num * inv;
        } else {
            out[c] = orig[c];
        }
    }
}

template <typename T>
void nlm_window_frame(const T* const* frames, const T* const* ref_frames, int width, int height, int channels, int d,
                      int a, int s, T h2, T noise_offset, const T* lut, const float* const* conf_fwd,
                      const float* const* conf_bwd, int conf_step, int blocks_x, int blocks_y, T wref,
                      T* out) {
    std::vector<Frame<T>> window, refs;
    for (int i = 0; i < 2 * d + 1; ++i) window.push_back(Frame<T>{frames[i], width, height, channels});
    for (int i = 0; i < 2 * d + 1; ++i)
        refs.push_back(Frame<T>{ref_frames ? ref_frames[i] : frames[i], width, height, channels});
    std::vector<Conf> conf;
    if (conf_fwd) {
        for (int k = 0; k < d; ++k) conf.push_back(Conf{conf_fwd[k], conf_bwd[k], conf_step, blocks_x, blocks_y});
    }
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < height; ++y) {
        for (int x = 0; x < width; ++x) {
            nlm_pixel<T>(window, refs, d, x, y, a, s, h2, noise_offset, lut, conf, wref,
                         out + ((size_t)y * width + x) * channels);
        }
    }
}

}  // namespace

extern "C" {

// av-denoise-core/src/engine/kernels.rs:25-63 (`ingest_words`): code / max (a division), U/V
// interleaved into one ring slot. `samples_per_word` is 4 (u8) or 2 (u16).
void orc_ingest_words(const uint32_t* plane0, const uint32_t* plane1, float* slot, int64_t pixels,
                      int channels, int samples_per_word, float max_value) {
    const uint32_t bits = 32u / (uint32_t)samples_per_word;
    const uint32_t mask = (bits == 32u) ? 0xffffffffu : ((1u << bits) - 1u);
    for (int64_t p = 0; p < pixels; ++p) {
        int64_t word = p / samples_per_word;
        uint32_t shift = (uint32_t)(p % samples_per_word) * bits;
        uint32_t c0 = (plane0[word] >> shift) & mask;
        slot[p * channels] = (float)c0 / max_value;
        if (channels > 1) {
            uint32_t c1 = (plane1[word] >> shift) & mask;
            slot[p * channels + 1] = (float)c1 / max_value;
        }
    }
}

// av-denoise-core/src/engine/kernels.rs:64-90 (`ingest_f32`).
void orc_ingest_f32(const float* plane0, const float* plane1, float* slot, int64_t pixels, int channels,
                    float bias) {
    for (int64_t p = 0; p < pixels; ++p) {
        slot[p * channels] = plane0[p] + bias;
        if (channels > 1) slot[p * channels + 1] = plane1[p] + bias;
    }
}

// av-denoise-core/src/engine/kernels.rs:103-153 (`egress_words`): clamp to [0,1], then
// `u32(v * max + 0.5)` (truncating cast), packed per 32-bit word, zero padding.
void orc_egress_words(const float* frame, uint32_t* plane0, uint32_t* plane1, int64_t pixels, int channels,
                      int samples_per_word, float max_value) {
    const uint32_t bits = 32u / (uint32_t)samples_per_word;
    int64_t words = (pixels + samples_per_word - 1) / samples_per_word;
    for (int64_t w = 0; w < words; ++w) {
        uint32_t p0 = 0, p1 = 0;
        for (int lane = 0; lane < samples_per_word; ++lane) {
            int64_t p = w * samples_per_word + lane;
            if (p >= pixels) continue;
            uint32_t shift = (uint32_t)lane * bits;
            float v0 = std::min(std::max(frame[p * channels], 0.0f), 1.0f);
            float s0 = v0 * max_value;
            p0 |= (uint32_t)(s0 + 0.5f) << shift;
            if (channels > 1) {
                float v1 = std::min(std::max(frame[p * channels + 1], 0.0f), 1.0f);
                float s1 = v1 * max_value;
                p1 |= (uint32_t)(s1 + 0.5f) << shift;
            }
        }
        plane0[w] = p0;
        if (channels > 1) plane1[w] = p1;
    }
}

// av-denoise-core/src/engine/kernels.rs:159-184 (`egress_f32`).
void orc_egress_f32(const float* frame, float* plane0, float* plane1, int64_t pixels, int channels, float bias) {
    for (int64_t p = 0; p < pixels; ++p) {
        plane0[p] = frame[p * channels] - bias;
        if (channels > 1) plane1[p] = frame[p * channels + 1] - bias;
    }
}

// av-denoise-core/src/nlmeans/params.rs:229-233 (`h2_inv_norm_with`):
// NLM_NORM / (NLM_LEGACY * strength * strength * patch_area).
float orc_h2_inv_norm(float strength, int patch_radius) {
    int area = (2 * patch_radius + 1) * (2 * patch_radius + 1);
    float denom = 3.0f * strength;
    denom = denom * strength;
    denom = denom * (float)area;
    return (255.0f * 255.0f) / denom;
}

// av-denoise-core/src/nlmeans/kernels/helpers.rs:70-73, exposed for the host-formula pin.
float orc_welsch_weight(float sum, float h2, float off) { return welsch<float>(sum, h2, off); }

// The FP32 mirror's exponential over an array (its accuracy pin and the GPU comparison).
void orc_exp_mirror(const float* x, float* out, int64_t n) {
    for (int64_t i = 0; i < n; ++i) out[i] = exp_mirror(x[i]);
}

// One denoised frame of the windowed NLM path, FP32 mirror. `frames` holds the 2d+1 window
// frames (normalised f32, interleaved), the centre at index d; `refs` (null = `frames`) the
// window's reference frames the distances compare. `lut` is the (2a+1)^2 spatial offset table
// (null = zeros). `conf_fwd`/`conf_bwd` (null = off) hold, for pair k (q_k = -d+k), the per-block
// confidence of the forward and backward neighbour.
void orc_nlm_frame_ref_f32(const float* const* frames, const float* const* refs, int width, int height, int channels,
                           int d, int a, int s, float h2, float noise_offset, const float* lut,
                           const float* const* conf_fwd, const float* const* conf_bwd, int conf_step, int blocks_x,
                           int blocks_y, float wref, float* out) {
    nlm_window_frame<float>(frames, refs, width, height, channels, d, a, s, h2, noise_offset, lut, conf_fwd,
                            conf_bwd, conf_step, blocks_x, blocks_y, wref, out);
}

void orc_nlm_frame_f32(const float* const* frames, int width, int height, int channels, int d, int a, int s,
                       float h2, float noise_offset, const float* lut, const float* const* conf_fwd,
                       const float* const* conf_bwd, int conf_step, int blocks_x, int blocks_y, float wref,
                       float* out) {
    orc_nlm_frame_ref_f32(frames, nullptr, width, height, channels, d, a, s, h2, noise_offset, lut, conf_fwd,
                          conf_bwd, conf_step, blocks_x, blocks_y, wref, out);
}

// The same maths in FP64 (inputs widened from f32).
void orc_nlm_frame_ref_f64(const float* const* frames, const float* const* refs, int width, int height, int channels,
                           int d, int a, int s, double h2, double noise_offset, const float* lut,
                           const float* const* conf_fwd, const float* const* conf_bwd, int conf_step, int blocks_x,
                           int blocks_y, double wref, double* out) {
    const size_t n = (size_t)width * height * channels;
    auto widen = [&](const float* const* src, std::vector<std::vector<double>>& wide, std::vector<const double*>& ptrs) {
        wide.assign(2 * d + 1, std::vector<double>(n));
        for (int i = 0; i < 2 * d + 1; ++i) {
            for (size_t j = 0; j < n; ++j) wide[i][j] = src[i][j];
            ptrs.push_back(wide[i].data());
        }
    };
    std::vector<std::vector<double>> wide, wide_ref;
    std::vector<const double*> ptrs, ref_ptrs;
    widen(frames, wide, ptrs);
    if (refs) widen(refs, wide_ref, ref_ptrs);
    std::vector<double> lut64;
    if (lut) {
        int side = 2 * a + 1;
        lut64.assign(lut, lut + side * side);
    }
    nlm_window_frame<double>(ptrs.data(), refs ? ref_ptrs.data() : nullptr, width, height, channels, d, a, s, h2,
                             noise_offset, lut ? lut64.data() : nullptr, conf_fwd, conf_bwd, conf_step, blocks_x,
                             blocks_y, wref, out);
}

void orc_nlm_frame_f64(const float* const* frames, int width, int height, int channels, int d, int a, int s,
                       double h2, double noise_offset, const float* lut, const float* const* conf_fwd,
                       const float* const* conf_bwd, int conf_step, int blocks_x, int blocks_y, double wref,
                       double* out) {
    orc_nlm_frame_ref_f64(frames, nullptr, width, height, channels, d, a, s, h2, noise_offset, lut, conf_fwd,
                          conf_bwd, conf_step, blocks_x, blocks_y, wref, out);
}

// av-denoise-core/src/nlmeans/kernels/bilateral.rs:16-107 (`nlm_bilateral`), FP32 mirror: the
// (2r+1)^2 clamped neighbours in row-major order, each weight
// exp(-((dx^2 + dy^2) * inv_s + sum_c (n_c - c_c)^2 * inv_r)), and the weighted sum times the
// reciprocal of the weight sum. `radius` is max(ceil(2 sigma_s), 1) and inv_s, inv_r are
// 1 / (2 sigma^2) (prefilter/bilateral.rs:11-22).
void orc_bilateral_f32(const float* frame, int width, int height, int channels, int radius, float inv_s,
                       float inv_r, float* out) {
    const Frame<float> f{frame, width, height, channels};
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < height; ++y) {
        for (int x = 0; x < width; ++x) {
            const float* c = f.at_clamped(x, y);
            float acc[2] = {0.0f, 0.0f};
            float wsum = 0.0f;
            for (int oy = 0; oy <= 2 * radius; ++oy) {
                for (int ox = 0; ox <= 2 * radius; ++ox) {
                    const int dy = oy - radius, dx = ox - radius;
                    const float* n = f.at_clamped(x + dx, y + dy);
                    float range_sq = 0.0f;
                    for (int ch = 0; ch < channels; ++ch) {
                        float lane = n[ch] - c[ch];
                        float sq = lane * lane;
                        range_sq = range_sq + sq;
                    }
                    float spatial = (float)(dx * dx + dy * dy) * inv_s;
                    float r = range_sq * inv_r;
                    float w = exp_mirror(-(spatial + r));
                    for (int ch = 0; ch < channels; ++ch) {
                        float t = n[ch] * w;
                        acc[ch] = acc[ch] + t;
                    }
                    wsum = wsum + w;
                }
            }
            const float inv = 1.0f / wsum;
            float* o = out + ((size_t)y * width + x) * channels;
            for (int ch = 0; ch < channels; ++ch) o[ch] = acc[ch] * inv;
        }
    }
}

}  // extern "C"
