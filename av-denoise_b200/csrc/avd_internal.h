// Internal types shared by the host engine and the CUDA kernels of libavd_b200.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

#include "avd.h"

namespace avd {

// av-denoise-core/src/nlmeans/params.rs:56-84.
constexpr uint32_t kSeparableThreshold = 8;
constexpr uint32_t kMaxPatchRadius = 16;
constexpr uint32_t kMaxSearchRadius = 8;
constexpr uint32_t kMaxTemporalRadius = 8;
constexpr uint32_t kMaxBilateralRadius = 22;
constexpr uint32_t kMinFrameDim = 3;  // params.rs:39
// av-denoise-core/src/motion/search.rs:158-194.
constexpr uint32_t kMotionMaxSearchRadius = 8;
constexpr uint32_t kMaxPyramidLevels = 3;
constexpr uint32_t kMaxBlksize = 32;
constexpr uint32_t kChainedRadiusThreshold = 3;
constexpr uint32_t kDefaultRefineRadius = 2;
// av-denoise-core/src/noise/history.rs (NOISE_WINDOW_RADIUS) = the HQ look-ahead depth,
// nlmeans/denoiser/lookahead.rs:30.
constexpr uint32_t kLookaheadFrames = 8;
// av-denoise-core/src/nl4d/params.rs:12-20.
constexpr float kMaxKaiserBeta = 8.0f;
constexpr uint32_t kMaxCoveringBlocks = 4;

enum class Channels : uint32_t { Luma = 1, Chroma = 2 };

// av-denoise-core/src/nlmeans/params.rs:113-145 (`HqParams`).
struct HqParams {
    bool auto_strength = true;
    bool noise_floor = true;
    bool has_sigma_override = false;
    float sigma_override = 0.0f;
    bool temporal_confidence = true;
    float thsad_scale = 1.0f;
    float sigma_scale = 1.0f;
};

// av-denoise-core/src/nlmeans/params.rs:170-198 (`NlmParams`), resolved.
struct NlmParams {
    uint32_t temporal_radius = 0;
    uint32_t search_radius = 2;
    uint32_t patch_radius = 4;
    float strength = 1.2f;
    float self_weight = 1.0f;
    Channels channels = Channels::Luma;
    AvdPrefilter prefilter{};
    AvdMotionCompensation motion{};
    bool hq = false;
    HqParams hq_params{};

    uint32_t total_frames() const { return 1 + 2 * temporal_radius; }
    uint32_t channel_count() const { return static_cast<uint32_t>(channels); }
};

// Resolves `NlmeansAlgorithm` into `NlmParams` (nlmeans/options.rs:106-137).
NlmParams resolve_nlm_params(const AvdNlmeansAlgorithm& algorithm, Channels channels);

// `NlmParams::validate` (nlmeans/params.rs:276-428); returns an empty string when valid.
std::string validate_nlm_params(const NlmParams& p);

// `NlmParams::h2_inv_norm_with` (params.rs:229-233).
float h2_inv_norm_with(const NlmParams& p, bool has_sigma, float sigma);
// `NlmParams::noise_offset_with` for equal sigmas on every active channel (params.rs:245-268).
float noise_offset_with(const NlmParams& p, const float* sigmas, int n);

// The bilateral prefilter's kernel radius, max(ceil(2 sigma_s), 1), and its Gaussian factor
// 1 / (2 sigma^2) (nlmeans/prefilter/bilateral.rs:11-22).
uint32_t bilateral_radius(float sigma_s);
float inv_two_sigma_sq(float sigma);

// The frames a pass holds before it emits one (nlmeans/engine.rs:24-26, 187-192;
// nl4d/engine.rs:217-222).
size_t nlm_held_frames(const AvdNlmeansAlgorithm& algorithm, Channels channels);
size_t nl4d_held_frames(const AvdNl4dOptions& options, Channels channels);

// nl4d/options.rs:101-132: the plane's resolved hard-threshold multiplier and pooled ratio.
float nl4d_lambda_ht(const AvdNl4dOptions& options, Channels channels);
float nl4d_pool_ratio(Channels channels);

// Sample-format helpers (engine/plane.rs:229-263).
float sample_max_value(const AvdSampleFormat& f);
uint32_t samples_per_word(const AvdSampleFormat& f);
uint64_t plane_bytes(const AvdSampleFormat& f, uint64_t pixels);
bool formats_equal(const AvdSampleFormat& a, const AvdSampleFormat& b);

// Plane dimensions of a geometry (engine/frame.rs:399-418, 469-477).
uint32_t plane_count(uint32_t chroma_layout);
void plane_dims(const AvdGeometry& g, size_t index, uint32_t* w, uint32_t* h);

// Full spec validation with the per-pass build checks; writes the message.
AvdStatus validate_spec(const AvdEngineSpec& spec, std::string* message);

// Automatic noise estimate (noise_host.cpp): noise/temporal.rs:83-100 and noise/fold.rs:118-146.
struct FoldCoefficients {
    float sigma_scale = 1.0f;
    bool curve_applies = false;
    float weight_g_max = 0.0f;
    float weight_floor = 1e-12f;
    bool h2_auto = false;
    float h2_per_inverse_variance = 0.0f;
    float h2_fixed = 0.0f;
    float pilot_h2_factor = 1.0f;
    float offset_per_variance = 0.0f;
    bool main_offset = true;
    float sad_per_sigma = 0.0f;
    float confidence_sad_per_sigma = 0.0f;
};
uint32_t min_static_blocks(uint32_t total);
float immerkaer_sigma_scale();
void noise_fold_words(uint32_t width, uint32_t height, const FoldCoefficients& k, float* words);

}  // namespace avd
