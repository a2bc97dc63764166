// Host-only half of the ABI: option defaults, presets, parameter resolution and validation.
// Nothing here touches the GPU, so every function runs (and is tested) on a machine without one.

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "avd_internal.h"

namespace avd {

namespace {

// av-denoise-core/src/nlmeans/params.rs:12-15.
constexpr float kHqStrengthLuma[9] = {0.45f, 0.45f, 0.42f, 0.42f, 0.35f, 0.35f, 0.35f, 0.30f, 0.30f};
constexpr float kHqStrengthChroma[9] = {1.00f, 0.85f, 0.70f, 0.70f, 0.70f, 0.70f, 0.70f, 0.70f, 0.70f};

std::string fmt(const char* f, ...) __attribute__((format(printf, 1, 2)));
std::string fmt(const char* f, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, f);
    vsnprintf(buf, sizeof(buf), f, ap);
    va_end(ap);
    return std::string(buf);
}

bool finite(float v) { return std::isfinite(v); }

// av-denoise-core/src/motion/search.rs:229-290 (`MotionCompensationMode::validate`) and
// :143-156 (`MotionEstimation::validate`).
std::string validate_motion(const AvdMotionCompensation& m) {
    if (!m.active) return {};
    const AvdMotionSearch& s = m.search;
    if (s.blksize < 4)
        return fmt("motion-compensation blksize=%u is too small, the minimum is 4 pixels per side", s.blksize);
    if (s.blksize > kMaxBlksize)
        return fmt("motion-compensation blksize=%u exceeds the supported maximum of %u", s.blksize, kMaxBlksize);
    if (s.blksize % 2 != 0)
        return fmt("motion-compensation blksize=%u must be even so the /2 coarse level is well-defined", s.blksize);
    if (s.overlap >= s.blksize)
        return fmt("motion-compensation overlap=%u must be strictly less than blksize, which is %u, so the step "
                   "between blocks stays positive",
                   s.overlap, s.blksize);
    if (s.search_radius == 0 || s.search_radius > kMotionMaxSearchRadius)
        return fmt("motion-compensation search_radius=%u must be in 1..=%u", s.search_radius, kMotionMaxSearchRadius);
    if (s.max_search_escalation < s.search_radius || s.max_search_escalation > kMotionMaxSearchRadius)
        return fmt("motion-compensation max_search_escalation=%u must be between search_radius, which is %u, and %u",
                   s.max_search_escalation, s.search_radius, kMotionMaxSearchRadius);
    if (s.pyramid_levels == 0 || s.pyramid_levels > kMaxPyramidLevels)
        return fmt("motion-compensation pyramid_levels=%u must be in 1..=%u", s.pyramid_levels, kMaxPyramidLevels);
    if (s.estimation > AVD_ESTIMATION_CHAINED) return fmt("unknown motion estimation kind %u", s.estimation);
    if (s.estimation == AVD_ESTIMATION_CHAINED && (s.refine_radius == 0 || s.refine_radius > kMotionMaxSearchRadius))
        return fmt("motion-estimation refine_radius=%u must be in 1..=%u", s.refine_radius, kMotionMaxSearchRadius);
    return {};
}

bool motion_equal(const AvdMotionCompensation& a, uint32_t ra, const AvdMotionCompensation& b, uint32_t rb) {
    // `PassSpec::motion` is `Some((mode, radius))` only when active and radius > 0 (spec.rs:75-86).
    bool aa = a.active && ra > 0, bb = b.active && rb > 0;
    if (aa != bb) return false;
    if (!aa) return true;
    const AvdMotionSearch &x = a.search, &y = b.search;
    bool chained_x = x.estimation == AVD_ESTIMATION_CHAINED, chained_y = y.estimation == AVD_ESTIMATION_CHAINED;
    return ra == rb && x.blksize == y.blksize && x.overlap == y.overlap && x.search_radius == y.search_radius &&
           x.max_search_escalation == y.max_search_escalation && x.pyramid_levels == y.pyramid_levels &&
           x.estimation == y.estimation && (!chained_x || !chained_y || x.refine_radius == y.refine_radius);
}

AvdMotionCompensation nl4d_motion(const AvdNl4dOptions& o) {
    AvdMotionCompensation m{};
    m.active = 1;
    m.search = o.motion;
    return m;
}

// av-denoise-core/src/nl4d/options.rs:101-106.
float nl4d_default_lambda_ht(Channels c) { return c == Channels::Luma ? 4.158f : 3.234f; }

// av-denoise-core/src/nl4d/options.rs:127-185 (`resolve_lambda_ht`, `resolve_params`) and
// nl4d/params.rs:119-197 (`Nl4dParams::validate`), then the front's `NlmParams::validate`.
std::string validate_nl4d(const AvdNl4dOptions& o, Channels c) {
    if (o.temporal_radius == 0) return "nl4d needs a temporal radius of at least 1";
    if (!(finite(o.lambda_ht_scale) && o.lambda_ht_scale >= 0.1f && o.lambda_ht_scale <= 10.0f))
        return fmt("lambda_ht_scale must be finite and in 0.1..=10.0, got %g", o.lambda_ht_scale);
    float lambda_ht = (o.has_lambda_ht ? o.lambda_ht : nl4d_default_lambda_ht(c)) * o.lambda_ht_scale;
    AvdMotionCompensation m = nl4d_motion(o);
    if (m.search.overlap < m.search.blksize) {
        uint32_t step = m.search.blksize - m.search.overlap;
        uint32_t covers = (m.search.blksize + step - 1) / step;
        if (covers > kMaxCoveringBlocks)
            return fmt("nlm.motion_compensation blksize=%u at overlap=%u gives a step of %u, so %u blocks cover a "
                       "patch on each axis, past the %u the temporal grouping kernel unrolls its search over. "
                       "Raise the step by lowering the overlap.",
                       m.search.blksize, m.search.overlap, step, covers, kMaxCoveringBlocks);
    }
    if (o.temporal_radius < 1 || o.temporal_radius > kMaxTemporalRadius)
        return fmt("temporal_radius=%u must be in 1..=%u", o.temporal_radius, kMaxTemporalRadius);
    if (o.refine < 1 || o.refine > 4) return fmt("refine=%u must be in 1..=4", o.refine);
    if (o.spatial_radius < 1 || o.spatial_radius > 16)
        return fmt("spatial_radius=%u must be in 1..=16", o.spatial_radius);
    if (!(finite(lambda_ht) && lambda_ht > 0.0f))
        return fmt("lambda_ht must be finite and greater than 0, got %g", lambda_ht);
    if (!(finite(o.c_min) && o.c_min >= 0.0f && o.c_min < 1.0f))
        return fmt("c_min must be finite, at least 0 and below 1, got %g", o.c_min);
    if (!(finite(o.kaiser_beta) && o.kaiser_beta >= 0.0f && o.kaiser_beta <= kMaxKaiserBeta))
        return fmt("kaiser_beta must be finite and in 0..=%g, got %g", kMaxKaiserBeta, o.kaiser_beta);
    if (!(finite(o.field_lambda) && o.field_lambda >= 0.0f))
        return fmt("field_lambda must be finite and at least 0, got %g", o.field_lambda);
    // The front end's own `NlmParams::validate` (nl4d/options.rs:149-160 builds it).
    NlmParams front;
    front.channels = c;
    front.temporal_radius = o.temporal_radius;
    front.motion = m;
    front.hq = true;
    front.hq_params.has_sigma_override = o.has_sigma != 0;
    front.hq_params.sigma_override = o.sigma;
    front.hq_params.sigma_scale = o.sigma_scale;
    front.hq_params.thsad_scale = o.thsad_scale;
    return validate_nlm_params(front);
}

}  // namespace

// av-denoise-core/src/nlmeans/prefilter/bilateral.rs:11-22.
uint32_t bilateral_radius(float sigma_s) {
    float r = std::ceil(2.0f * sigma_s);
    uint32_t radius = r > 0.0f ? static_cast<uint32_t>(r) : 0u;
    return std::max(radius, 1u);
}
float inv_two_sigma_sq(float sigma) { return 1.0f / (2.0f * sigma * sigma); }

float sample_max_value(const AvdSampleFormat& f) {
    switch (f.kind) {
        case AVD_SAMPLE_U8: return 255.0f;
        case AVD_SAMPLE_U16: return static_cast<float>((1u << f.depth) - 1u);
        default: return 1.0f;
    }
}

uint32_t samples_per_word(const AvdSampleFormat& f) {
    switch (f.kind) {
        case AVD_SAMPLE_U8: return 4;
        case AVD_SAMPLE_U16: return 2;
        default: return 1;
    }
}

uint64_t plane_bytes(const AvdSampleFormat& f, uint64_t pixels) {
    uint64_t spw = samples_per_word(f);
    return (pixels + spw - 1) / spw * 4;
}

bool formats_equal(const AvdSampleFormat& a, const AvdSampleFormat& b) {
    if (a.kind != b.kind) return false;
    return a.kind != AVD_SAMPLE_U16 || a.depth == b.depth;
}

uint32_t plane_count(uint32_t chroma_layout) { return chroma_layout == AVD_CHROMA_GRAY ? 1u : 3u; }

void plane_dims(const AvdGeometry& g, size_t index, uint32_t* w, uint32_t* h) {
    *w = g.width;
    *h = g.height;
    if (index == 0) return;
    switch (g.chroma) {
        case AVD_CHROMA_YUV420: *w = (g.width + 1) / 2; *h = (g.height + 1) / 2; break;
        case AVD_CHROMA_YUV422: *w = (g.width + 1) / 2; break;
        default: break;
    }
}

NlmParams resolve_nlm_params(const AvdNlmeansAlgorithm& alg, Channels channels) {
    NlmParams p;
    p.channels = channels;
    p.temporal_radius = alg.mode.temporal ? alg.mode.radius : 0;
    p.hq = alg.variant == 1;
    if (p.hq) {
        p.hq_params.auto_strength = alg.hq.auto_strength != 0;
        p.hq_params.noise_floor = alg.hq.noise_floor != 0;
        p.hq_params.has_sigma_override = alg.hq.has_sigma_override != 0;
        p.hq_params.sigma_override = alg.hq.sigma_override;
        p.hq_params.temporal_confidence = alg.hq.temporal_confidence != 0;
        p.hq_params.thsad_scale = alg.hq.thsad_scale;
        p.hq_params.sigma_scale = alg.hq.sigma_scale;
    }
    float default_strength = 1.2f;
    if (p.hq && p.hq_params.auto_strength) default_strength = avd_hq_default_strength(p.channel_count(), p.temporal_radius);
    p.strength = alg.tuning.has_strength ? alg.tuning.strength : default_strength;
    p.search_radius = alg.tuning.has_search_radius ? alg.tuning.search_radius : 2u;
    p.patch_radius = alg.tuning.has_patch_radius ? alg.tuning.patch_radius : 4u;
    p.self_weight = alg.tuning.has_self_weight ? alg.tuning.self_weight : 1.0f;
    p.prefilter = alg.prefilter;
    p.motion = alg.motion_compensation;
    return p;
}

std::string validate_nlm_params(const NlmParams& p) {
    if (p.patch_radius > kMaxPatchRadius)
        return fmt("patch_radius=%u exceeds the supported maximum of %u, because larger patches exhaust on-chip "
                   "shared memory in the fused and windowed kernels",
                   p.patch_radius, kMaxPatchRadius);
    if (p.search_radius > kMaxSearchRadius)
        return fmt("search_radius=%u exceeds the supported maximum of %u. The windowed kernel's search window loop "
                   "is fully unrolled, so both its compiled size and its build time grow with search_radius",
                   p.search_radius, kMaxSearchRadius);
    if (p.temporal_radius > kMaxTemporalRadius)
        return fmt("temporal_radius=%u exceeds the supported maximum of %u, because the ring buffer grows in step "
                   "with the window size",
                   p.temporal_radius, kMaxTemporalRadius);
    if (!(finite(p.strength) && p.strength > 0.0f))
        return fmt("strength must be finite and greater than 0, got %g. A strength of 0 produces an infinite "
                   "Welsch normalisation factor",
                   p.strength);
    if (!finite(p.self_weight) || p.self_weight < 0.0f)
        return fmt("self_weight must be finite and 0 or greater, got %g", p.self_weight);
    if (p.hq) {
        const HqParams& hq = p.hq_params;
        if (hq.has_sigma_override &&
            (!finite(hq.sigma_override) || hq.sigma_override <= 0.0f || hq.sigma_override > 1.0f))
            return fmt("hq sigma_override must be finite, above 0 and at most 1 in normalised units, got %g",
                       hq.sigma_override);
        if (!(finite(hq.thsad_scale) && hq.thsad_scale > 0.0f))
            return fmt("hq thsad_scale must be finite and greater than 0, got %g. A thsad_scale of 0 collapses every "
                       "block's confidence to zero no matter how well it matches",
                       hq.thsad_scale);
        if (!(finite(hq.sigma_scale) && hq.sigma_scale >= 0.1f && hq.sigma_scale <= 10.0f))
            return fmt("hq sigma_scale must be finite and in 0.1..=10.0, got %g", hq.sigma_scale);
    }
    if (p.prefilter.kind > AVD_PREFILTER_NLM_SPATIAL) return fmt("unknown prefilter kind %u", p.prefilter.kind);
    if (p.prefilter.kind == AVD_PREFILTER_BILATERAL) {
        float ss = p.prefilter.sigma_s, sr = p.prefilter.sigma_r;
        if (!finite(ss) || ss <= 0.0f)
            return fmt("bilateral prefilter sigma_s must be finite and greater than 0, got %g. A sigma_s of 0 "
                       "produces an infinite spatial-weight normalisation factor",
                       ss);
        if (!finite(sr) || sr <= 0.0f)
            return fmt("bilateral prefilter sigma_r must be finite and greater than 0, got %g. A sigma_r of 0 "
                       "produces an infinite range-weight normalisation factor, which turns the centre tap into NaN",
                       sr);
        uint32_t r = bilateral_radius(ss);
        if (r > kMaxBilateralRadius)
            return fmt("bilateral prefilter sigma_s=%g implies a shared-memory tile radius of %u, from radius = "
                       "ceil(2 * sigma_s) with a minimum of 1. That is past the supported maximum of %u, and larger "
                       "radii exhaust on-chip shared memory in the bilateral kernel",
                       ss, r, kMaxBilateralRadius);
        if (!finite(inv_two_sigma_sq(ss)))
            return fmt("bilateral prefilter sigma_s is too small, got %g. Squaring it underflows to 0 in f32, which "
                       "makes the spatial-weight normalisation factor infinite",
                       ss);
        if (!finite(inv_two_sigma_sq(sr)))
            return fmt("bilateral prefilter sigma_r is too small, got %g. Squaring it underflows to 0 in f32, which "
                       "makes the range-weight normalisation factor infinite and the centre tap NaN",
                       sr);
    }
    if (p.prefilter.kind == AVD_PREFILTER_NLM_SPATIAL) {
        float sc = p.prefilter.strength_scale;
        if (!finite(sc) || sc <= 0.0f)
            return fmt("nlm pilot strength_scale must be finite and greater than 0, got %g", sc);
        if (p.patch_radius > kSeparableThreshold)
            return fmt("the nlm pilot uses the windowed spatial kernel, which supports patch_radius up to %u (got %u)",
                       kSeparableThreshold, p.patch_radius);
    }
    return validate_motion(p.motion);
}

float h2_inv_norm_with(const NlmParams& p, bool has_sigma, float sigma) {
    uint32_t area = (2 * p.patch_radius + 1) * (2 * p.patch_radius + 1);
    float strength = p.strength;
    if (p.hq && p.hq_params.auto_strength && has_sigma) strength = p.strength * sigma * 255.0f;
    float denom = 3.0f * strength;
    denom = denom * strength;
    denom = denom * static_cast<float>(area);
    return (255.0f * 255.0f) / denom;
}

float noise_offset_with(const NlmParams& p, const float* sigmas, int n) {
    if (!(p.hq && p.hq_params.noise_floor) || sigmas == nullptr) return 0.0f;
    uint32_t area = (2 * p.patch_radius + 1) * (2 * p.patch_radius + 1);
    float scale = p.channels == Channels::Luma ? 3.0f : 1.5f;
    int count = std::min<int>(n, static_cast<int>(p.channel_count()));
    float sum_sq = 0.0f;
    for (int i = 0; i < count; ++i) sum_sq = sum_sq + sigmas[i] * sigmas[i];
    float r = 2.0f * scale;
    r = r * sum_sq;
    return r * static_cast<float>(area);
}

size_t nlm_held_frames(const AvdNlmeansAlgorithm& alg, Channels channels) {
    NlmParams p = resolve_nlm_params(alg, channels);
    bool measures = p.hq && !p.hq_params.has_sigma_override;  // denoiser/noise.rs:50-52
    return p.temporal_radius + (measures ? kLookaheadFrames : 0u);
}

// nl4d/engine.rs:33-35: the whole window either side, plus the noise look-ahead when measured.
size_t nl4d_held_frames(const AvdNl4dOptions& o, Channels) {
    bool measures = o.has_sigma == 0;
    return 2 * o.temporal_radius + (measures ? kLookaheadFrames : 0u);
}

float nl4d_lambda_ht(const AvdNl4dOptions& o, Channels c) {
    return (o.has_lambda_ht ? o.lambda_ht : nl4d_default_lambda_ht(c)) * o.lambda_ht_scale;
}

// nl4d/options.rs:108-117: the calibrated pooled threshold 2.42 over the plane's default lambda.
float nl4d_pool_ratio(Channels c) { return 2.42f / nl4d_default_lambda_ht(c); }

AvdStatus validate_spec(const AvdEngineSpec& spec, std::string* message) {
    auto fail = [&](AvdStatus st, std::string m) {
        if (message) *message = std::move(m);
        return st;
    };
    const AvdGeometry& g = spec.geometry;
    if (spec.kind > AVD_ENGINE_NL4D) return fail(AVD_ERR_INVALID_OPTIONS, fmt("unknown engine kind %u", spec.kind));
    if (g.chroma > AVD_CHROMA_YUV444) return fail(AVD_ERR_INVALID_GEOMETRY, fmt("unknown chroma layout %u", g.chroma));
    for (const AvdSampleFormat* f : {&g.input, &g.output}) {
        if (f->kind > AVD_SAMPLE_F32) return fail(AVD_ERR_INVALID_GEOMETRY, fmt("unknown sample kind %u", f->kind));
        if (f->kind == AVD_SAMPLE_U16 && (f->depth < 9 || f->depth > 16))
            return fail(AVD_ERR_INVALID_GEOMETRY, fmt("U16 depth must be between 9 and 16, got %u", f->depth));
    }
    bool has_luma = spec.has_luma != 0, has_chroma = spec.has_chroma != 0;
    if (!has_luma && !has_chroma) return fail(AVD_ERR_INVALID_OPTIONS, "a spec must clean luma, chroma or both");
    bool gray = g.chroma == AVD_CHROMA_GRAY;
    if (has_chroma && gray) return fail(AVD_ERR_INVALID_GEOMETRY, "a gray frame has no chroma planes to clean");
    bool passes_through = !gray && has_luma != has_chroma;
    if (passes_through && !formats_equal(g.input, g.output))
        return fail(AVD_ERR_INVALID_GEOMETRY, "an uncleaned plane needs the same input and output format");

    bool nl4d = spec.kind == AVD_ENGINE_NL4D;
    // Window spans and motion of the luma (or guide) pass against the chroma pass (spec.rs:320-341).
    auto span_and_motion = [&](bool luma_side, size_t* held, AvdMotionCompensation* m, uint32_t* radius) {
        Channels c = luma_side ? Channels::Luma : Channels::Chroma;
        if (nl4d) {
            const AvdNl4dOptions& o = luma_side ? (has_luma ? spec.nl4d_luma : spec.nl4d_chroma) : spec.nl4d_chroma;
            *held = nl4d_held_frames(o, c);
            *m = nl4d_motion(o);
            *radius = o.temporal_radius;
        } else {
            const AvdNlmeansAlgorithm& a = luma_side ? (has_luma ? spec.nlm_luma : spec.nlm_chroma) : spec.nlm_chroma;
            *held = nlm_held_frames(a, c);
            NlmParams p = resolve_nlm_params(a, c);
            *m = p.motion;
            *radius = p.temporal_radius;
        }
    };
    if (has_chroma) {
        bool chroma_motion;
        size_t held_c;
        AvdMotionCompensation mc;
        uint32_t rc;
        span_and_motion(false, &held_c, &mc, &rc);
        chroma_motion = mc.active && rc > 0;
        // The luma motion pass is the luma pass, or the guide built from the chroma settings.
        if (has_luma || chroma_motion) {
            size_t held_l;
            AvdMotionCompensation ml;
            uint32_t rl;
            span_and_motion(true, &held_l, &ml, &rl);
            if (held_l != held_c)
                return fail(AVD_ERR_INVALID_OPTIONS,
                            fmt("the luma pass reads %zu frames either side but the chroma pass reads %zu", held_l,
                                held_c));
            if (!motion_equal(ml, rl, mc, rc))
                return fail(AVD_ERR_INVALID_OPTIONS,
                            "the chroma pass takes its motion from the luma pass, so both need the same motion search "
                            "and temporal radius");
        }
    }

    // Per-pass build checks (nlmeans/engine.rs:64-91; nl4d/engine.rs builds through the same front).
    for (int side = 0; side < 2; ++side) {
        bool present = side == 0 ? has_luma : has_chroma;
        if (!present) continue;
        Channels c = side == 0 ? Channels::Luma : Channels::Chroma;
        uint32_t w, h;
        plane_dims(g, side == 0 ? 0 : 1, &w, &h);
        if (w < kMinFrameDim || h < kMinFrameDim)
            return fail(AVD_ERR_INVALID_GEOMETRY,
                        fmt("frame dimensions %ux%u are below the supported minimum of %ux%u, because the noise "
                            "estimate needs at least one interior pixel",
                            w, h, kMinFrameDim, kMinFrameDim));
        uint32_t slots;
        if (nl4d) {
            std::string e = validate_nl4d(side == 0 ? spec.nl4d_luma : spec.nl4d_chroma, c);
            if (!e.empty()) return fail(AVD_ERR_INVALID_OPTIONS, e);
            slots = 2 * (side == 0 ? spec.nl4d_luma : spec.nl4d_chroma).temporal_radius + 1;
        } else {
            NlmParams p = resolve_nlm_params(side == 0 ? spec.nlm_luma : spec.nlm_chroma, c);
            std::string e = validate_nlm_params(p);
            if (!e.empty()) return fail(AVD_ERR_INVALID_OPTIONS, e);
            slots = p.total_frames();
        }
        // engine/plane.rs:330-346 (`check_ring_fits`).
        uint64_t elements = static_cast<uint64_t>(w) * h * static_cast<uint32_t>(c) * slots;
        if (elements > 0xffffffffull)
            return fail(AVD_ERR_INVALID_GEOMETRY,
                        fmt("a %u frame ring of %ux%u planes stores more than u32::MAX elements", slots, w, h));
    }
    return AVD_OK;
}

}  // namespace avd

using namespace avd;

// Defined with the engine; records the message `avd_last_error` returns.
void avd_set_last_error(const std::string& m);

extern "C" {

uint32_t avd_abi_version(void) { return AVD_ABI_VERSION; }

const char* avd_status_message(AvdStatus status) {
    switch (status) {
        case AVD_OK: return "ok";
        case AVD_ERR_INVALID_OPTIONS: return "invalid options";
        case AVD_ERR_INVALID_GEOMETRY: return "invalid geometry";
        case AVD_ERR_PLANE_MISMATCH: return "plane mismatch";
        case AVD_ERR_OUTPUTS_PENDING: return "every ready frame must be emitted before the next push";
        case AVD_ERR_NOTHING_TO_EMIT: return "no frame is ready to emit";
        case AVD_ERR_CONTEXT_AFTER_PUSH: return "context frames must come before the first push of a stream";
        case AVD_ERR_NEEDS_RESET: return "an earlier call failed, reset the engine before using it again";
        case AVD_ERR_GPU: return "gpu error";
        case AVD_ERR_NULL_ARG: return "null argument";
        case AVD_ERR_QUEUE_FULL: return "frames in flight must be collected before the next push";
        case AVD_ERR_POISONED: return "an earlier call failed, reset the stream before using it again";
    }
    return "unknown status";
}

void avd_default_motion_search(AvdMotionSearch* out) {
    if (!out) return;
    std::memset(out, 0, sizeof(*out));
    out->blksize = 16;
    out->overlap = 8;
    out->search_radius = 4;
    out->max_search_escalation = 4;
    out->pyramid_levels = 2;
    out->estimation = AVD_ESTIMATION_AUTO;
    out->refine_radius = kDefaultRefineRadius;
}

void avd_default_nlmeans(AvdNlmeansAlgorithm* out) {
    if (!out) return;
    std::memset(out, 0, sizeof(*out));
    out->variant = 0;
    out->prefilter.kind = AVD_PREFILTER_NONE;
    out->motion_compensation.active = 0;
    avd_default_motion_search(&out->motion_compensation.search);
    out->mode.temporal = 0;
    out->hq.auto_strength = 1;
    out->hq.noise_floor = 1;
    out->hq.has_sigma_override = 0;
    out->hq.temporal_confidence = 1;
    out->hq.thsad_scale = 1.0f;
    out->hq.sigma_scale = 1.0f;
}

void avd_default_nl4d(AvdNl4dOptions* out) {
    if (!out) return;
    std::memset(out, 0, sizeof(*out));
    avd_default_motion_search(&out->motion);
    out->has_sigma = 0;
    out->sigma_scale = 1.0f;
    out->thsad_scale = 1.0f;
    out->refine = 2;
    out->spatial_radius = 9;
    out->has_lambda_ht = 0;
    out->lambda_ht_scale = 1.0f;
    out->c_min = 0.05f;
    out->kaiser_beta = 2.0f;
    out->field_lambda = 1.0f;
    out->noise_map = 1;
    out->pooled_threshold = 1;
    out->grain_data = 0;
    out->temporal_radius = 2;
}

uint32_t avd_nlmeans_variant_for(uint32_t preset) { return preset == AVD_PRESET_VERYFAST ? 0u : 1u; }

uint32_t avd_nlmeans_temporal_radius_for(uint32_t preset) {
    switch (preset) {
        case AVD_PRESET_VERYFAST: return 0;
        case AVD_PRESET_FAST: return 1;
        case AVD_PRESET_BASE: return 2;
        case AVD_PRESET_SLOW: return 4;
        default: return 8;
    }
}

uint32_t avd_nlmeans_search_radius_for(uint32_t preset) { return preset >= AVD_PRESET_SLOW ? 4u : 2u; }

uint32_t avd_search_escalation_for(uint32_t preset) { return preset >= AVD_PRESET_SLOW ? kMotionMaxSearchRadius : 0u; }

float avd_hq_default_strength(uint32_t channels, uint32_t temporal_radius) {
    uint32_t i = std::min(temporal_radius, kMaxTemporalRadius);
    return channels == 1 ? kHqStrengthLuma[i] : kHqStrengthChroma[i];
}

AvdStatus avd_spec_validate(const AvdEngineSpec* spec, char* msg, size_t msg_len) {
    if (!spec) return AVD_ERR_NULL_ARG;
    std::string m;
    AvdStatus st = validate_spec(*spec, &m);
    avd_set_last_error(m);
    if (msg && msg_len) {
        std::snprintf(msg, msg_len, "%s", m.c_str());
    }
    return st;
}

AvdStatus avd_spec_window_span(const AvdEngineSpec* spec, AvdWindowSpan* out) {
    if (!spec || !out) return AVD_ERR_NULL_ARG;
    bool nl4d = spec->kind == AVD_ENGINE_NL4D;
    size_t held = 0;
    if (spec->has_luma) {
        held = nl4d ? nl4d_held_frames(spec->nl4d_luma, Channels::Luma)
                    : nlm_held_frames(spec->nlm_luma, Channels::Luma);
    } else if (spec->has_chroma) {
        held = nl4d ? nl4d_held_frames(spec->nl4d_chroma, Channels::Chroma)
                    : nlm_held_frames(spec->nlm_chroma, Channels::Chroma);
    }
    out->behind = held;
    out->ahead = held;
    out->edges = nl4d ? 1u : 0u;
    out->reserved = 0;
    return AVD_OK;
}

}  // extern "C"
