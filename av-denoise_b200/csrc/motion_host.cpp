// Host side of the motion search and noise estimator entry points: argument checks, then the
// launches of motion.cu and immerkaer.cu.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "avd_internal.h"
#include "kernels.h"

void avd_set_last_error(const std::string& m);

namespace {
AvdStatus fail(AvdStatus s, const std::string& m) {
    avd_set_last_error(m);
    return s;
}
}  // namespace

extern "C" {

uint64_t avd_motion_pyramid_floats(uint32_t width, uint32_t height, uint32_t frame_count, uint32_t levels) {
    return static_cast<uint64_t>(avd::pyramid_floats(static_cast<int>(width), static_cast<int>(height),
                                                     static_cast<int>(frame_count), static_cast<int>(levels)));
}

AvdStatus avd_motion_pyramid_build(uint64_t ring, uint32_t channels, uint32_t width, uint32_t height,
                                   uint32_t frame_count, uint32_t ring_slot, uint32_t levels, uint64_t pyramid,
                                   uint32_t pyramid_slot, void* stream) {
    if (!ring || !pyramid) return fail(AVD_ERR_NULL_ARG, "motion pyramid: null buffer");
    if (channels < 1 || channels > 2 || width == 0 || height == 0)
        return fail(AVD_ERR_INVALID_GEOMETRY, "motion pyramid: bad geometry");
    if (levels < 1 || levels > 3) return fail(AVD_ERR_INVALID_OPTIONS, "motion pyramid: levels must be in 1..=3");
    if (pyramid_slot >= frame_count) return fail(AVD_ERR_INVALID_OPTIONS, "motion pyramid: slot past frame_count");
    cudaError_t e = avd::launch_pyramid_build(reinterpret_cast<const float*>(ring), static_cast<int>(channels),
                                              static_cast<int>(width), static_cast<int>(height),
                                              static_cast<int>(frame_count), static_cast<int>(ring_slot),
                                              static_cast<int>(levels), reinterpret_cast<float*>(pyramid),
                                              static_cast<int>(pyramid_slot), static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, std::string("motion pyramid launch: ") + cudaGetErrorString(e));
    return AVD_OK;
}

AvdStatus avd_motion_search(const AvdMotionPass* p, void* stream) {
    if (!p || !p->pyramid || !p->neighbour_slots || !p->mv_field)
        return fail(AVD_ERR_NULL_ARG, "motion search: null buffer");
    if (p->width == 0 || p->height == 0 || p->neighbours == 0 || p->centre_slot >= p->frame_count)
        return fail(AVD_ERR_INVALID_GEOMETRY, "motion search: bad geometry");
    if (p->blksize < 2 || p->blksize > 32 || p->overlap >= p->blksize)
        return fail(AVD_ERR_INVALID_OPTIONS, "motion search: blksize must be in 2..=32 and overlap below it");
    if (p->search_radius > 8) return fail(AVD_ERR_INVALID_OPTIONS, "motion search: search_radius must be at most 8");
    if (p->levels < 1 || p->levels > 3) return fail(AVD_ERR_INVALID_OPTIONS, "motion search: levels must be in 1..=3");
    if (p->confidence && (!p->noise || !(p->thsad > 0.0f)))
        return fail(AVD_ERR_INVALID_OPTIONS, "motion search: confidence needs the noise words and a positive thsad");
    const uint32_t step = p->blksize - p->overlap;
    const uint32_t bx = (p->width + step - 1) / step, by = (p->height + step - 1) / step;
    if (p->mv_stride < 2 * bx * by || (p->confidence && p->conf_stride < bx * by))
        return fail(AVD_ERR_INVALID_OPTIONS, "motion search: field strides below the block count");
    avd::MotionLaunch m{};
    m.pyramid = reinterpret_cast<const float*>(p->pyramid);
    m.neighbour_slots = reinterpret_cast<const uint32_t*>(p->neighbour_slots);
    m.mv_field = reinterpret_cast<int32_t*>(p->mv_field);
    m.confidence = reinterpret_cast<float*>(p->confidence);
    m.noise = reinterpret_cast<const float*>(p->noise);
    m.width = static_cast<int>(p->width);
    m.height = static_cast<int>(p->height);
    m.frame_count = static_cast<int>(p->frame_count);
    m.centre_slot = static_cast<int>(p->centre_slot);
    m.neighbours = static_cast<int>(p->neighbours);
    m.blksize = static_cast<int>(p->blksize);
    m.overlap = static_cast<int>(p->overlap);
    m.search_radius = static_cast<int>(p->search_radius);
    m.coarse_radius = static_cast<int>(p->coarse_radius ? p->coarse_radius : p->search_radius);
    m.coarse_block_factor = p->coarse_block_factor > 1 ? static_cast<int>(p->coarse_block_factor) : 1;
    if (p->levels > 1 && (m.coarse_radius > 12 || (m.coarse_radius > 8 && m.coarse_radius != 12)))
        return fail(AVD_ERR_INVALID_OPTIONS, "motion search: coarse_radius must be in 1..=8 or 12");
    if (p->levels > 1 && m.coarse_block_factor > 4)
        return fail(AVD_ERR_INVALID_OPTIONS, "motion search: coarse_block_factor must be at most 4");
    if (p->predictions && !p->noise)
        return fail(AVD_ERR_INVALID_OPTIONS, "motion search: the camera model needs the noise words");
    if (p->sad && p->conf_stride < bx * by)
        return fail(AVD_ERR_INVALID_OPTIONS, "motion search: SAD output needs conf_stride >= blocks");
    m.predictions = reinterpret_cast<const float*>(p->predictions);
    m.sad = reinterpret_cast<float*>(p->sad);
    m.levels = static_cast<int>(p->levels);
    m.mv_stride = static_cast<int>(p->mv_stride);
    m.conf_stride = static_cast<int>(p->conf_stride);
    m.sad_floor_word = static_cast<int>(p->sad_floor_word);
    m.thsad = p->thsad;
    m.seeded = p->seeded ? 1 : 0;
    m.keep_seeds = reinterpret_cast<int32_t*>(p->keep_seeds);
    if (p->escalation && p->ceiling > p->search_radius) {
        if (p->ceiling > 8) return fail(AVD_ERR_INVALID_OPTIONS, "motion search: ceiling must be at most 8");
        if (!p->noise || !(p->thsad > 0.0f) || p->conf_stride < bx * by)
            return fail(AVD_ERR_INVALID_OPTIONS,
                        "motion search: escalation needs the noise words, a positive thsad and conf_stride >= blocks");
        m.escalation = reinterpret_cast<float*>(p->escalation);
        m.ceiling = static_cast<int>(p->ceiling);
        m.esc_reads_floor = p->esc_reads_floor ? 1 : 0;
    }
    cudaError_t e = avd::launch_motion_search(m, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, std::string("motion search launch: ") + cudaGetErrorString(e));
    return AVD_OK;
}

uint64_t avd_escalation_state_floats(uint32_t neighbours, uint32_t conf_stride) {
    return static_cast<uint64_t>(avd::escalation_state_floats(static_cast<int>(neighbours), static_cast<int>(conf_stride)));
}

AvdStatus avd_truemotion_pass(const AvdTruemotionPass* p, void* stream) {
    if (!p || !p->pyramid || !p->neighbour_slots || !p->mv_in || !p->mv_out || !p->noise)
        return fail(AVD_ERR_NULL_ARG, "truemotion: null buffer");
    if (p->mv_in == p->mv_out) return fail(AVD_ERR_INVALID_OPTIONS, "truemotion: mv_out must not be mv_in");
    if (p->width == 0 || p->height == 0 || p->neighbours == 0 || p->centre_slot >= p->frame_count)
        return fail(AVD_ERR_INVALID_GEOMETRY, "truemotion: bad geometry");
    if (p->blksize < 2 || p->blksize > 32 || p->overlap >= p->blksize)
        return fail(AVD_ERR_INVALID_OPTIONS, "truemotion: blksize must be in 2..=32 and overlap below it");
    if (!(p->field_lambda > 0.0f) || !std::isfinite(p->field_lambda) || !(p->thsad >= 0.0f))
        return fail(AVD_ERR_INVALID_OPTIONS, "truemotion: field_lambda must be finite and positive");
    const uint32_t step = p->blksize - p->overlap;
    const uint32_t bx = std::max<uint32_t>((p->width + step - 1) / step, 1);
    const uint32_t by = std::max<uint32_t>((p->height + step - 1) / step, 1);
    if (p->mv_stride < 2 * bx * by || (p->confidence && p->conf_stride < bx * by))
        return fail(AVD_ERR_INVALID_OPTIONS, "truemotion: field strides below the block count");
    avd::TruemotionLaunch t{};
    t.pyramid = reinterpret_cast<const float*>(p->pyramid);
    t.slot_pixels = avd::pyramid_slot_pixels(static_cast<int>(p->width), static_cast<int>(p->height), 0);
    t.neighbour_slots = reinterpret_cast<const uint32_t*>(p->neighbour_slots);
    t.mv_in = reinterpret_cast<const int32_t*>(p->mv_in);
    t.seeds = reinterpret_cast<const int32_t*>(p->seeds);
    t.mv_out = reinterpret_cast<int32_t*>(p->mv_out);
    t.confidence = reinterpret_cast<float*>(p->confidence);
    t.noise = reinterpret_cast<const float*>(p->noise);
    t.width = static_cast<int>(p->width);
    t.height = static_cast<int>(p->height);
    t.centre_slot = static_cast<int>(p->centre_slot);
    t.neighbours = static_cast<int>(p->neighbours);
    t.blksize = static_cast<int>(p->blksize);
    t.step = static_cast<int>(step);
    t.blocks_x = static_cast<int>(bx);
    t.blocks_y = static_cast<int>(by);
    t.mv_stride = static_cast<int>(p->mv_stride);
    t.conf_stride = static_cast<int>(p->conf_stride);
    t.sad_field = static_cast<int>(p->sad_field);
    t.reads_floor = p->reads_floor ? 1 : 0;
    t.refine_radius = 1;
    // motion/truemotion/stage.rs:52-62 with params.rs:4-33.
    t.lambda_base = p->field_lambda * static_cast<float>(p->blksize * p->blksize) * 0.02f;
    t.lambda_noise = p->field_lambda * 1.0f;
    t.surcharge = 0.125f;
    t.fade_level = 2.0f * std::max(p->thsad, 0.0f);
    t.thsad = p->thsad;
    t.predictions = reinterpret_cast<const float*>(p->predictions);
    t.sad = reinterpret_cast<float*>(p->sad);
    if (t.sad && p->conf_stride < bx * by)
        return fail(AVD_ERR_INVALID_OPTIONS, "truemotion: SAD output needs conf_stride >= blocks");
    cudaError_t e = avd::launch_truemotion(t, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, std::string("truemotion launch: ") + cudaGetErrorString(e));
    return AVD_OK;
}

AvdStatus avd_chain_compose(uint64_t pair_ring, uint64_t mv_field, uint32_t mv_stride, uint32_t centre,
                            uint32_t temporal_radius, uint32_t head_mod, uint32_t dir_stride, uint32_t width,
                            uint32_t height, uint32_t blksize, uint32_t overlap, void* stream) {
    if (!pair_ring || !mv_field) return fail(AVD_ERR_NULL_ARG, "chain compose: null buffer");
    if (temporal_radius < 1 || temporal_radius > avd::kMaxTemporalRadius || centre > 2 * temporal_radius ||
        overlap >= blksize || width == 0 || height == 0)
        return fail(AVD_ERR_INVALID_OPTIONS, "chain compose: bad window or geometry");
    const int step = static_cast<int>(blksize - overlap);
    const int bx = std::max<int>((static_cast<int>(width) + step - 1) / step, 1);
    const int by = std::max<int>((static_cast<int>(height) + step - 1) / step, 1);
    cudaError_t e = avd::launch_chain_compose(
        reinterpret_cast<const int32_t*>(pair_ring), reinterpret_cast<int32_t*>(mv_field), static_cast<int>(mv_stride),
        static_cast<int>(centre), static_cast<int>(temporal_radius), static_cast<int>(head_mod),
        static_cast<int>(dir_stride), 2 * static_cast<int>(dir_stride), step, static_cast<int>(width),
        static_cast<int>(height), bx, by, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, std::string("chain compose launch: ") + cudaGetErrorString(e));
    return AVD_OK;
}

// confidence.rs:17-21: area * 2 * sigma / sqrt(pi), evaluated left to right in f32, with sqrt(pi)
// the f32 square root of the f32 pi.
float avd_sad_noise_floor(uint32_t blksize, float sigma) {
    const float area = static_cast<float>(blksize * blksize);
    const volatile float pi = 3.14159265358979323846f;
    return area * 2.0f * sigma / std::sqrt(static_cast<float>(pi));
}

// confidence.rs:27-30.
float avd_thsad(uint32_t blksize, float thsad_scale) {
    const float area = static_cast<float>(blksize * blksize);
    return thsad_scale * area * 0.02f;
}

uint64_t avd_immerkaer_partials_len(uint32_t width, uint32_t height) {
    return avd::immerkaer_partials_len(static_cast<int>(width), static_cast<int>(height));
}

// noise/spatial.rs:142-144: the scale is the f32 square root of the f32 pi / 2.
AvdStatus avd_immerkaer(uint64_t frame, uint32_t channels, uint32_t width, uint32_t height, uint64_t partials,
                        uint64_t results, uint64_t sigma_low, void* stream) {
    if (!frame || !partials) return fail(AVD_ERR_NULL_ARG, "immerkaer: null buffer");
    if (channels < 1 || channels > 2 || width == 0 || height == 0)
        return fail(AVD_ERR_INVALID_GEOMETRY, "immerkaer: bad geometry");
    const volatile float half_pi = 1.57079632679489661923f;
    const float scale = std::sqrt(static_cast<float>(half_pi));
    cudaError_t e = avd::launch_immerkaer(reinterpret_cast<const float*>(frame), static_cast<int>(channels),
                                          static_cast<int>(width), static_cast<int>(height), scale,
                                          reinterpret_cast<float*>(partials), reinterpret_cast<float*>(results),
                                          reinterpret_cast<float*>(sigma_low), static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, std::string("immerkaer launch: ") + cudaGetErrorString(e));
    return AVD_OK;
}

uint64_t avd_nlm_backward_scratch_bytes(uint32_t width, uint32_t height) {
    return avd::nlm_backward_scratch_floats(static_cast<int>(width), static_cast<int>(height)) * sizeof(float);
}

AvdStatus avd_nlm_backward(const AvdNlmBackward* p, void* stream) {
    if (!p || !p->window || !p->grad_out || !p->grad_window || !p->grad_strength || !p->scratch)
        return fail(AVD_ERR_NULL_ARG, "nlm backward: null buffer");
    if (p->channels < 1 || p->channels > 2 || p->width < 1 || p->height < 1)
        return fail(AVD_ERR_INVALID_GEOMETRY, "nlm backward: bad geometry");
    if (p->temporal_radius > avd::kMaxTemporalRadius || p->search_radius > avd::kMaxSearchRadius ||
        p->patch_radius > avd::kMaxPatchRadius)
        return fail(AVD_ERR_INVALID_OPTIONS, "nlm backward: radius past the NLMeans limits");
    if (avd::nlm_backward_smem_bytes(static_cast<int>(p->channels), static_cast<int>(p->temporal_radius),
                                     static_cast<int>(p->search_radius), static_cast<int>(p->patch_radius)) >
        226u * 1024u)
        return fail(AVD_ERR_INVALID_OPTIONS,
                    "nlm backward: the staged frames and gradient tiles exceed the 226 KiB of dynamic shared memory a "
                    "CTA may hold");
    if (!(p->strength > 0.0f)) return fail(AVD_ERR_INVALID_OPTIONS, "nlm backward: strength must be positive");
    avd::NlmBackwardLaunch l{};
    l.window = reinterpret_cast<const float*>(p->window);
    l.grad_out = reinterpret_cast<const float*>(p->grad_out);
    l.grad_window = reinterpret_cast<float*>(p->grad_window);
    l.grad_strength = reinterpret_cast<float*>(p->grad_strength);
    l.scratch = reinterpret_cast<float*>(p->scratch);
    l.width = static_cast<int>(p->width);
    l.height = static_cast<int>(p->height);
    l.channels = static_cast<int>(p->channels);
    l.temporal_radius = static_cast<int>(p->temporal_radius);
    l.search_radius = static_cast<int>(p->search_radius);
    l.patch_radius = static_cast<int>(p->patch_radius);
    l.strength = p->strength;
    // nlmeans/params.rs:229-233, in the same f32 order as the forward's strength word.
    const float area = static_cast<float>((2 * p->patch_radius + 1) * (2 * p->patch_radius + 1));
    l.h2 = (255.0f * 255.0f) / ((3.0f * p->strength * p->strength) * area);
    l.wref = p->self_weight;
    l.pair_offset = p->pair_offset;
    l.spatial_offset = p->spatial_offset;
    cudaError_t e = avd::launch_nlm_backward(l, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, std::string("nlm backward launch: ") + cudaGetErrorString(e));
    return AVD_OK;
}

uint64_t avd_nlm_window_scratch_bytes(uint32_t search_radius) {
    return (8 + static_cast<uint64_t>(2 * search_radius + 1) * (2 * search_radius + 1)) * sizeof(float);
}

AvdStatus avd_nlm_window(const AvdNlmBackward* p, void* stream) {
    if (!p || !p->window || !p->grad_out || !p->scratch) return fail(AVD_ERR_NULL_ARG, "nlm window: null buffer");
    if (p->channels < 1 || p->channels > 2 || p->width < avd::kMinFrameDim || p->height < avd::kMinFrameDim)
        return fail(AVD_ERR_INVALID_GEOMETRY, "nlm window: bad geometry");
    if (p->temporal_radius > avd::kMaxTemporalRadius || p->search_radius > avd::kMaxSearchRadius ||
        p->patch_radius > avd::kMaxPatchRadius)
        return fail(AVD_ERR_INVALID_OPTIONS, "nlm window: radius past the NLMeans limits");
    if (!(p->strength > 0.0f)) return fail(AVD_ERR_INVALID_OPTIONS, "nlm window: strength must be positive");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const float area = static_cast<float>((2 * p->patch_radius + 1) * (2 * p->patch_radius + 1));
    const float h2 = (255.0f * 255.0f) / ((3.0f * p->strength * p->strength) * area);
    float* words = reinterpret_cast<float*>(p->scratch);
    cudaError_t e = avd::launch_window_words(words, h2, p->pair_offset, p->spatial_offset,
                                             static_cast<int>(p->search_radius), s);
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, cudaGetErrorString(e));
    const int d = static_cast<int>(p->temporal_radius);
    avd::NlmLaunch a{};
    a.ring = reinterpret_cast<const float*>(p->window);
    a.width = static_cast<int>(p->width);
    a.height = static_cast<int>(p->height);
    a.channels = static_cast<int>(p->channels);
    a.frame_elems = static_cast<int64_t>(p->width) * p->height * p->channels;
    a.slot_centre = d;
    a.pairs = d;
    for (int k = 0; k < d; ++k) {
        a.slot_fwd[k] = k;
        a.slot_bwd[k] = 2 * d - k;
    }
    a.patch_radius = static_cast<int>(p->patch_radius);
    a.search_radius = static_cast<int>(p->search_radius);
    a.derived = words;
    a.h2_word = 0;
    a.offset_word = 1;
    const bool plain = p->pair_offset == 0.0f && p->spatial_offset == 0.0f;
    a.spatial_lut = plain ? nullptr : words + 8;
    a.conf = nullptr;
    a.wref = p->self_weight;
    a.fast = plain ? 1 : 0;
    a.out = reinterpret_cast<float*>(p->grad_out);
    e = avd::launch_nlm(a, s);
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, std::string("nlm window launch: ") + cudaGetErrorString(e));
    return AVD_OK;
}

}  // extern "C"

AvdStatus avd_exp_mirror(uint64_t x, uint64_t out, uint64_t n, void* stream) {
    if ((x == 0 || out == 0) && n > 0) return AVD_ERR_NULL_ARG;
    cudaError_t e = avd::launch_exp_mirror(reinterpret_cast<const float*>(x), reinterpret_cast<float*>(out),
                                           static_cast<int64_t>(n), static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        avd_set_last_error(cudaGetErrorString(e));
        return AVD_ERR_GPU;
    }
    return AVD_OK;
}

// ---- the camera model (include/avd.h) --------------------------------------------------------------

uint64_t avd_model_fit_scratch_floats(uint32_t blocks) {
    return static_cast<uint64_t>(avd::model_fit_scratch_floats(static_cast<int>(blocks)));
}

AvdStatus avd_model_fit(const AvdModelFit* p, void* stream) {
    if (!p || !p->field || !p->models || !p->scratch) return fail(AVD_ERR_NULL_ARG, "model fit: null buffer");
    if (p->width == 0 || p->height == 0 || p->blksize < 2 || p->blksize > 32 || p->overlap >= p->blksize)
        return fail(AVD_ERR_INVALID_GEOMETRY, "model fit: bad geometry");
    if (p->has_contrast && !p->sad) return fail(AVD_ERR_INVALID_OPTIONS, "model fit: contrast needs the SADs");
    const uint32_t step = p->blksize - p->overlap;
    const uint32_t bx = std::max<uint32_t>((p->width + step - 1) / step, 1);
    const uint32_t by = std::max<uint32_t>((p->height + step - 1) / step, 1);
    if (p->has_contrast && p->means_offset < bx * by)
        return fail(AVD_ERR_INVALID_OPTIONS, "model fit: means_offset below the block count");
    if (bx + by > 12 * 1024) return fail(AVD_ERR_INVALID_GEOMETRY, "model fit: block grid too large");
    avd::ModelFitLaunch l{};
    l.field = reinterpret_cast<const int32_t*>(p->field);
    l.sad = reinterpret_cast<const float*>(p->sad);
    l.has_contrast = p->has_contrast != 0;
    l.means_offset = static_cast<int>(p->means_offset);
    l.older_to_newer = p->older_to_newer != 0;
    l.width = static_cast<int>(p->width);
    l.height = static_cast<int>(p->height);
    l.blksize = static_cast<int>(p->blksize);
    l.step = static_cast<int>(step);
    l.prior = p->prior;
    l.models = reinterpret_cast<float*>(p->models);
    l.slot = static_cast<int>(p->slot);
    l.scratch = reinterpret_cast<float*>(p->scratch);
    cudaError_t e = avd::launch_model_fit(l, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, std::string("model fit launch: ") + cudaGetErrorString(e));
    return AVD_OK;
}

AvdStatus avd_compose_models(uint64_t models, uint64_t gaps, uint64_t out, uint32_t neighbours, uint32_t max_steps,
                             uint32_t past_neighbours, void* stream) {
    if (!models || !out || (max_steps && !gaps)) return fail(AVD_ERR_NULL_ARG, "compose models: null buffer");
    if (neighbours == 0 || past_neighbours > neighbours) return fail(AVD_ERR_INVALID_OPTIONS, "compose models: bad counts");
    cudaError_t e = avd::launch_compose_models(reinterpret_cast<const float*>(models),
                                               reinterpret_cast<const uint32_t*>(gaps), reinterpret_cast<float*>(out),
                                               static_cast<int>(neighbours), static_cast<int>(max_steps),
                                               static_cast<int>(past_neighbours), static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, std::string("compose models launch: ") + cudaGetErrorString(e));
    return AVD_OK;
}

AvdStatus avd_block_means(uint64_t plane, uint64_t out, uint32_t width, uint32_t height, uint32_t blksize,
                          uint32_t overlap, void* stream) {
    if (!plane || !out) return fail(AVD_ERR_NULL_ARG, "block means: null buffer");
    if (width == 0 || height == 0 || blksize == 0 || overlap >= blksize)
        return fail(AVD_ERR_INVALID_GEOMETRY, "block means: bad geometry");
    cudaError_t e = avd::launch_block_means(reinterpret_cast<const float*>(plane), reinterpret_cast<float*>(out),
                                            static_cast<int>(width), static_cast<int>(height), static_cast<int>(blksize),
                                            static_cast<int>(blksize - overlap), static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, std::string("block means launch: ") + cudaGetErrorString(e));
    return AVD_OK;
}

AvdStatus avd_high_pass(uint64_t plane, uint64_t rows, uint64_t out, uint32_t width, uint32_t height, uint32_t radius,
                        void* stream) {
    if (!plane || !rows || !out) return fail(AVD_ERR_NULL_ARG, "high pass: null buffer");
    if (width == 0 || height == 0 || radius > 64) return fail(AVD_ERR_INVALID_GEOMETRY, "high pass: bad geometry");
    cudaError_t e = avd::launch_high_pass(reinterpret_cast<const float*>(plane), reinterpret_cast<float*>(rows),
                                          reinterpret_cast<float*>(out), static_cast<int>(width),
                                          static_cast<int>(height), static_cast<int>(radius),
                                          static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, std::string("high pass launch: ") + cudaGetErrorString(e));
    return AVD_OK;
}
