// Host side of the camera models: the pair-model producer (av-denoise-core/src/motion/global/
// producer.rs) and the window and pair predictions the luma motion pass searches from
// (nlmeans/denoiser/seeds.rs).

#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "engine_parts.h"
#include "kernels.h"

namespace avd {

namespace {
constexpr int kPyramidSlots = 2;           // producer.rs:41-42: the newest frame and the one before it
constexpr int kHighPassRadius = 8;         // producer.rs:44-49
constexpr int kAcquisitionRadius = 12;     // producer.rs:51-52
constexpr int kAcquisitionFactor = 2;      // producer.rs:54-57
constexpr int kDeepLevels = 3;             // motion/search.rs:183 (MAX_PYRAMID_LEVELS)
constexpr int kZeroNoiseWords = 64;        // covers every noise word a search reads
constexpr uint32_t kNoPair = 0xFFFFFFFFu;  // global/compose.rs:11-12

float thsad_of(int blksize) {  // motion/confidence.rs:26-29 at thsad_scale 1
    return 1.0f * static_cast<float>(blksize * blksize) * 0.02f;
}
}  // namespace

std::optional<Failure> PairModels::allocate(const AvdGeometry& g, const PairModelMode& mode, size_t depth) {
    geometry_ = g;
    mode_ = mode;
    depth_ = depth;
    const int w = static_cast<int>(g.width), h = static_cast<int>(g.height);
    const int step = mode.blksize - mode.overlap;
    blocks_x_ = std::max((w + step - 1) / step, 1);
    blocks_y_ = std::max((h + step - 1) / step, 1);
    const size_t blocks = static_cast<size_t>(blocks_x_) * blocks_y_;
    conf_stride_ = static_cast<int>((blocks + 7) / 8 * 8);
    mv_stride_ = 2 * conf_stride_;
    const size_t plane = static_cast<size_t>(w) * h;
    cudaError_t e;
    if ((e = models_.alloc(depth * kModelWords * sizeof(float))) != cudaSuccess ||
        (e = luma_.alloc(plane * sizeof(float))) != cudaSuccess || (e = rows_.alloc(plane * sizeof(float))) != cudaSuccess ||
        (e = high_.alloc(plane * sizeof(float))) != cudaSuccess ||
        (e = pyramid_.alloc(static_cast<size_t>(pyramid_floats(w, h, kPyramidSlots, kDeepLevels)) * sizeof(float))) !=
            cudaSuccess ||
        (e = field_.alloc(mv_stride_ * sizeof(int32_t))) != cudaSuccess ||
        (e = seeds_.alloc(mv_stride_ * sizeof(int32_t))) != cudaSuccess ||
        (e = tm_field_.alloc(mv_stride_ * sizeof(int32_t))) != cudaSuccess ||
        (e = changes_.alloc(conf_stride_ * sizeof(uint32_t))) != cudaSuccess ||
        (e = sad_.alloc(3 * conf_stride_ * sizeof(float))) != cudaSuccess ||
        (e = predictions_.alloc(kAffineWords * sizeof(float))) != cudaSuccess ||
        (e = escalation_.alloc(escalation_state_floats(1, conf_stride_) * sizeof(float))) != cudaSuccess ||
        (e = scratch_.alloc(model_fit_scratch_floats(static_cast<int>(blocks)) * sizeof(float))) != cudaSuccess ||
        (e = zero_noise_.alloc(kZeroNoiseWords * sizeof(float))) != cudaSuccess)
        return Failure{AVD_ERR_GPU, cuda_message("camera model buffers", e)};
    // global/model.rs:21-27: every model starts invalid.
    if ((e = cudaMemset(models_.ptr, 0, models_.bytes)) != cudaSuccess ||
        (e = cudaMemset(zero_noise_.ptr, 0, zero_noise_.bytes)) != cudaSuccess)
        return Failure{AVD_ERR_GPU, cuda_message("camera model clear", e)};
    return std::nullopt;
}

// producer.rs:433-480 (`match_pair`): the older frame's blocks matched into the newer one, the deep
// first search ending with the truemotion stage (whose SADs replace the search's), the refit search
// with the mode's own reach around the prediction.
std::optional<Failure> PairModels::match(bool deep, int older, int newer, cudaStream_t s) {
    const bool escalates = mode_.ceiling > mode_.search_radius;
    MotionLaunch m{};
    m.pyramid = pyramid_.as<float>();
    m.inline_slots[0] = static_cast<uint32_t>(newer);
    m.mv_field = field_.as<int32_t>();
    m.noise = zero_noise();  // the producer has no noise reading (producer.rs:189-190)
    m.width = static_cast<int>(geometry_.width);
    m.height = static_cast<int>(geometry_.height);
    m.frame_count = kPyramidSlots;
    m.centre_slot = older;
    m.neighbours = 1;
    m.blksize = mode_.blksize;
    m.overlap = mode_.overlap;
    m.search_radius = mode_.search_radius;
    m.coarse_radius = deep ? kAcquisitionRadius : mode_.search_radius;
    m.coarse_block_factor = deep ? kAcquisitionFactor : 1;
    m.levels = deep ? kDeepLevels : mode_.levels;
    m.mv_stride = mv_stride_;
    m.conf_stride = conf_stride_;
    m.sad_floor_word = 0;
    m.thsad = thsad_of(mode_.blksize);  // the library's unscaled thsad (producer.rs:428-431)
    m.sad = sad_.as<float>();
    if (escalates) {
        m.escalation = escalation_.as<float>();
        m.ceiling = mode_.ceiling;
        m.esc_reads_floor = 0;
    }
    const bool coarse = m.levels > 1;
    if (!deep) m.predictions = predictions_.as<float>();
    if (deep && coarse) m.keep_seeds = seeds_.as<int32_t>();
    cudaError_t e = launch_motion_search(m, s);
    if (e != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("camera model search", e)};
    if (!deep) return std::nullopt;
    // motion/truemotion/stage.rs:29-145 at the default field_lambda 1, the floor unread.
    TruemotionLaunch t{};
    t.pyramid = m.pyramid;
    t.slot_pixels = pyramid_slot_pixels(m.width, m.height, 0);
    t.inline_slots[0] = m.inline_slots[0];
    t.mv_in = field_.as<int32_t>();
    t.seeds = coarse ? seeds_.as<int32_t>() : nullptr;
    t.mv_out = tm_field_.as<int32_t>();
    t.noise = zero_noise();
    t.width = m.width;
    t.height = m.height;
    t.centre_slot = older;
    t.neighbours = 1;
    t.blksize = mode_.blksize;
    t.step = mode_.blksize - mode_.overlap;
    t.blocks_x = blocks_x_;
    t.blocks_y = blocks_y_;
    t.mv_stride = mv_stride_;
    t.conf_stride = conf_stride_;
    t.refine_radius = 1;
    t.lambda_base = 1.0f * static_cast<float>(mode_.blksize * mode_.blksize) * 0.02f;
    t.lambda_noise = 1.0f * 1.0f;
    t.surcharge = 0.125f;
    t.fade_level = 2.0f * std::max(m.thsad, 0.0f);
    t.thsad = m.thsad;
    t.sad = sad_.as<float>();
    if (escalates) {
        // truemotion/stage.rs:82-142: two passes, the second rescoring the blocks next to a change.
        t.changes_out = changes_.as<uint32_t>();
        if ((e = launch_truemotion(t, s)) != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("camera model truemotion", e)};
        t.mv_in = tm_field_.as<int32_t>();
        t.mv_out = field_.as<int32_t>();
        t.changes_in = changes_.as<uint32_t>();
        t.changes_out = nullptr;
        if ((e = launch_truemotion(t, s)) != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("camera model truemotion", e)};
        return std::nullopt;
    }
    if ((e = launch_truemotion(t, s)) != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("camera model truemotion", e)};
    e = cudaMemcpyAsync(field_.ptr, tm_field_.ptr, mv_stride_ * sizeof(int32_t), cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("camera model field copy", e)};
    return std::nullopt;
}

std::optional<Failure> PairModels::push(const AvdPlane& luma, uint32_t frame, cudaStream_t s) {
    const int w = static_cast<int>(geometry_.width), h = static_cast<int>(geometry_.height);
    const int newer = static_cast<int>(frame % kPyramidSlots);
    // producer.rs:374-413 (`build_pyramid`): the normalised luma, its block means (the third SAD
    // section), its high pass at level 0 of the newer pyramid slot, and the coarser levels.
    cudaError_t e = launch_ingest(reinterpret_cast<const void*>(luma.ptr), nullptr, luma_.as<float>(),
                                  static_cast<int64_t>(w) * h, 1, plane_format(geometry_.input), 0.0f, s);
    if (e == cudaSuccess)
        e = launch_block_means(luma_.as<float>(), sad_.as<float>() + 2 * conf_stride_, w, h, mode_.blksize,
                               mode_.blksize - mode_.overlap, s);
    if (e == cudaSuccess) e = launch_high_pass(luma_.as<float>(), rows_.as<float>(), high_.as<float>(), w, h, kHighPassRadius, s);
    if (e == cudaSuccess)
        e = launch_pyramid_build(high_.as<float>(), 1, w, h, kPyramidSlots, 0, kDeepLevels, pyramid_.as<float>(), newer, s);
    if (e != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("camera model pyramid", e)};
    // producer.rs:110-125 (`Run::continues_to`): the next frame, or the last one again.
    const bool follows = running_ && run_first_ < frame && (run_last_ == frame || run_last_ + 1 == frame);
    if (!follows) {
        running_ = true;
        run_first_ = run_last_ = frame;
        if ((e = launch_model_identity(models_.as<float>(), static_cast<int>(slot(frame)), s)) != cudaSuccess)
            return Failure{AVD_ERR_GPU, cuda_message("camera model identity", e)};
        return std::nullopt;
    }
    run_last_ = frame;
    const int older = static_cast<int>((frame - 1) % kPyramidSlots);
    const int fit_slot = static_cast<int>(slot(frame));
    ModelFitLaunch fit{};
    fit.field = field_.as<int32_t>();
    fit.sad = sad_.as<float>();
    fit.has_contrast = true;
    fit.means_offset = conf_stride_;
    fit.older_to_newer = true;
    fit.width = w;
    fit.height = h;
    fit.blksize = mode_.blksize;
    fit.step = mode_.blksize - mode_.overlap;
    fit.models = models_.as<float>();
    fit.slot = fit_slot;
    fit.scratch = scratch_.as<float>();
    // producer.rs:360-369: the deep match fitted from scratch, its prediction, the mode's match around
    // it, and the refit from the first fit.
    if (auto f = match(true, older, newer, s)) return f;
    fit.prior = -1;
    if ((e = launch_model_fit(fit, s)) != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("camera model fit", e)};
    const uint32_t gap = static_cast<uint32_t>(fit_slot);
    if ((e = launch_compose_inline(models_.as<float>(), &gap, predictions_.as<float>(), 1, 1, 0, s)) != cudaSuccess)
        return Failure{AVD_ERR_GPU, cuda_message("camera model prediction", e)};
    if (auto f = match(false, older, newer, s)) return f;
    fit.prior = fit_slot;
    if ((e = launch_model_fit(fit, s)) != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("camera model refit", e)};
    return std::nullopt;
}

std::optional<Failure> PairModels::compose_window(const uint32_t* frames, int count, int centre, float* out,
                                                  cudaStream_t s) const {
    // global/compose.rs:18-64 (`compose_gaps`): each neighbour's pairs from the centre outward, a pair
    // that does not step exactly one stream frame (an edge duplicate) composing as no motion.
    const int neighbours = count - 1, steps = neighbours;
    std::vector<uint32_t> gaps(static_cast<size_t>(neighbours) * steps, kNoPair);
    int row = 0;
    for (int p = 0; p < count; ++p) {
        if (p == centre) continue;
        const int distance = std::abs(p - centre);
        for (int step = 0; step < distance; ++step) {
            const int older = p < centre ? centre - step - 1 : centre + step;
            const bool one_step = frames[older + 1] == frames[older] + 1;
            gaps[static_cast<size_t>(row) * steps + step] = one_step ? slot(frames[older + 1]) : kNoPair;
        }
        ++row;
    }
    cudaError_t e = launch_compose_inline(models_.as<float>(), gaps.data(), out, neighbours, steps, centre, s);
    if (e != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("window prediction", e)};
    return std::nullopt;
}

std::optional<Failure> PairModels::compose_pair(uint32_t older, uint32_t newer, float* older_to_newer,
                                                float* newer_to_older, cudaStream_t s) const {
    const uint32_t gap = newer == older + 1 ? slot(newer) : kNoPair;
    cudaError_t e = cudaSuccess;
    if (older_to_newer) e = launch_compose_inline(models_.as<float>(), &gap, older_to_newer, 1, 1, 0, s);
    if (e == cudaSuccess) e = launch_compose_inline(models_.as<float>(), &gap, newer_to_older, 1, 1, 1, s);
    if (e != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("pair prediction", e)};
    return std::nullopt;
}

}  // namespace avd
