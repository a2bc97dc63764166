// The noise look-ahead of a front that measures the noise (av-denoise-core/src/nlmeans/denoiser/
// lookahead.rs with the measured state of noise/state.rs, noise/slot.rs, noise/history.rs and
// noise/fold.rs), shared by the NLMeans-HQ and NL4D passes.
//
// A pushed frame is ingested into one of 8 look-ahead slots and read there: its Immerkaer words and
// totals, its temporal records against the frame before it (along the motion between the two when
// the front follows motion) and its reading, recorded in history slot frame % (17 + d). The frame
// enters the pass's ring 8 pushes later, so every window a pass folds is recorded by then. Before
// each pass the window around the pass's centre frame is folded into the derived words and, for
// NLMeans, the offset tables. The reads run on the front's own high-priority stream, ordered after
// the ingest by an event, so they overlap the pass's work; the fold and the next ingest into a
// look-ahead slot wait for them on the pass's stream.

#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "avd_internal.h"
#include "engine_parts.h"
#include "kernels.h"

namespace avd {

namespace {
constexpr int kReadingWords = 30;       // noise/reading.rs:33
constexpr int kNoiseWindowRadius = 8;   // noise/history.rs:10
constexpr int kOlderToNewer = 0, kNewerToOlder = 1;  // lookahead.rs:43-46

int64_t pad8(int64_t n) { return (n + 7) / 8 * 8; }
}  // namespace

NoiseFront::~NoiseFront() {
    if (side_) cudaStreamSynchronize(side_);
    if (ingested_) cudaEventDestroy(ingested_);
    if (read_done_) cudaEventDestroy(read_done_);
    if (snapshot_) cudaEventDestroy(snapshot_);
    for (cudaEvent_t ev : frame_read_) cudaEventDestroy(ev);
    if (side_) cudaStreamDestroy(side_);
}

std::optional<Failure> NoiseFront::allocate(const NoiseFrontConfig& cfg) {
    cfg_ = cfg;
    const int w = static_cast<int>(cfg.width), h = static_cast<int>(cfg.height);
    const int c = static_cast<int>(cfg.channels);
    const size_t fe = static_cast<size_t>(cfg.width) * cfg.height * cfg.channels;
    capacity_ = 2 * kNoiseWindowRadius + 1 + cfg.temporal_radius;  // history.rs:19-22
    const uint32_t side = 2 * cfg.table_radius + 1;
    auto fail = [](const char* what, cudaError_t e) { return Failure{AVD_ERR_GPU, cuda_message(what, e)}; };
    cudaError_t e;
    if ((e = lookahead_.alloc(fe * kFrames * sizeof(float))) != cudaSuccess) return fail("look-ahead ring", e);
    if ((e = partials_.alloc(immerkaer_partials_len(w, h) * sizeof(float))) != cudaSuccess)
        return fail("noise partials", e);
    if (cfg.temporal_radius > 0) {
        if ((e = records_.alloc(noise_records_floats(w, h, c) * sizeof(float))) != cudaSuccess)
            return fail("noise records", e);
        if ((e = scratch_.alloc(noise_scratch_floats(w, h) * sizeof(float))) != cudaSuccess)
            return fail("noise scratch", e);
    }
    if ((e = history_records_.alloc(capacity_ * kReadingWords * sizeof(float))) != cudaSuccess)
        return fail("noise history", e);
    if ((e = history_results_.alloc(capacity_ * 2 * sizeof(float))) != cudaSuccess) return fail("noise history", e);
    if ((e = settings_.alloc(16 * sizeof(float))) != cudaSuccess) return fail("fold settings", e);
    if ((e = state_.alloc(32 * sizeof(float))) != cudaSuccess) return fail("fold state", e);
    if ((e = derived_.alloc(16 * sizeof(float))) != cudaSuccess) return fail("derived words", e);
    if ((e = spatial_.alloc(side * side * sizeof(float))) != cudaSuccess) return fail("offset table", e);
    if ((e = pilot_.alloc(side * side * sizeof(float))) != cudaSuccess) return fail("pilot table", e);
    for (DeviceBuffer* b : {&history_records_, &history_results_, &state_, &derived_, &spatial_, &pilot_})
        if ((e = cudaMemset(b->ptr, 0, b->bytes)) != cudaSuccess) return fail("noise state clear", e);
    // The reads of each pushed frame run on a stream of their own, at the highest priority so their
    // small grids start between the pass's tiles.
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if ((e = cudaStreamCreateWithPriority(&side_, cudaStreamNonBlocking, greatest)) != cudaSuccess)
        return fail("noise stream", e);
    if ((e = cudaEventCreateWithFlags(&ingested_, cudaEventDisableTiming)) != cudaSuccess) return fail("noise event", e);
    if ((e = cudaEventCreateWithFlags(&read_done_, cudaEventDisableTiming)) != cudaSuccess)
        return fail("noise event", e);
    if ((e = cudaEventCreateWithFlags(&snapshot_, cudaEventDisableTiming)) != cudaSuccess)
        return fail("noise event", e);
    frame_read_.assign(capacity_, nullptr);
    for (cudaEvent_t& ev : frame_read_)
        if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return fail("noise event", e);
    if ((e = search_words_.alloc(16 * sizeof(float))) != cudaSuccess) return fail("look-ahead noise words", e);
    if ((e = cudaMemset(search_words_.ptr, 0, search_words_.bytes)) != cudaSuccess)
        return fail("look-ahead noise words", e);
    float words[16];
    noise_fold_words(cfg.width, cfg.height, cfg.coefficients, words);
    if ((e = cudaMemcpy(settings_.ptr, words, sizeof(words), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail("fold settings upload", e);
    if (cfg.motion) {
        // lookahead.rs:70-111: a luma pyramid per held frame and one pair slot of two directions.
        step_ = cfg.blksize - cfg.overlap;
        blocks_x_ = std::max((w + step_ - 1) / step_, 1);
        blocks_y_ = std::max((h + step_ - 1) / step_, 1);
        mv_stride_ = static_cast<int>(pad8(2LL * blocks_x_ * blocks_y_));
        const int64_t pyr = pyramid_floats(w, h, static_cast<int>(kFrames), cfg.levels);
        if ((e = pyramid_.alloc(static_cast<size_t>(pyr) * sizeof(float))) != cudaSuccess)
            return fail("look-ahead pyramid", e);
        if ((e = pair_.alloc(2 * mv_stride_ * sizeof(int32_t))) != cudaSuccess) return fail("look-ahead pair", e);
        if (cfg.ceiling > cfg.search_radius) {
            conf_stride_ = static_cast<int>(pad8(static_cast<int64_t>(blocks_x_) * blocks_y_));
            if ((e = escalation_.alloc(escalation_state_floats(1, conf_stride_) * sizeof(float))) != cudaSuccess)
                return fail("look-ahead escalation state", e);
        }
    }
    return std::nullopt;
}

float* NoiseFront::slot(size_t frame) const {
    const size_t fe = static_cast<size_t>(cfg_.width) * cfg_.height * cfg_.channels;
    return lookahead_.as<float>() + (frame % kFrames) * fe;
}

std::optional<size_t> NoiseFront::take_oldest() {
    if (held() == 0) return std::nullopt;
    return released_++;
}

// One direction of the look-ahead pair between two held frames: `centre`'s blocks matched in
// `neighbour` (lookahead.rs:460-541, with the camera model's pair prediction when the engine fits
// models, and no truemotion stage). A search that
// escalates measures its own floor: the look-ahead's noise words belong to no window (lookahead.rs:
// 509-515).
std::optional<Failure> NoiseFront::attach_models(const PairModels* models) {
    models_ = models;
    if (!models_ || !cfg_.motion) return std::nullopt;
    cudaError_t e = pair_predictions_.alloc(2 * kAffineWords * sizeof(float));
    if (e != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("look-ahead pair predictions", e)};
    return std::nullopt;
}

std::optional<Failure> NoiseFront::search(size_t centre_frame, size_t neighbour_frame, int direction,
                                          cudaStream_t s) {
    MotionLaunch m{};
    m.pyramid = pyramid_.as<float>();
    m.neighbour_slots = nullptr;
    m.inline_slots[0] = static_cast<uint32_t>(neighbour_frame % kFrames);
    m.mv_field = pair_.as<int32_t>() + direction * mv_stride_;
    m.confidence = nullptr;
    m.noise = search_words_.as<float>();
    m.width = static_cast<int>(cfg_.width);
    m.height = static_cast<int>(cfg_.height);
    m.frame_count = static_cast<int>(kFrames);
    m.centre_slot = static_cast<int>(centre_frame % kFrames);
    m.neighbours = 1;
    m.blksize = cfg_.blksize;
    m.overlap = cfg_.overlap;
    m.search_radius = cfg_.search_radius;
    m.coarse_radius = cfg_.search_radius;
    m.coarse_block_factor = 1;
    m.levels = cfg_.levels;
    m.mv_stride = mv_stride_;
    m.conf_stride = 1;
    m.sad_floor_word = 4;
    m.thsad = cfg_.thsad;
    if (escalation_.ptr) {
        m.escalation = escalation_.as<float>();
        m.ceiling = cfg_.ceiling;
        m.conf_stride = conf_stride_;
        m.esc_reads_floor = 0;
    }
    if (models_) {
        // lookahead.rs:500-541: with the camera models each direction also searches around its pair
        // prediction, scored against zeroed noise words.
        m.predictions = pair_predictions_.as<float>() + direction * kAffineWords;
        m.noise = models_->zero_noise();
    }
    cudaError_t e = launch_motion_search(m, s);
    if (e != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("look-ahead search launch", e)};
    return std::nullopt;
}

// The records of held frame `frame` against `prev`, along the pair's `direction` with motion, then
// its reading into its history slot (noise/slot.rs:32-137, 158-175). Words 0-1 of the slot already
// hold the frame's Immerkaer lower quartiles.
std::optional<Failure> NoiseFront::read_against(size_t frame, std::optional<size_t> prev, int direction,
                                                cudaStream_t s) {
    const int w = static_cast<int>(cfg_.width), h = static_cast<int>(cfg_.height);
    const int c = static_cast<int>(cfg_.channels);
    float* reading = history_records_.as<float>() + (frame % capacity_) * kReadingWords;
    const float* records = nullptr;
    cudaError_t e;
    if (cfg_.temporal_radius > 0) {
        const float* p = prev ? slot(*prev) : nullptr;
        const int32_t* field = (cfg_.motion && prev) ? pair_.as<int32_t>() + direction * mv_stride_ : nullptr;
        e = launch_temporal_stats(slot(frame), p, c, w, h, field, blocks_x_, blocks_y_, step_, cfg_.luma_fields,
                                  records_.as<float>(), s);
        if (e != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("temporal noise stats launch", e)};
        records = records_.as<float>();
    }
    const uint32_t blocks = ((cfg_.width + 15) / 16) * ((cfg_.height + 15) / 16);
    e = launch_noise_reading(records, c, w, h, scratch_.as<float>(), min_static_blocks(blocks),
                             cfg_.luma_fields && cfg_.temporal_radius > 0, reading, s);
    if (e != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("noise reading launch", e)};
    if (colour_ && records) {
        // noise/colour.rs:765-790 (`queue_colour_cells`): the reading's blocks pooled into the
        // frame's cell sums, replacing any earlier read of the same frame.
        const float* means = colour_->held(colour_luma_, static_cast<uint32_t>(frame));
        if (!means)
            return Failure{AVD_ERR_GPU, "the block colour of stream frame " + std::to_string(frame) + " is not held"};
        e = launch_colour_accumulate(records, means, w, h, c, colour_luma_, colour_->grain_scale(),
                                     colour_cells_.as<int32_t>() + (frame % capacity_) * colour_words_, s);
        if (e != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("colour cells launch", e)};
    }
    return std::nullopt;
}

std::optional<Failure> NoiseFront::measure_colour(const ColourMeans* means, bool luma_grid) {
    if (cfg_.temporal_radius == 0) return std::nullopt;  // colour.rs:737-745: no temporal stats, no cells
    colour_ = means;
    colour_luma_ = luma_grid;
    const int planes = static_cast<int>(cfg_.channels);
    colour_words_ = colour_records(planes, luma_grid) * kColourCellWords;
    auto fail = [](const char* what, cudaError_t e) { return Failure{AVD_ERR_GPU, cuda_message(what, e)}; };
    cudaError_t e;
    if ((e = colour_cells_.alloc(capacity_ * colour_words_ * sizeof(int32_t))) != cudaSuccess ||
        (e = colour_window_.alloc(colour_words_ * sizeof(float))) != cudaSuccess ||
        (e = colour_scratch_.alloc(colour_fit_scratch_floats(planes) * sizeof(float))) != cudaSuccess ||
        (e = colour_table_.alloc(static_cast<size_t>(planes) * kColourCells * sizeof(float))) != cudaSuccess ||
        (e = colour_gains_.alloc(static_cast<size_t>(planes) * kColourCells * sizeof(float))) != cudaSuccess)
        return fail("colour cells", e);
    for (DeviceBuffer* b : {&colour_cells_, &colour_gains_})
        if ((e = cudaMemset(b->ptr, 0, b->bytes)) != cudaSuccess) return fail("colour cells clear", e);
    return std::nullopt;
}

std::optional<Failure> NoiseFront::before_ingest(cudaStream_t main) {
    if (!reads_queued_) return std::nullopt;
    cudaError_t e = cudaStreamWaitEvent(main, read_done_, 0);
    if (e != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("noise read wait", e)};
    return std::nullopt;
}

// lookahead.rs:182-216 and 283-458: the new frame's pyramid and pair search (with motion), then its
// noise read against the frame before it, and, at the stream's second frame, the first frame read
// again along the motion to it.
std::optional<Failure> NoiseFront::read_pushed(cudaStream_t main) {
    cudaError_t ev = cudaEventRecord(ingested_, main);
    if (ev == cudaSuccess) ev = cudaStreamWaitEvent(side_, ingested_, 0);
    // The searches read the derived words of the folds queued before this push.
    if (ev == cudaSuccess)
        ev = cudaMemcpyAsync(search_words_.ptr, derived_.ptr, search_words_.bytes, cudaMemcpyDeviceToDevice, side_);
    if (ev == cudaSuccess) ev = cudaEventRecord(snapshot_, side_);
    if (ev != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("noise read order", ev)};
    snapshot_pending_ = true;
    const cudaStream_t s = side_;
    const size_t frame = pushed_;
    const int w = static_cast<int>(cfg_.width), h = static_cast<int>(cfg_.height);
    const int c = static_cast<int>(cfg_.channels);
    const std::optional<size_t> prev = frame > 0 ? std::optional<size_t>(frame - 1) : std::nullopt;
    if (cfg_.motion) {
        cudaError_t e = launch_pyramid_build(lookahead_.as<float>(), c, w, h, static_cast<int>(kFrames),
                                             static_cast<int>(frame % kFrames), cfg_.levels, pyramid_.as<float>(),
                                             static_cast<int>(frame % kFrames), s);
        if (e != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("look-ahead pyramid launch", e)};
        if (prev) {
            if (models_)
                if (auto f = models_->compose_pair(static_cast<uint32_t>(*prev), static_cast<uint32_t>(frame),
                                                   frame == 1 ? pair_predictions_.as<float>() : nullptr,
                                                   pair_predictions_.as<float>() + kAffineWords, s))
                    return f;
            if (auto f = search(frame, *prev, kNewerToOlder, s)) return f;
            if (frame == 1)
                if (auto f = search(*prev, frame, kOlderToNewer, s)) return f;
        }
    }
    const size_t hs = frame % capacity_;
    cudaError_t e = launch_immerkaer(slot(frame), c, w, h, immerkaer_sigma_scale(), partials_.as<float>(),
                                     history_results_.as<float>() + hs * 2,
                                     history_records_.as<float>() + hs * kReadingWords, s);
    if (e != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("noise estimate launch", e)};
    if (auto f = read_against(frame, prev, kNewerToOlder, s)) return f;
    if (cfg_.motion && frame == 1)
        if (auto f = read_against(0, std::optional<size_t>(1), kOlderToNewer, s)) return f;
    if ((e = cudaEventRecord(read_done_, s)) != cudaSuccess ||
        (e = cudaEventRecord(frame_read_[frame % capacity_], s)) != cudaSuccess)
        return Failure{AVD_ERR_GPU, cuda_message("noise read", e)};
    reads_queued_ = true;
    pushed_ += 1;
    recorded_ = std::max(recorded_, frame + 1);
    return std::nullopt;
}

// nlmeans/denoiser/noise.rs:171-185 (`update_noise_estimate`).
std::optional<Failure> NoiseFront::fold(uint32_t centre, cudaStream_t s) {
    const int64_t newest = static_cast<int64_t>(recorded_) - 1;
    const int first = static_cast<int>(std::max<int64_t>(static_cast<int64_t>(centre) - kNoiseWindowRadius, 0));
    const int last = static_cast<int>(std::min<int64_t>(static_cast<int64_t>(centre) + kNoiseWindowRadius, newest));
    // The window's readings (the reads of its newest frame and every earlier one: the reads run in
    // order on the side stream, and a window reaching frame 1 includes frame 0 read again) have
    // landed, and the newest reads' searches have taken their copy of the derived words this fold
    // overwrites. Frames newer than the window keep reading meanwhile: their history slots lie
    // outside it, as the history holds 17 + d slots.
    cudaError_t e = cudaSuccess;
    if (snapshot_pending_) e = cudaStreamWaitEvent(s, snapshot_, 0);
    if (e == cudaSuccess && last >= 0) e = cudaStreamWaitEvent(s, frame_read_[last % capacity_], 0);
    if (e != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("noise fold wait", e)};
    e = launch_noise_fold(history_records_.as<float>(), history_results_.as<float>(),
                                      static_cast<int>(capacity_), first, last, settings_.as<float>(),
                                      static_cast<int>(cfg_.channels), static_cast<int>(cfg_.table_radius),
                                      state_.as<float>(), derived_.as<float>(), spatial_.as<float>(),
                                      pilot_.as<float>(), s);
    if (e != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("noise fold launch", e)};
    if (colour_) {
        // noise/colour.rs:793-808 (`queue_colour_window`): the window's cell sums, then the grain
        // model fitted from them against the curve and derived words the fold just wrote.
        e = launch_colour_window(colour_cells_.as<int32_t>(), static_cast<int>(capacity_), first, last,
                                 static_cast<int>(colour_words_), colour_window_.as<float>(), s);
        if (e != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("colour window launch", e)};
        const int planes = static_cast<int>(cfg_.channels);
        ColourFitLaunch a{};
        a.window = colour_window_.as<float>();
        a.planes = planes;
        a.luma = colour_luma_;
        a.curve = curve_ratios();
        a.derived = derived_.as<float>();
        a.levels = colour_scratch_.as<float>();
        a.ceilings = a.levels + 2 * planes * kColourCells;
        a.fit_cells = a.ceilings + planes * kColourCells;
        a.fit_planes = a.fit_cells + 5 * planes * kColourCells;
        a.bases = a.fit_planes + planes * kColourFitPlaneWords;
        a.table = colour_table_.as<float>();
        a.gains = colour_gains_.as<float>();
        if ((e = launch_colour_fit(a, s)) != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("colour fit launch", e)};
    }
    return std::nullopt;
}

void NoiseFront::reset() {
    pushed_ = 0;
    released_ = 0;
    recorded_ = 0;
}

}  // namespace avd
