// NL4D pass over one plane group: the collaborative denoiser of av-denoise-core/src/nl4d with its
// NLMeans-HQ front end, for a pinned sigma or (luma without the noise map) the automatic estimate.
//
//   engine       <- nl4d/engine.rs:208-410 (push, push_context, emit_into, finish, reset, pending
//                   regions, the lazily queued tail)
//   denoiser     <- nl4d/denoiser.rs:363-600, 772-816 (head passes at a scene start, one middle pass
//                   per push, tail passes at the end, accumulator regions cleared and normalised)
//   pass         <- nl4d/collab_pass.rs:45-250 (regions zeroed, then one `collab_fused` launch)
//   front ring   <- nlmeans/denoiser/ring.rs with shifted edges (nlmeans/edges.rs: no leading copies,
//                   a short stream padded with its last frame at flush)
//   motion       <- nlmeans/dispatch/motion.rs:173-229 (`match_neighbours`): every neighbour in
//                   logical order against the pass's centre, confidence against the SAD floor
//   derived      <- nlmeans/denoiser/noise.rs:343-382 (`fixed_derived_values`) for the pinned sigma:
//                   sigma per channel, weight scale sigma^2 * g_max^2 (floored), no noise curve, the
//                   motion SAD floor sad_noise_floor(blksize, sigma)
//
// Device layout: the f32 frame ring (slots x pixels x channels, interleaved), its luma pyramid,
// the i32 accumulator ring (slots x pixels x channels) and weight ring (slots x pixels), two f32
// output frames, and one table of neighbour slots for every (ring start, centre) pair so no pass
// uploads anything. Every launch is queued on the caller's stream; nothing synchronises the host.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <deque>
#include <string>
#include <vector>

#include "avd_internal.h"
#include "engine_parts.h"
#include "kernels.h"

namespace avd {
namespace {

constexpr int kPatch = 8;
constexpr int kMaxK = 8;
// Derived words of this pass: sigma per channel, then the weight scale, the curve flag and the
// motion search's SAD floor.
constexpr int kSigmaWord = 0, kWeightScaleWord = 2, kCurveValidWord = 3, kSadFloorWord = 4;

int64_t pad8(int64_t n) { return (n + 7) / 8 * 8; }

class Nl4dPass final : public Pass {
   public:
    static std::optional<Failure> create(const AvdNl4dOptions& o, Channels channels, uint32_t width,
                                         uint32_t height, const AvdSampleFormat& in, const AvdSampleFormat& out,
                                         bool colour_frames, std::unique_ptr<Pass>* result,
                                         bool guides_only = false) {
        // nl4d/denoiser.rs:228-233: a luma filter pass applies the noise map (the measured luma noise
        // curve); a measured pass over frames with chroma also scales its thresholds by the colour
        // grain gains when it applies the noise map or filters chroma (the engine hands it the
        // block means, engine/planar.rs:176-192).
        const bool noise_map = o.noise_map && channels == Channels::Luma && !guides_only;
        const bool colour_gains = !o.has_sigma && colour_frames && (noise_map || channels == Channels::Chroma);
        const AvdMotionSearch& m = o.motion;
        // motion/search.rs:133-139: Auto resolves to Chained { refine_radius: 2 } at d >= 3.
        const bool chained = m.estimation == AVD_ESTIMATION_CHAINED ||
                             (m.estimation == AVD_ESTIMATION_AUTO && o.temporal_radius >= kChainedRadiusThreshold);
        const uint32_t refine_radius = m.estimation == AVD_ESTIMATION_CHAINED ? m.refine_radius : kDefaultRefineRadius;
        if (width < kPatch || height < kPatch) {
            char msg[200];
            std::snprintf(msg, sizeof(msg),
                          "frame dimensions %ux%u must be at least %dx%d for the collaborative filter's patch grid",
                          width, height, kPatch, kPatch);
            return Failure{AVD_ERR_INVALID_GEOMETRY, msg};
        }
        auto p = std::unique_ptr<Nl4dPass>(new Nl4dPass());
        p->opts_ = o;
        p->channels_ = channels;
        p->width_ = width;
        p->height_ = height;
        p->in_ = in;
        p->out_ = out;
        p->d_ = o.temporal_radius;
        p->held_ = nl4d_held_frames(o, channels);
        p->lambda_ = nl4d_lambda_ht(o, channels);
        p->pool_ratio_ = nl4d_pool_ratio(channels);
        p->accum_scale_ = avd_cross_frame_accum_scale(o.spatial_radius, o.temporal_radius);
        p->step_ = static_cast<int>(m.blksize - m.overlap);
        p->blocks_x_ = std::max<int>((static_cast<int>(width) + p->step_ - 1) / p->step_, 1);
        p->blocks_y_ = std::max<int>((static_cast<int>(height) + p->step_ - 1) / p->step_, 1);
        p->mv_stride_ = static_cast<int>(pad8(2LL * p->blocks_x_ * p->blocks_y_));
        p->conf_stride_ = static_cast<int>(pad8(static_cast<int64_t>(p->blocks_x_) * p->blocks_y_));
        p->thsad_ = avd_thsad(m.blksize, o.thsad_scale);
        p->chained_ = chained;
        p->refine_radius_ = static_cast<int>(refine_radius);
        // motion/context.rs:55-71: the schedule escalates to max_search_escalation.
        p->ceiling_ = m.max_search_escalation > m.search_radius ? static_cast<int>(m.max_search_escalation) : 0;
        p->measures_ = !o.has_sigma;
        p->guides_ = guides_only;
        p->noise_map_ = noise_map;
        p->colour_gains_ = colour_gains;
        if (auto f = p->allocate()) return f;
        *result = std::move(p);
        return std::nullopt;
    }

    // nl4d/engine.rs:287-308.
    std::optional<Failure> push(const AvdPlane* planes, size_t* ready) override {
        if (poisoned_) return status(AVD_ERR_NEEDS_RESET);
        if (!pending_.empty() || tail_remaining_ > 0) return status(AVD_ERR_OUTPUTS_PENDING);
        if (auto f = check_planes(planes, in_)) return f;
        cudaEvent_t start{};
        const bool timed = timer_.begin(stream, &start);
        if (auto f = guard(push_planes(planes))) return f;
        pushed_ = true;
        std::optional<uint32_t> region;
        if (auto f = guard(submit_passes(&region))) return f;
        if (timed) timer_.end(stream, start);
        if (region) pending_.push_back(*region);
        pushes_ += 1;
        *ready = pending_.size();
        return std::nullopt;
    }

    // nl4d/engine.rs:310-327.
    std::optional<Failure> push_context(const AvdPlane* planes) override {
        if (poisoned_) return status(AVD_ERR_NEEDS_RESET);
        if (!pending_.empty() || tail_remaining_ > 0) return status(AVD_ERR_OUTPUTS_PENDING);
        if (auto f = check_planes(planes, in_)) return f;
        if (pushed_) return status(AVD_ERR_CONTEXT_AFTER_PUSH);
        if (pushes_ == 0) continuation_ = true;
        if (auto f = guard(push_planes(planes))) return f;
        pushes_ += 1;
        return std::nullopt;
    }

    // nl4d/engine.rs:329-366.
    std::optional<Failure> emit_into(const AvdPlane* planes) override {
        if (poisoned_) return status(AVD_ERR_NEEDS_RESET);
        if (auto f = check_planes(planes, out_)) return f;
        if (pending_.empty() && tail_remaining_ > 0) {
            if (auto f = guard(queue_tail_regions())) return f;
        }
        if (pending_.empty()) return status(AVD_ERR_NOTHING_TO_EMIT);
        const uint32_t slot = pending_.front();
        pending_.pop_front();
        emitted_ = slot_frames_[slot];
        int out_slot = 0;
        if (auto f = guard(normalise_region(slot, &out_slot))) return f;
        if (auto f = guard(write_out(out_slot, planes))) return f;
        if (tail_remaining_ > 0) {
            tail_remaining_ -= 1;
            if (tail_remaining_ == 0) restart_stream();
        }
        return std::nullopt;
    }

    // nl4d/engine.rs:368-381 with nl4d/denoiser.rs:496-545 (`finish_count`): the regions the held
    // frames' passes complete, then the tail's.
    std::optional<Failure> finish(size_t* tail) override {
        if (poisoned_) return status(AVD_ERR_NEEDS_RESET);
        if (!pending_.empty() || tail_remaining_ > 0) return status(AVD_ERR_OUTPUTS_PENDING);
        const size_t count = drained_region_count() + std::min<size_t>(real_pushes_ + held(), 2 * d_);
        if (count == 0)
            restart_stream();
        else
            tail_remaining_ = count;
        *tail = count;
        return std::nullopt;
    }

    void reset() override {
        // Only a reset forgets the shared motion (a stream that ends on its own keeps it for the
        // other pass's last reads).
        if (share_) share_->clear();
        pending_.clear();
        emitted_.reset();
        poisoned_ = false;
        restart_stream();
    }

    size_t max_held_frames() const override { return held_; }
    AvdWindowSpan window_span() const override {
        AvdWindowSpan s{};
        s.behind = held_;
        s.ahead = held_;
        s.edges = 1;  // EdgePadding::Shifted
        return s;
    }
    // nlmeans/edges.rs:26-31: the stream frame the next push takes, held frames included.
    uint32_t next_frame() const override { return static_cast<uint32_t>(real_pushes_ + held()); }
    std::optional<uint32_t> emitted_frame() const override { return emitted_; }
    AvdEngineTiming timing() override { return timer_.collect(); }
    void sample_device_time(uint32_t every) override { timer_.every = every; }
    bool measures_colour() const override { return colour_gains_; }
    // nl4d/denoiser.rs:732-745 (`measure_colour`).
    std::optional<Failure> measure_colour(const ColourMeans* means, bool luma_grid) override {
        if (!colour_gains_ || !measures_) return std::nullopt;
        colour_means_ = means;
        colour_luma_grid_ = luma_grid;
        return noise_.measure_colour(means, luma_grid);
    }
    std::optional<Failure> fail_for_test() override {
        poisoned_ = true;
        return Failure{AVD_ERR_GPU, "forced failure"};
    }
    bool reads_luma() const override { return reads_share_; }

    std::optional<std::pair<PairModelMode, int>> pair_model_mode() const override {
        if (d_ == 0 || reads_share_) return std::nullopt;
        PairModelMode mode;
        mode.blksize = static_cast<int>(opts_.motion.blksize);
        mode.overlap = static_cast<int>(opts_.motion.overlap);
        mode.search_radius = static_cast<int>(opts_.motion.search_radius);
        mode.ceiling = ceiling_;
        mode.levels = static_cast<int>(opts_.motion.pyramid_levels);
        return std::make_pair(mode, static_cast<int>(d_));
    }
    // nl4d/denoiser.rs:463-466 with nlmeans/denoiser/seeds.rs:162-208.
    std::optional<Failure> attach_models(const PairModels* models) override {
        if (d_ == 0 || reads_share_) return std::nullopt;
        models_ = models;
        cudaError_t e = pred_window_.alloc(2 * d_ * kAffineWords * sizeof(float));
        if (e == cudaSuccess) e = pred_pair_.alloc(2 * kAffineWords * sizeof(float));
        if (e != cudaSuccess) return gpu_failure("prediction buffers", e);
        if (measures_)
            if (auto f = noise_.attach_models(models)) return f;
        return std::nullopt;
    }

   private:
    Nl4dPass() = default;

    static Failure status(AvdStatus s) { return Failure{s, avd_status_message(s)}; }
    static Failure gpu_failure(const char* what, cudaError_t e) { return Failure{AVD_ERR_GPU, cuda_message(what, e)}; }
    std::optional<Failure> guard(std::optional<Failure> f) {
        if (f && f->status == AVD_ERR_GPU) poisoned_ = true;
        return f;
    }

    uint32_t C() const { return static_cast<uint32_t>(channels_); }
    uint32_t tf() const { return 2 * d_ + 1; }
    size_t pixels() const { return static_cast<size_t>(width_) * height_; }
    size_t frame_elems() const { return pixels() * C(); }
    float bias() const { return channels_ == Channels::Chroma ? 0.5f : 0.0f; }
    float* slot_ptr(size_t slot) const { return ring_.as<float>() + slot * frame_elems(); }

    std::optional<Failure> allocate() {
        cudaError_t e;
        const size_t fe = frame_elems(), t = tf();
        const int levels = static_cast<int>(opts_.motion.pyramid_levels);
        if ((e = ring_.alloc(fe * t * sizeof(float))) != cudaSuccess) return gpu_failure("frame ring", e);
        const int64_t pyr = pyramid_floats(static_cast<int>(width_), static_cast<int>(height_), static_cast<int>(t),
                                           levels);
        if ((e = pyramid_.alloc(static_cast<size_t>(pyr) * sizeof(float))) != cudaSuccess)
            return gpu_failure("motion pyramid", e);
        const size_t nbrs = 2 * d_;
        if ((e = mv_.alloc(nbrs * mv_stride_ * sizeof(int32_t))) != cudaSuccess) return gpu_failure("motion field", e);
        if ((e = conf_.alloc(nbrs * conf_stride_ * sizeof(float))) != cudaSuccess) return gpu_failure("confidence", e);
        if (ceiling_) {
            if ((e = esc_state_.alloc(escalation_state_floats(static_cast<int>(nbrs), conf_stride_) * sizeof(float))) !=
                cudaSuccess)
                return gpu_failure("escalation state", e);
            if ((e = tm_changes_.alloc(nbrs * conf_stride_ * sizeof(uint32_t))) != cudaSuccess)
                return gpu_failure("truemotion change flags", e);
        }
        if (truemotion()) {
            // motion/truemotion/stage.rs:14-27: the search's seeds and the field between passes.
            if ((e = tm_seeds_.alloc(nbrs * mv_stride_ * sizeof(int32_t))) != cudaSuccess)
                return gpu_failure("truemotion seeds", e);
            if ((e = tm_field_.alloc(nbrs * mv_stride_ * sizeof(int32_t))) != cudaSuccess)
                return gpu_failure("truemotion field", e);
        }
        if (chained_) {
            // motion/context.rs:110-140: 2d pair slots of two directions, each a padded field.
            if ((e = pair_ring_.alloc(nbrs * 2 * mv_stride_ * sizeof(int32_t))) != cudaSuccess)
                return gpu_failure("pair ring", e);
            if ((e = cudaMemset(pair_ring_.ptr, 0, pair_ring_.bytes)) != cudaSuccess) return gpu_failure("pair ring", e);
        }
        // nl4d/denoiser.rs:257-260: a guide never runs the filter, so its filter buffers are placeholders.
        const size_t filter = guides_ ? 0 : 1;
        if ((e = accum_.alloc(filter * fe * t * sizeof(int32_t))) != cudaSuccess)
            return gpu_failure("accumulator ring", e);
        if ((e = wsum_.alloc(filter * pixels() * t * sizeof(int32_t))) != cudaSuccess)
            return gpu_failure("weight ring", e);
        const size_t refs = static_cast<size_t>((width_ - kPatch + 3) / 4 + 1) * ((height_ - kPatch + 3) / 4 + 1);
        if ((e = group_weight_.alloc(filter * refs * sizeof(float))) != cudaSuccess)
            return gpu_failure("group weights", e);
        const size_t member_words = collab_member_words(static_cast<int>(width_), static_cast<int>(height_));
        if ((e = members_.alloc(filter * member_words * sizeof(uint32_t))) != cudaSuccess)
            return gpu_failure("group members", e);
        for (auto& o : outputs_)
            if ((e = o.alloc(filter * fe * sizeof(float))) != cudaSuccess) return gpu_failure("output slot", e);

        // Fixed tables: derived words, the (unused) noise curve, the white-noise DCT profile
        // (nl4d/denoiser.rs:273-277) and the Kaiser taps.
        float words[8] = {0};
        const float sigma = opts_.sigma;
        words[kSigmaWord] = sigma;
        words[kSigmaWord + 1] = sigma;
        float profile[8], kaiser[8];
        avd_dct_noise_profile(0.0f, profile);
        avd_kaiser_window(opts_.kaiser_beta, kaiser);
        float g_max = 0.0f;
        for (float g : profile) g_max = std::max(g_max, g);
        const float norm = sigma * sigma * g_max * g_max;
        words[kWeightScaleWord] = (std::isfinite(norm) && norm > 1e-12f) ? norm : 1e-12f;
        words[kCurveValidWord] = 0.0f;
        words[kSadFloorWord] = avd_sad_noise_floor(opts_.motion.blksize, sigma);
        std::vector<float> tables(8 + 16 + 8 + 8, 0.0f);
        std::copy(words, words + 8, tables.begin());
        std::copy(profile, profile + 8, tables.begin() + 24);
        std::copy(kaiser, kaiser + 8, tables.begin() + 32);
        if ((e = tables_.alloc(tables.size() * sizeof(float))) != cudaSuccess) return gpu_failure("tables", e);
        if ((e = cudaMemcpy(tables_.ptr, tables.data(), tables.size() * sizeof(float), cudaMemcpyHostToDevice)) !=
            cudaSuccess)
            return gpu_failure("tables upload", e);

        // Neighbour slots of every (ring start, centre): logical order with the centre skipped.
        std::vector<uint32_t> slot_tables(static_cast<size_t>(t) * t * nbrs);
        for (uint32_t start = 0; start < t; ++start)
            for (uint32_t centre = 0; centre < t; ++centre) {
                uint32_t* row = slot_tables.data() + (static_cast<size_t>(start) * t + centre) * nbrs;
                uint32_t n = 0;
                for (uint32_t l = 0; l < t; ++l)
                    if (l != centre) row[n++] = (start + l) % t;
            }
        if ((e = slot_tables_.alloc(slot_tables.size() * sizeof(uint32_t))) != cudaSuccess)
            return gpu_failure("slot tables", e);
        if ((e = cudaMemcpy(slot_tables_.ptr, slot_tables.data(), slot_tables.size() * sizeof(uint32_t),
                            cudaMemcpyHostToDevice)) != cudaSuccess)
            return gpu_failure("slot tables upload", e);
        slot_frames_.assign(t, 0u);
        zeroed_.assign(t, false);
        if (measures_) {
            // nl4d/denoiser.rs:268-284 and nlmeans/denoiser/noise.rs:200-246: the front's fold
            // coefficients (its own NLMeans defaults, strength 1.2 and patch radius 4, at a sigma of
            // 1), the consumer's DCT gain and the motion SAD floor per unit sigma.
            NoiseFrontConfig cfg;
            cfg.width = width_;
            cfg.height = height_;
            cfg.channels = C();
            cfg.temporal_radius = d_;
            FoldCoefficients& k = cfg.coefficients;
            k.sigma_scale = opts_.sigma_scale;
            k.curve_applies = noise_map_;
            k.weight_g_max = g_max;
            k.h2_auto = true;
            const float area = 81.0f, unit_strength = 1.2f * 1.0f * 255.0f;
            k.h2_per_inverse_variance = (255.0f * 255.0f) / (3.0f * unit_strength * unit_strength * area);
            k.h2_fixed = (255.0f * 255.0f) / (3.0f * 1.2f * 1.2f * area);
            k.offset_per_variance = 2.0f * (channels_ == Channels::Luma ? 3.0f : 1.5f) * 1.0f * area;
            k.sad_per_sigma = avd_sad_noise_floor(opts_.motion.blksize, 1.0f);
            cfg.motion = true;
            cfg.blksize = static_cast<int>(opts_.motion.blksize);
            cfg.overlap = static_cast<int>(opts_.motion.overlap);
            cfg.search_radius = static_cast<int>(opts_.motion.search_radius);
            cfg.levels = static_cast<int>(opts_.motion.pyramid_levels);
            cfg.thsad = thsad_;
            cfg.ceiling = ceiling_;
            cfg.luma_fields = noise_map_;
            if (auto f = noise_.allocate(cfg)) return f;
        }
        return std::nullopt;
    }

    // The derived words a pass reads (sigma per channel, weight scale, curve flag, motion SAD floor):
    // the measured front's, or the pinned sigma's.
    const float* noise_words() const { return measures_ ? noise_.derived() : tables_.as<float>(); }
    // The luma noise curve's ratios: the measured front's (read only while its derived curve flag is
    // set), or the pinned sigma's zeros.
    const float* noise_curve() const { return measures_ ? noise_.curve_ratios() : tables_.as<float>() + 8; }
    const float* dct_profile() const { return tables_.as<float>() + 24; }
    const float* kaiser_taps() const { return tables_.as<float>() + 32; }

    std::optional<Failure> check_planes(const AvdPlane* planes, const AvdSampleFormat& fmt) const {
        const uint64_t need = plane_bytes(fmt, pixels());
        for (uint32_t i = 0; i < C(); ++i) {
            const AvdPlane& p = planes[i];
            if (p.width != width_ || p.height != height_) {
                char m[160];
                std::snprintf(m, sizeof(m), "plane %u is %ux%u, expected %ux%u", i, p.width, p.height, width_, height_);
                return Failure{AVD_ERR_PLANE_MISMATCH, m};
            }
            if (p.bytes < need) {
                char m[160];
                std::snprintf(m, sizeof(m), "plane %u handle holds %llu bytes, needs %llu", i,
                              (unsigned long long)p.bytes, (unsigned long long)need);
                return Failure{AVD_ERR_PLANE_MISMATCH, m};
            }
            if (p.ptr == 0) return Failure{AVD_ERR_PLANE_MISMATCH, "a plane has a null device pointer"};
        }
        return std::nullopt;
    }

    // ---- front ring (shifted edges) ----------------------------------------------------------

    size_t ring_start() const { return ring_head_ % tf(); }
    uint32_t phys(uint32_t logical) const { return static_cast<uint32_t>((ring_start() + logical) % tf()); }
    bool window_ready() const { return frames_loaded_ >= tf(); }

    // A pass that refines the luma pass's motion matches on one level (seeds.rs:184-208).
    int pyramid_levels() const { return reads_share_ ? 1 : static_cast<int>(opts_.motion.pyramid_levels); }

    std::optional<Failure> build_pyramid(size_t slot) {
        cudaError_t e = launch_pyramid_build(ring_.as<float>(), static_cast<int>(C()), static_cast<int>(width_),
                                             static_cast<int>(height_), static_cast<int>(tf()),
                                             static_cast<int>(slot), pyramid_levels(), pyramid_.as<float>(),
                                             static_cast<int>(slot), stream);
        if (e != cudaSuccess) return gpu_failure("pyramid launch", e);
        return std::nullopt;
    }

    // nlmeans/denoiser/mod.rs:484-512: a measured front reads the frame in the look-ahead and
    // releases the frame pushed 8 pushes earlier into the ring.
    std::optional<Failure> push_planes(const AvdPlane* planes) {
        if (measures_) {
            if (noise_.held() == NoiseFront::kFrames) {
                bool released = false;
                if (auto f = release_held_frame(&released)) return f;
            }
            if (auto f = noise_.before_ingest(stream)) return f;
            if (auto f = ingest_into(planes, noise_.slot(noise_.pushed()))) return f;
            return noise_.read_pushed(stream);
        }
        const size_t slot = ring_head_ % tf();
        if (auto f = ingest_into(planes, slot_ptr(slot))) return f;
        return enter_ring(slot);
    }

    std::optional<Failure> ingest_into(const AvdPlane* planes, float* dst) {
        const void* p0 = reinterpret_cast<const void*>(planes[0].ptr);
        const void* p1 = C() > 1 ? reinterpret_cast<const void*>(planes[1].ptr) : nullptr;
        cudaError_t e = launch_ingest(p0, p1, dst, static_cast<int64_t>(pixels()), static_cast<int>(C()),
                                      plane_format(in_), bias(), stream);
        if (e != cudaSuccess) return gpu_failure("ingest launch", e);
        return std::nullopt;
    }

    // nlmeans/denoiser/stages.rs:15-40: the per-frame stages of a frame entering ring slot `slot`.
    std::optional<Failure> enter_ring(size_t slot) {
        if (auto f = build_pyramid(slot)) return f;
        if (auto f = pair_analyse(slot)) return f;
        slot_frames_[slot] = static_cast<uint32_t>(real_pushes_);
        ring_head_ += 1;
        if (frames_loaded_ < tf()) frames_loaded_ += 1;
        real_pushes_ += 1;
        return std::nullopt;
    }

    size_t held() const { return measures_ ? noise_.held() : 0; }

    // nlmeans/denoiser/lookahead.rs:226-259 (`release_held_frame`).
    std::optional<Failure> release_held_frame(bool* released) {
        *released = false;
        if (!measures_) return std::nullopt;
        const std::optional<size_t> frame = noise_.take_oldest();
        if (!frame) return std::nullopt;
        const size_t slot = ring_head_ % tf();
        cudaError_t e = cudaMemcpyAsync(slot_ptr(slot), noise_.slot(*frame), frame_elems() * sizeof(float),
                                        cudaMemcpyDeviceToDevice, stream);
        if (e != cudaSuccess) return gpu_failure("look-ahead release", e);
        *released = true;
        return enter_ring(slot);
    }

    // nl4d/denoiser.rs:511-538 (`drained_region_count`): the regions the passes of the held frames
    // complete, following the pass count submit_passes keeps.
    size_t drained_region_count() const {
        uint64_t passes = passes_run_;
        size_t regions = 0;
        for (size_t taken = real_pushes_ + 1; taken <= real_pushes_ + held(); ++taken) {
            if (taken < tf()) continue;
            if (passes == 0 && !continuation_) passes += d_;
            passes += 1;
            if (passes > d_) regions += 1;
        }
        return regions;
    }

    // nlmeans/denoiser/ring.rs:128-146 and nlmeans/edges.rs:41-48.
    std::optional<Failure> fill_ring_with_last_frame() {
        while (!window_ready()) {
            const size_t last = (ring_head_ - 1) % tf(), next = ring_head_ % tf();
            cudaError_t e = cudaMemcpyAsync(slot_ptr(next), slot_ptr(last), frame_elems() * sizeof(float),
                                            cudaMemcpyDeviceToDevice, stream);
            if (e != cudaSuccess) return gpu_failure("slot copy", e);
            if (auto f = build_pyramid(next)) return f;
            if (chained_) {
                // nlmeans/denoiser/stages.rs:201-209: a duplicated frame's pair is zero motion.
                int32_t* pair = pair_ring_.as<int32_t>() + (ring_head_ % (2 * d_)) * 2 * mv_stride_;
                if ((e = cudaMemsetAsync(pair, 0, 2 * mv_stride_ * sizeof(int32_t), stream)) != cudaSuccess)
                    return gpu_failure("pair clear", e);
            }
            slot_frames_[next] = slot_frames_[last];
            ring_head_ += 1;
            frames_loaded_ += 1;
        }
        return std::nullopt;
    }

    // nlmeans/denoiser/stages.rs:146-197 with motion/chain.rs:18-96: both directions between the
    // frame just written and the one before it, into pair slot ring_head mod 2d (before the head
    // advances). A stream's first frame has no older partner.
    std::optional<Failure> pair_analyse(size_t newer) {
        if (!chained_ || ring_head_ == 0) return std::nullopt;
        const size_t older = (newer + tf() - 1) % tf();
        int32_t* pair = pair_ring_.as<int32_t>() + (ring_head_ % (2 * d_)) * 2 * mv_stride_;
        // stages.rs:15-22, 172-180 with seeds.rs:104-134: both directions' predictions between the
        // older slot's frame and the frame entering now (its slot records it after this search), the
        // searches scored against zeroed noise words.
        if (models_)
            if (auto f = models_->compose_pair(slot_frames_[older], static_cast<uint32_t>(real_pushes_), pred_pair_.as<float>(),
                                               pred_pair_.as<float>() + kAffineWords, stream))
                return f;
        for (int dir = 0; dir < 2; ++dir) {
            MotionLaunch m = search_launch();
            m.neighbour_slots = nullptr;
            m.inline_slots[0] = static_cast<uint32_t>(dir == 0 ? newer : older);
            m.centre_slot = static_cast<int>(dir == 0 ? older : newer);
            m.neighbours = 1;
            m.mv_field = pair + dir * mv_stride_;
            m.confidence = nullptr;
            if (models_) {
                m.predictions = pred_pair_.as<float>() + dir * kAffineWords;
                m.noise = models_->zero_noise();
            }
            // motion/chain.rs:54-62: each direction ends with the stage at the unscaled penalty.
            if (auto f = search_then_truemotion(m, false)) return f;
        }
        return std::nullopt;
    }

    // ---- the truemotion stage (motion/analyse.rs:175-312, truemotion/stage.rs) ----
    bool truemotion() const { return opts_.field_lambda > 0.0f; }

    // The search `m`, then, with the stage on, one truemotion pass over its field with the coarse
    // pass's field as the seed candidates; the pass's field lands back in `m.mv_field`.
    std::optional<Failure> search_then_truemotion(MotionLaunch m, bool reads_floor) {
        const bool coarse = m.levels > 1 && !m.seeded;
        if (truemotion() && coarse) m.keep_seeds = tm_seeds_.as<int32_t>();
        // truemotion/params.rs:9-12, 79-90: two passes after a search that escalates.
        const bool two_passes = m.escalation && m.ceiling > m.search_radius;
        cudaError_t e = launch_motion_search(m, stream);
        if (e != cudaSuccess) return gpu_failure("motion search launch", e);
        if (!truemotion()) return std::nullopt;
        TruemotionLaunch t{};
        t.pyramid = m.pyramid;
        t.slot_pixels = pyramid_slot_pixels(m.width, m.height, 0);
        t.neighbour_slots = m.neighbour_slots;
        for (int i = 0; i < TruemotionLaunch::kMaxInlineSlots; ++i) t.inline_slots[i] = m.inline_slots[i];
        t.mv_in = m.mv_field;
        t.seeds = coarse ? tm_seeds_.as<int32_t>() : nullptr;
        t.mv_out = tm_field_.as<int32_t>();
        t.confidence = m.confidence;
        t.noise = m.noise;
        t.width = m.width;
        t.height = m.height;
        t.centre_slot = m.centre_slot;
        t.neighbours = m.neighbours;
        t.blksize = m.blksize;
        t.step = step_;
        t.blocks_x = blocks_x_;
        t.blocks_y = blocks_y_;
        t.mv_stride = mv_stride_;
        t.conf_stride = conf_stride_;
        t.sad_field = kSadFloorWord;
        t.reads_floor = reads_floor ? 1 : 0;
        t.refine_radius = 1;  // truemotion/params.rs:15
        // truemotion/stage.rs:52-62 with params.rs:4-33 (noise weight 1, surcharge 1/8, fade 2 thsad).
        const float lambda = opts_.field_lambda;
        t.lambda_base = lambda * static_cast<float>(m.blksize * m.blksize) * 0.02f;
        t.lambda_noise = lambda * 1.0f;
        t.surcharge = 0.125f;
        t.fade_level = 2.0f * std::max(m.thsad, 0.0f);
        t.predictions = m.predictions;
        t.thsad = m.thsad;
        if (two_passes) {
            // truemotion/stage.rs:82-142: the second pass reads the first's field back into the
            // search's and rescores only the blocks next to one the first changed.
            t.changes_out = tm_changes_.as<uint32_t>();
            if ((e = launch_truemotion(t, stream)) != cudaSuccess) return gpu_failure("truemotion launch", e);
            t.mv_in = tm_field_.as<int32_t>();
            t.mv_out = m.mv_field;
            t.changes_in = tm_changes_.as<uint32_t>();
            t.changes_out = nullptr;
            if ((e = launch_truemotion(t, stream)) != cudaSuccess) return gpu_failure("truemotion launch", e);
            return std::nullopt;
        }
        if ((e = launch_truemotion(t, stream)) != cudaSuccess) return gpu_failure("truemotion launch", e);
        e = cudaMemcpyAsync(m.mv_field, t.mv_out, static_cast<size_t>(m.neighbours) * mv_stride_ * sizeof(int32_t),
                            cudaMemcpyDeviceToDevice, stream);
        if (e != cudaSuccess) return gpu_failure("truemotion field copy", e);
        return std::nullopt;
    }

    MotionLaunch search_launch() const {
        MotionLaunch m{};
        m.pyramid = pyramid_.as<float>();
        m.noise = noise_words();
        m.width = static_cast<int>(width_);
        m.height = static_cast<int>(height_);
        m.frame_count = static_cast<int>(tf());
        m.blksize = static_cast<int>(opts_.motion.blksize);
        m.overlap = static_cast<int>(opts_.motion.overlap);
        m.search_radius = static_cast<int>(opts_.motion.search_radius);
        m.coarse_radius = m.search_radius;
        m.coarse_block_factor = 1;
        m.levels = static_cast<int>(opts_.motion.pyramid_levels);
        m.mv_stride = mv_stride_;
        m.conf_stride = conf_stride_;
        m.sad_floor_word = kSadFloorWord;
        m.thsad = thsad_;
        if (ceiling_) {
            m.escalation = esc_state_.as<float>();
            m.ceiling = ceiling_;
        }
        return m;
    }

    // ---- passes ----------------------------------------------------------------------------

    const uint32_t* slot_table(uint32_t centre) const {
        return slot_tables_.as<uint32_t>() + (ring_start() * tf() + centre) * (2 * d_);
    }

    // nlmeans/denoiser/machinery.rs:45-102 then dispatch/motion.rs:104-229.
    std::optional<Failure> machinery_at(uint32_t centre) {
        // machinery.rs:60-66: the look-ahead has read every frame the window reaches, so the fold
        // around the pass's centre frame runs first and the match scores confidence against it.
        if (measures_)
            if (auto f = noise_.fold(slot_frames_[phys(centre)], stream)) return f;
        if (reads_share_) return refine_luma_motion(centre);
        if (auto f = estimate_motion(centre)) return f;
        return share_window_motion(centre);
    }

    // dispatch/motion.rs:231-253 (`share_window_motion`): the window's fields mapped onto the chroma
    // block grid, into the shared slot of the centre's stream frame.
    std::optional<Failure> share_window_motion(uint32_t centre) {
        if (!writes_share_) return std::nullopt;
        const uint32_t frame = slot_frames_[phys(centre)];
        const int slot = static_cast<int>(frame % static_cast<uint32_t>(share_->slots));
        MapLaunch mp{};
        mp.luma = mv_.as<int32_t>();
        mp.chroma = share_->slot_ptr(slot);
        mp.fields = static_cast<int>(2 * d_);
        mp.luma_bx = blocks_x_;
        mp.luma_by = blocks_y_;
        mp.luma_step = step_;
        mp.luma_blksize = static_cast<int>(opts_.motion.blksize);
        mp.luma_stride = mv_stride_;
        mp.chroma_bx = share_->blocks_x;
        mp.chroma_by = share_->blocks_y;
        mp.chroma_step = share_->step;
        mp.chroma_blksize = share_->blksize;
        mp.chroma_stride = share_->mv_stride;
        mp.shift_x = share_->shift_x;
        mp.shift_y = share_->shift_y;
        cudaError_t e = launch_map_luma_fields(mp, stream);
        if (e != cudaSuccess) return gpu_failure("luma motion map launch", e);
        share_->tags[slot] = frame;
        return std::nullopt;
    }

    // dispatch/motion.rs:255-310 (`refine_luma_motion`): the luma pass's mapped vectors of the centre's
    // stream frame, searched one pixel around on this plane at one level, with confidence.
    std::optional<Failure> refine_luma_motion(uint32_t centre) {
        const uint32_t frame = slot_frames_[phys(centre)];
        const int slot = static_cast<int>(frame % static_cast<uint32_t>(share_->slots));
        if (share_->tags[slot] != static_cast<int64_t>(frame)) {
            char m[120];
            std::snprintf(m, sizeof(m), "the luma pass has not shared the motion of stream frame %u", frame);
            return Failure{AVD_ERR_GPU, m};
        }
        cudaError_t e = cudaMemcpyAsync(mv_.as<int32_t>(), share_->slot_ptr(slot),
                                        2 * d_ * static_cast<size_t>(mv_stride_) * sizeof(int32_t),
                                        cudaMemcpyDeviceToDevice, stream);
        if (e != cudaSuccess) return gpu_failure("mapped motion copy", e);
        MotionLaunch m = search_launch();
        m.neighbour_slots = slot_table(centre);
        m.mv_field = mv_.as<int32_t>();
        m.confidence = conf_.as<float>();
        m.centre_slot = static_cast<int>(phys(centre));
        m.neighbours = static_cast<int>(2 * d_);
        m.search_radius = 1;  // dispatch/motion.rs:44 (MAPPED_REFINE_RADIUS)
        m.coarse_radius = 1;
        m.levels = 1;
        m.seeded = 1;
        m.escalation = nullptr;  // motion/context.rs:95-112: the mapped refine runs a fixed schedule
        m.ceiling = 0;
        if ((e = launch_motion_search(m, stream)) != cudaSuccess) return gpu_failure("mapped refine launch", e);
        return std::nullopt;
    }

   public:
    // engine/spec.rs:350-365 and nlmeans/denoiser/seeds.rs:168-208: the chroma pass reads the luma
    // pass's motion, so it drops its own search (pair ring, truemotion, coarse level).
    static std::optional<Failure> link(Nl4dPass& luma, Nl4dPass& chroma, int shift_x, int shift_y) {
        if (luma.d_ != chroma.d_) return Failure{AVD_ERR_INVALID_OPTIONS, "the luma and chroma windows differ"};
        auto share = std::make_shared<LumaMotionShare>();
        share->slots = static_cast<int>(chroma.tf());
        share->neighbours = static_cast<int>(2 * chroma.d_);
        share->blocks_x = chroma.blocks_x_;
        share->blocks_y = chroma.blocks_y_;
        share->step = chroma.step_;
        share->blksize = static_cast<int>(chroma.opts_.motion.blksize);
        share->mv_stride = chroma.mv_stride_;
        share->shift_x = shift_x;
        share->shift_y = shift_y;
        share->tags.assign(share->slots, -1);
        cudaError_t e = share->fields.alloc(static_cast<size_t>(share->slots) * share->neighbours * share->mv_stride *
                                            sizeof(int32_t));
        if (e != cudaSuccess) return gpu_failure("luma motion share", e);
        luma.share_ = share;
        luma.writes_share_ = true;
        chroma.share_ = share;
        chroma.reads_share_ = true;
        chroma.chained_ = false;
        return std::nullopt;
    }

   private:
    std::optional<Failure> estimate_motion(uint32_t centre) {
        if (chained_) {
            // nlmeans/dispatch/motion.rs:138-171 then analyse.rs:273-316: every neighbour's seed
            // chained from the pair ring, then refined `refine_radius` around it with confidence.
            cudaError_t e = launch_chain_compose(pair_ring_.as<int32_t>(), mv_.as<int32_t>(), mv_stride_,
                                                 static_cast<int>(centre), static_cast<int>(d_),
                                                 static_cast<int>(ring_head_ % (2 * d_)), mv_stride_, 2 * mv_stride_,
                                                 step_, static_cast<int>(width_), static_cast<int>(height_), blocks_x_,
                                                 blocks_y_, stream);
            if (e != cudaSuccess) return gpu_failure("chain compose launch", e);
            MotionLaunch m = search_launch();
            m.neighbour_slots = slot_table(centre);
            m.mv_field = mv_.as<int32_t>();
            m.confidence = conf_.as<float>();
            m.centre_slot = static_cast<int>(phys(centre));
            m.neighbours = static_cast<int>(2 * d_);
            m.search_radius = refine_radius_;
            m.coarse_radius = refine_radius_;
            m.seeded = 1;
            m.esc_reads_floor = 1;  // the window's floor, as the window search reads it
            e = launch_motion_search(m, stream);
            if (e != cudaSuccess) return gpu_failure("seeded refine launch", e);
            return std::nullopt;
        }
        MotionLaunch m{};
        m.pyramid = pyramid_.as<float>();
        m.neighbour_slots = slot_table(centre);
        m.mv_field = mv_.as<int32_t>();
        m.confidence = conf_.as<float>();
        m.noise = noise_words();
        m.width = static_cast<int>(width_);
        m.height = static_cast<int>(height_);
        m.frame_count = static_cast<int>(tf());
        m.centre_slot = static_cast<int>(phys(centre));
        m.neighbours = static_cast<int>(2 * d_);
        m.blksize = static_cast<int>(opts_.motion.blksize);
        m.overlap = static_cast<int>(opts_.motion.overlap);
        m.search_radius = static_cast<int>(opts_.motion.search_radius);
        m.coarse_radius = m.search_radius;
        m.coarse_block_factor = 1;
        m.levels = static_cast<int>(opts_.motion.pyramid_levels);
        m.mv_stride = mv_stride_;
        m.conf_stride = conf_stride_;
        m.sad_floor_word = kSadFloorWord;
        m.thsad = thsad_;
        if (ceiling_) {
            // nlmeans/dispatch/motion.rs:197-201: the window's derived noise is the escalation floor.
            m.escalation = esc_state_.as<float>();
            m.ceiling = ceiling_;
            m.esc_reads_floor = 1;
        }
        if (models_) {
            // dispatch/motion.rs:190-195 with seeds.rs:136-160: every neighbour's prediction for the
            // window's stream frames (the chained seeds already carry the camera's motion).
            uint32_t frames[2 * kMaxTemporalRadius + 1];
            for (uint32_t l = 0; l < tf(); ++l) frames[l] = slot_frames_[phys(l)];
            if (auto f = models_->compose_window(frames, static_cast<int>(tf()), static_cast<int>(centre),
                                                 pred_window_.as<float>(), stream))
                return f;
            m.predictions = pred_window_.as<float>();
        }
        // nlmeans/dispatch/motion.rs:201-206: the window's floor scales the stage's penalty.
        return search_then_truemotion(m, true);
    }

    enum class Clear { WholeRing, NewestRegion, Nothing };

    // nl4d/collab_pass.rs:45-130 and 131-190.
    std::optional<Failure> run_pass(uint32_t centre, Clear clear) {
        if (guides_) {
            // nl4d/collab_pass.rs:50-55: a guide's pass runs only the front's machinery.
            passes_run_ += 1;
            return std::nullopt;
        }
        const uint32_t centre_slot = phys(centre);
        uint32_t c0 = 0, c1 = 0;
        if (clear == Clear::WholeRing) {
            c1 = tf();
        } else if (clear == Clear::NewestRegion) {
            const uint32_t newest = (centre_slot + d_) % tf();
            c0 = newest;
            c1 = zeroed_[newest] ? newest : newest + 1;
        }
        std::fill(zeroed_.begin(), zeroed_.end(), false);
        passes_run_ += 1;
        for (uint32_t s = c0; s < c1; ++s) {
            cudaError_t e = cudaMemsetAsync(accum_.as<int32_t>() + s * frame_elems(), 0, frame_elems() * sizeof(int32_t),
                                            stream);
            if (e == cudaSuccess)
                e = cudaMemsetAsync(wsum_.as<int32_t>() + s * pixels(), 0, pixels() * sizeof(int32_t), stream);
            if (e != cudaSuccess) return gpu_failure("accumulator clear", e);
        }
        CollabLaunch a{};
        a.ring = ring_.as<float>();
        a.width = static_cast<int>(width_);
        a.height = static_cast<int>(height_);
        a.channels = static_cast<int>(C());
        a.centre_slot = static_cast<int>(centre_slot);
        a.frame_elems = static_cast<int64_t>(frame_elems());
        a.mv_field = mv_.as<int32_t>();
        a.confidence = conf_.as<float>();
        a.neighbour_slots = slot_table(centre);
        a.noise = noise_words();
        a.sigma_word = kSigmaWord;
        a.weight_scale_word = kWeightScaleWord;
        a.curve_valid_word = kCurveValidWord;
        a.noise_curve = noise_curve();
        a.dct_profile = dct_profile();
        a.kaiser = kaiser_taps();
        a.accum = accum_.as<int32_t>();
        a.wsum = wsum_.as<int32_t>();
        a.group_weight = group_weight_.as<float>();
        a.members = members_.as<uint32_t>();
        a.c_min = opts_.c_min;
        a.lambda_ht = lambda_;
        a.accum_scale = accum_scale_;
        a.pool_ratio = pool_ratio_;
        a.pooled = opts_.pooled_threshold ? 1 : 0;
        a.wiener = opts_.wiener ? 1 : 0;
        a.radius = static_cast<int>(d_);
        a.refine = static_cast<int>(opts_.refine);
        a.spatial_radius = static_cast<int>(opts_.spatial_radius);
        a.k_max = kMaxK;
        a.mv_stride = mv_stride_;
        a.conf_stride = conf_stride_;
        a.blk_step = step_;
        a.blksize = static_cast<int>(opts_.motion.blksize);
        a.blocks_x = blocks_x_;
        a.blocks_y = blocks_y_;
        if (colour_means_) {
            // collab_pass.rs:71-75 (`colour_gain_inputs`): the gains of the window's fit and the
            // block means of the pass's centre frame, on this plane's grid.
            const uint32_t frame = slot_frames_[centre_slot];
            a.colour_means = colour_means_->held(colour_luma_grid_, frame);
            if (!a.colour_means)
                return Failure{AVD_ERR_GPU, "the block colour of stream frame " + std::to_string(frame) + " is not held"};
            a.colour_gains = noise_.colour_gains();
            a.colour_scale = colour_means_->grain_scale();
            a.colour_on = 1;
            a.colour_blocks_x = (static_cast<int>(width_) + 15) / 16;
        }
        cudaEvent_t core{};
        timer_.core_begin(stream, &core);
        cudaError_t e = launch_collab(a, stream);
        timer_.core_end(stream, core);
        if (e != cudaSuccess) return gpu_failure("collab launch", e);
        return std::nullopt;
    }

    // nl4d/denoiser.rs:370-406 (`submit_passes`).
    std::optional<Failure> submit_passes(std::optional<uint32_t>* region) {
        region->reset();
        if (!window_ready()) return std::nullopt;
        const bool opens_scene = passes_run_ == 0 && !continuation_;
        Clear clear = passes_run_ == 0 ? Clear::WholeRing : Clear::NewestRegion;
        if (opens_scene) {
            for (uint32_t centre = 0; centre < d_; ++centre) {
                if (auto f = machinery_at(centre)) return f;
                if (auto f = run_pass(centre, clear)) return f;
                clear = Clear::Nothing;
            }
        }
        if (auto f = machinery_at(d_)) return f;
        if (auto f = run_pass(d_, clear)) return f;
        if (passes_run_ <= d_) return std::nullopt;
        *region = (phys(d_) + tf() - d_) % tf();
        return std::nullopt;
    }

    // nl4d/engine.rs:181-196 (`queue_tail_regions`): the look-ahead drains one region at a time
    // (nl4d/denoiser.rs:478-494, `drain_lookahead`), then the tail passes run.
    std::optional<Failure> queue_tail_regions() {
        for (;;) {
            bool released = false;
            if (auto f = release_held_frame(&released)) return f;
            if (!released) break;
            std::optional<uint32_t> region;
            if (auto f = submit_passes(&region)) return f;
            if (region) {
                pending_.push_back(*region);
                return std::nullopt;
            }
        }
        return finish_passes();
    }

    // nl4d/denoiser.rs:544-596 (`finish_passes`).
    std::optional<Failure> finish_passes() {
        const uint32_t emit = static_cast<uint32_t>(std::min<size_t>(real_pushes_, 2 * d_));
        if (emit == 0) return std::nullopt;
        const bool short_stream = real_pushes_ < tf();
        if (short_stream) {
            if (auto f = fill_ring_with_last_frame()) return f;
        }
        const uint32_t first = short_stream ? 0 : d_ + 1;
        const uint32_t end = short_stream ? emit : 2 * d_ + 1;
        const uint32_t last_real = short_stream ? emit - 1 : 2 * d_;
        Clear clear = (short_stream || passes_run_ == 0) ? Clear::WholeRing : Clear::Nothing;
        for (uint32_t centre = first; centre < end; ++centre) {
            if (auto f = machinery_at(centre)) return f;
            if (auto f = run_pass(centre, clear)) return f;
            clear = Clear::Nothing;
        }
        const size_t owed = tail_remaining_;
        if (emit != owed) {
            char m[120];
            std::snprintf(m, sizeof(m), "the tail completed %u of %zu owed regions", emit, owed);
            return Failure{AVD_ERR_GPU, m};
        }
        for (uint32_t logical = last_real + 1 - emit; logical <= last_real; ++logical) pending_.push_back(phys(logical));
        return std::nullopt;
    }

    // nl4d/denoiser.rs:772-816 and collab/kernels/aggregate.rs:240-290.
    std::optional<Failure> normalise_region(uint32_t slot, int* out_slot) {
        *out_slot = next_output_slot_;
        next_output_slot_ = (next_output_slot_ + 1) % 2;
        if (guides_) {
            zeroed_[slot] = true;
            return std::nullopt;
        }
        cudaError_t e = launch_collab_normalise(accum_.as<int32_t>() + slot * frame_elems(),
                                                wsum_.as<int32_t>() + slot * pixels(), outputs_[*out_slot].as<float>(),
                                                static_cast<int64_t>(pixels()), static_cast<int>(C()), stream);
        if (e != cudaSuccess) return gpu_failure("normalise launch", e);
        zeroed_[slot] = true;
        return std::nullopt;
    }

    std::optional<Failure> write_out(int slot, const AvdPlane* planes) {
        if (guides_) return std::nullopt;  // nl4d/engine.rs:318-321: a guide writes nothing
        void* p0 = reinterpret_cast<void*>(planes[0].ptr);
        void* p1 = C() > 1 ? reinterpret_cast<void*>(planes[1].ptr) : nullptr;
        cudaError_t e = launch_egress(outputs_[slot].as<float>(), p0, p1, static_cast<int64_t>(pixels()),
                                      static_cast<int>(C()), plane_format(out_), bias(), stream);
        if (e != cudaSuccess) return gpu_failure("egress launch", e);
        return std::nullopt;
    }

    // nl4d/engine.rs:166-171 with nl4d/denoiser.rs:598-610.
    void restart_stream() {
        ring_head_ = 0;
        frames_loaded_ = 0;
        real_pushes_ = 0;
        passes_run_ = 0;
        next_output_slot_ = 0;
        continuation_ = false;
        std::fill(zeroed_.begin(), zeroed_.end(), false);
        tail_remaining_ = 0;
        pushes_ = 0;
        pushed_ = false;
        if (measures_) noise_.reset();
    }

    AvdNl4dOptions opts_{};
    Channels channels_ = Channels::Luma;
    uint32_t width_ = 0, height_ = 0, d_ = 1;
    AvdSampleFormat in_{}, out_{};
    size_t held_ = 0;
    float lambda_ = 0.0f, pool_ratio_ = 0.0f, accum_scale_ = 0.0f, thsad_ = 0.0f;
    int step_ = 8, blocks_x_ = 1, blocks_y_ = 1, mv_stride_ = 2, conf_stride_ = 1;

    DeviceBuffer ring_, pyramid_, mv_, conf_, accum_, wsum_, group_weight_, members_, tables_, slot_tables_;
    DeviceBuffer pair_ring_;
    DeviceBuffer tm_seeds_, tm_field_;  // the truemotion stage's seeds and output field
    std::shared_ptr<LumaMotionShare> share_;
    bool writes_share_ = false, reads_share_ = false;
    bool guides_ = false;  // a chroma-only engine's luma pass: motion only (engine/spec.rs:220-236)
    bool chained_ = false;
    const PairModels* models_ = nullptr;  // the camera models the searches start from, or none
    DeviceBuffer pred_window_, pred_pair_;  // window predictions (2d x 6), pair predictions (2 x 6)
    int refine_radius_ = 2;
    int ceiling_ = 0;                   // the escalation ceiling; 0 when the search does not escalate
    DeviceBuffer esc_state_, tm_changes_;  // escalation state, truemotion change flags
    bool measures_ = false;
    NoiseFront noise_;
    DeviceBuffer outputs_[2];

    size_t ring_head_ = 0, frames_loaded_ = 0, real_pushes_ = 0;
    std::vector<uint32_t> slot_frames_;
    uint64_t passes_run_ = 0;
    bool continuation_ = false;
    std::vector<bool> zeroed_;
    int next_output_slot_ = 0;

    std::deque<uint32_t> pending_;
    size_t tail_remaining_ = 0, pushes_ = 0;
    bool pushed_ = false, poisoned_ = false;
    bool noise_map_ = false;  // the filter scales the luma threshold by the measured noise curve
    bool colour_gains_ = false;  // the filter scales its thresholds by the measured colour grain gains
    const ColourMeans* colour_means_ = nullptr;
    bool colour_luma_grid_ = true;
    std::optional<uint32_t> emitted_;
    DeviceTimer timer_;
};

}  // namespace

std::optional<Failure> create_nl4d_pass(const AvdNl4dOptions& options, Channels channels, uint32_t width,
                                        uint32_t height, const AvdSampleFormat& in, const AvdSampleFormat& out,
                                        bool colour_frames, std::unique_ptr<Pass>* result, bool guides_only) {
    return Nl4dPass::create(options, channels, width, height, in, out, colour_frames, result, guides_only);
}

std::optional<Failure> link_nl4d_luma_motion(Pass* luma, Pass* chroma, int shift_x, int shift_y) {
    auto* l = dynamic_cast<Nl4dPass*>(luma);
    auto* c = dynamic_cast<Nl4dPass*>(chroma);
    if (!l || !c) return std::nullopt;
    return Nl4dPass::link(*l, *c, shift_x, shift_y);
}

}  // namespace avd
