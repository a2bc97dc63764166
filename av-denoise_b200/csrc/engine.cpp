// The engine behind the C ABI: a planar engine (luma pass, chroma pass, passthrough ring) over
// per-plane-group passes, mirroring av-denoise-core's engine layer:
//   - PlanarEngine  <- engine/planar.rs:104-580
//   - NlmPass       <- nlmeans/engine.rs:29-318 with the NlmDenoiser ring of
//                      nlmeans/denoiser/{mod.rs,ring.rs,stages.rs}
// Host state (ring head, loaded frames, ready slot, tail, poison flag) follows the reference
// step for step; the GPU work is queued on the caller's stream with no host synchronisation on
// the push / emit path.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <optional>
#include <string>
#include <vector>

#include "avd_internal.h"
#include "engine_parts.h"
#include "tune.h"
#include "kernels.h"

namespace avd {

namespace {

// ---------------------------------------------------------------------------------------------
// NLMeans pass: nlmeans/engine.rs:29-318 over the ring of nlmeans/denoiser/mod.rs:40-591.
class NlmPass final : public Pass {
   public:
    // With `guides_only` the pass is a chroma-only engine's luma guide: it runs the noise estimate
    // and the window motion for the chroma pass to read, and no denoise (nlmeans/engine.rs:53-100).
    // With `exact_all` (a deterministic tuning) every sample of the denoise pass and of the NLM
    // pilot is computed by the exact kernel in the FP32 mirror's operation order.
    static std::optional<Failure> create(const AvdNlmeansAlgorithm& alg, Channels channels, uint32_t width,
                                         uint32_t height, const AvdSampleFormat& in, const AvdSampleFormat& out,
                                         std::unique_ptr<Pass>* result, bool guides_only = false,
                                         bool exact_all = false, const TuneOptions& tune = TuneOptions{}) {
        auto pass = std::unique_ptr<NlmPass>(new NlmPass());
        pass->guides_ = guides_only;
        pass->exact_all_ = exact_all;
        pass->tune_ = tune;
        pass->params_ = resolve_nlm_params(alg, channels);
        pass->held_ = nlm_held_frames(alg, channels);
        pass->width_ = width;
        pass->height_ = height;
        pass->in_ = in;
        pass->out_ = out;
        const NlmParams& p = pass->params_;
        // nlmeans/denoiser/noise.rs:50-52 (`measures_noise`): HQ without a pinned sigma measures it.
        pass->measures_ = p.hq && !p.hq_params.has_sigma_override;
        // nlmeans/denoiser/mod.rs:242-246: motion compensation needs a temporal window.
        pass->mc_ = p.motion.active && p.temporal_radius > 0;
        if (pass->mc_) {
            const AvdMotionSearch& m = p.motion.search;
            // motion/context.rs:55-71: the schedule escalates to max_search_escalation.
            pass->mc_ceiling_ = m.max_search_escalation > m.search_radius ? static_cast<int>(m.max_search_escalation) : 0;
            // motion/search.rs:133-139: Auto resolves to Chained { refine_radius: 2 } at d >= 3.
            pass->mc_chained_ = m.estimation == AVD_ESTIMATION_CHAINED ||
                                (m.estimation == AVD_ESTIMATION_AUTO && p.temporal_radius >= kChainedRadiusThreshold);
            pass->mc_refine_radius_ =
                static_cast<int>(m.estimation == AVD_ESTIMATION_CHAINED ? m.refine_radius : kDefaultRefineRadius);
        }
        // nlmeans/denoiser/mod.rs:340-370: confidence without motion compensation scores every
        // neighbour block where it stands (blksize 16, step 8, radius 0, one level); with it the
        // window search scores its own blocks.
        const bool confidence = p.hq && p.hq_params.temporal_confidence && p.temporal_radius > 0;
        pass->conf_pass_ = confidence && !pass->mc_;
        pass->mc_conf_ = confidence && pass->mc_;
        if (auto f = pass->allocate()) return f;
        *result = std::move(pass);
        return std::nullopt;
    }

    std::optional<Failure> push(const AvdPlane* planes, size_t* ready) override {
        if (poisoned_) return Failure{AVD_ERR_NEEDS_RESET, avd_status_message(AVD_ERR_NEEDS_RESET)};
        if (ready_slot_ >= 0 || tail_remaining_ > 0)
            return Failure{AVD_ERR_OUTPUTS_PENDING, avd_status_message(AVD_ERR_OUTPUTS_PENDING)};
        if (auto f = check_planes(planes, in_)) return f;
        if (auto f = guard(push_planes(planes))) return f;
        pushed_ = true;
        int slot = -1;
        if (auto f = guard(denoise_submit(&slot))) return f;
        ready_slot_ = slot;
        *ready = slot >= 0 ? 1 : 0;
        return std::nullopt;
    }

    std::optional<Failure> push_context(const AvdPlane* planes) override {
        if (poisoned_) return Failure{AVD_ERR_NEEDS_RESET, avd_status_message(AVD_ERR_NEEDS_RESET)};
        if (ready_slot_ >= 0 || tail_remaining_ > 0)
            return Failure{AVD_ERR_OUTPUTS_PENDING, avd_status_message(AVD_ERR_OUTPUTS_PENDING)};
        if (auto f = check_planes(planes, in_)) return f;
        if (pushed_) return Failure{AVD_ERR_CONTEXT_AFTER_PUSH, avd_status_message(AVD_ERR_CONTEXT_AFTER_PUSH)};
        return guard(push_planes(planes));
    }

    std::optional<Failure> emit_into(const AvdPlane* planes) override {
        if (poisoned_) return Failure{AVD_ERR_NEEDS_RESET, avd_status_message(AVD_ERR_NEEDS_RESET)};
        if (auto f = check_planes(planes, out_)) return f;
        if (ready_slot_ >= 0) {
            int slot = ready_slot_;
            ready_slot_ = -1;
            emitted_ = centre_frame();
            return guard(write_out(slot, planes));
        }
        if (tail_remaining_ == 0) return Failure{AVD_ERR_NOTHING_TO_EMIT, avd_status_message(AVD_ERR_NOTHING_TO_EMIT)};
        int slot = -1;
        if (auto f = guard(next_tail_frame(&slot))) return f;
        emitted_ = centre_frame();
        if (auto f = guard(write_out(slot, planes))) return f;
        tail_remaining_ -= 1;
        if (tail_remaining_ == 0) restart_stream();
        return std::nullopt;
    }

    std::optional<Failure> finish(size_t* tail) override {
        if (poisoned_) return Failure{AVD_ERR_NEEDS_RESET, avd_status_message(AVD_ERR_NEEDS_RESET)};
        if (ready_slot_ >= 0 || tail_remaining_ > 0)
            return Failure{AVD_ERR_OUTPUTS_PENDING, avd_status_message(AVD_ERR_OUTPUTS_PENDING)};
        // nlmeans/denoiser/mod.rs:534-545 (`flush_target`): the look-ahead's frames, then the ring's.
        tail_remaining_ = held() + std::min<size_t>(real_pushes_, params_.temporal_radius);
        if (tail_remaining_ == 0) restart_stream();
        *tail = tail_remaining_;
        return std::nullopt;
    }

    void reset() override {
        // Only a reset forgets the shared motion: a stream that ends on its own restarts the luma pass
        // before the chroma pass has read the last window's motion.
        if (share_) share_->clear();
        ready_slot_ = -1;
        emitted_.reset();
        tail_remaining_ = 0;
        poisoned_ = false;
        restart_stream();
    }

    size_t max_held_frames() const override { return held_; }

    AvdWindowSpan window_span() const override {
        AvdWindowSpan s{};
        s.behind = held_;
        s.ahead = held_;
        s.edges = 0;
        return s;
    }

    // The stream frame the next push takes: frames in the look-ahead count (nlmeans/edges.rs:26-31).
    uint32_t next_frame() const override { return static_cast<uint32_t>(real_pushes_ + held()); }
    std::optional<uint32_t> emitted_frame() const override { return emitted_; }
    AvdEngineTiming timing() override { return timer_.collect(); }
    void sample_device_time(uint32_t every) override { timer_.every = every; }
    std::optional<Failure> fail_for_test() override {
        poisoned_ = true;
        return Failure{AVD_ERR_GPU, "forced failure"};
    }

    bool reads_luma() const override { return reads_share_; }

    std::optional<std::pair<PairModelMode, int>> pair_model_mode() const override {
        if (!mc_ || reads_share_) return std::nullopt;
        const AvdMotionSearch& m = params_.motion.search;
        PairModelMode mode;
        mode.blksize = static_cast<int>(m.blksize);
        mode.overlap = static_cast<int>(m.overlap);
        mode.search_radius = static_cast<int>(m.search_radius);
        mode.ceiling = mc_ceiling_;
        mode.levels = static_cast<int>(m.pyramid_levels);
        return std::make_pair(mode, static_cast<int>(params_.temporal_radius));
    }

    std::optional<Failure> attach_models(const PairModels* models) override {
        if (!mc_ || reads_share_) return std::nullopt;
        models_ = models;
        cudaError_t e = pred_window_.alloc(2 * params_.temporal_radius * kAffineWords * sizeof(float));
        if (e == cudaSuccess) e = pred_pair_.alloc(2 * kAffineWords * sizeof(float));
        if (e != cudaSuccess) return gpu_failure("prediction buffers", e);
        if (measures_)
            if (auto f = noise_.attach_models(models)) return f;
        return std::nullopt;
    }

   private:
    NlmPass() = default;

    static constexpr int kConfBlk = 16;
    static constexpr int kConfStep = 8;
    bool conf_pass_ = false;
    uint32_t conf_bx_ = 0, conf_by_ = 0;
    float thsad_ = 0.0f;
    DeviceBuffer pyramid_, mv_scratch_, conf_;

    size_t pixels() const { return static_cast<size_t>(width_) * height_; }
    size_t frame_elems() const { return pixels() * params_.channel_count(); }
    uint32_t total_frames() const { return params_.total_frames(); }

    std::optional<Failure> allocate() {
        const size_t fe = frame_elems();
        cudaError_t e;
        if ((e = ring_.alloc(fe * total_frames() * sizeof(float))) != cudaSuccess) return gpu_failure("ring", e);
        // nlmeans/denoiser/mod.rs:225 (`needs_reference_buf`): every prefilter keeps a reference ring.
        if (has_reference() && (e = ref_.alloc(fe * total_frames() * sizeof(float))) != cudaSuccess)
            return gpu_failure("reference ring", e);
        for (auto& o : outputs_)
            if ((e = o.alloc(fe * sizeof(float))) != cudaSuccess) return gpu_failure("output slot", e);
        if ((e = derived_.alloc(16 * sizeof(float))) != cudaSuccess) return gpu_failure("derived words", e);
        // Integer outputs: the list of pixels the exact finish recomputes (nlm_exact.cu) and its count.
        if (out_.kind != AVD_SAMPLE_F32 && !exact_all_ && (e = fix_.alloc((pixels() + 1) * sizeof(int))) != cudaSuccess)
            return gpu_failure("exact-finish list", e);
        // Fixed derived words (nlmeans/denoiser/noise.rs `fixed_derived_values`): the strength and,
        // with an HQ sigma override, the noise offset.
        float words[16] = {0};
        const bool has_sigma = params_.hq && params_.hq_params.has_sigma_override;
        const float sigma = params_.hq_params.sigma_override;
        words[0] = h2_inv_norm_with(params_, has_sigma, sigma);
        float sig[2] = {sigma, sigma};
        const float input_offset = has_sigma ? noise_offset_with(params_, sig, 2) : 0.0f;
        // noise.rs:343-390: under the NLM pilot the main pass compares pilot outputs, which carry
        // no noise floor, and the pilot (word 3) runs at h2 / strength_scale^2 (dispatch/mod.rs:40-43).
        words[1] = runs_pilot() ? 0.0f : input_offset;
        if (runs_pilot()) {
            const float sc = params_.prefilter.strength_scale;
            words[3] = words[0] / (sc * sc);
        }
        if (mc_ && (e = allocate_motion()) != cudaSuccess) return gpu_failure("motion compensation buffers", e);
        if (mc_) {
            // noise.rs:360-363 with dispatch/motion.rs:28-72: the window search's SAD floor (word 4)
            // at the pinned sigma times the prefilter's residual fraction (0 for both prefilters).
            const float residual = has_reference() ? 0.0f : 1.0f;
            words[kFixedSadFloor] = avd_sad_noise_floor(mc_blksize(), (has_sigma ? sigma : 0.0f) * residual);
        }
        if (conf_pass_) {
            // motion/confidence.rs:17-30; nlmeans/denoiser/noise.rs:365-368: the confidence floor
            // uses the pinned sigma unscaled by any prefilter.
            conf_bx_ = std::max<uint32_t>((width_ + kConfStep - 1) / kConfStep, 1);
            conf_by_ = std::max<uint32_t>((height_ + kConfStep - 1) / kConfStep, 1);
            const size_t blocks = static_cast<size_t>(conf_bx_) * conf_by_;
            const size_t nbrs = 2 * params_.temporal_radius;
            const size_t pyr = static_cast<size_t>(pyramid_floats(static_cast<int>(width_), static_cast<int>(height_),
                                                                  static_cast<int>(total_frames()), 1));
            if ((e = pyramid_.alloc(pyr * sizeof(float))) != cudaSuccess) return gpu_failure("confidence pyramid", e);
            if ((e = mv_scratch_.alloc(nbrs * blocks * 2 * sizeof(int32_t))) != cudaSuccess)
                return gpu_failure("confidence vectors", e);
            if ((e = conf_.alloc(nbrs * blocks * sizeof(float))) != cudaSuccess) return gpu_failure("confidence", e);
            words[2] = avd_sad_noise_floor(kConfBlk, has_sigma ? sigma : 0.0f);
            thsad_ = avd_thsad(kConfBlk, params_.hq_params.thsad_scale);
        }
        if ((e = cudaMemcpy(derived_.ptr, words, sizeof(words), cudaMemcpyHostToDevice)) != cudaSuccess)
            return gpu_failure("derived upload", e);
        if (params_.hq) {
            // noise/correlation.rs:71-88 (`build_spatial_offset_lut`): with no measured grain
            // correlation (rho = 0) every candidate but the centre takes the flat noise offset; the
            // main pass's table holds its own offset, the pilot's the input's (noise/fold.rs:96-109).
            const uint32_t side = 2 * params_.search_radius + 1;
            auto upload = [&](DeviceBuffer& dst, float offset, const char* what) -> std::optional<Failure> {
                std::vector<float> lut(side * side, offset);
                lut[params_.search_radius * side + params_.search_radius] = 0.0f;
                cudaError_t err;
                if ((err = dst.alloc(lut.size() * sizeof(float))) != cudaSuccess) return gpu_failure(what, err);
                if ((err = cudaMemcpy(dst.ptr, lut.data(), lut.size() * sizeof(float), cudaMemcpyHostToDevice)) !=
                    cudaSuccess)
                    return gpu_failure(what, err);
                return std::nullopt;
            };
            if (auto f = upload(lut_, words[1], "offset table")) return f;
            if (runs_pilot())
                if (auto f = upload(pilot_lut_, input_offset, "pilot offset table")) return f;
        }
        slot_frames_.assign(total_frames(), 0u);
        if (measures_) return allocate_noise();
        return std::nullopt;
    }

    // The measured noise state (noise/state.rs:172-330 `measurement_buffers`, lookahead.rs:53-112)
    // with the fold coefficients of nlmeans/denoiser/noise.rs:200-246 (each factor at a sigma of 1).
    std::optional<Failure> allocate_noise() {
        NoiseFrontConfig cfg;
        cfg.width = width_;
        cfg.height = height_;
        cfg.channels = params_.channel_count();
        cfg.temporal_radius = params_.temporal_radius;
        cfg.table_radius = params_.search_radius;
        FoldCoefficients& k = cfg.coefficients;
        k.sigma_scale = params_.hq_params.sigma_scale;
        k.h2_auto = params_.hq_params.auto_strength;
        k.h2_per_inverse_variance = h2_inv_norm_with(params_, true, 1.0f);
        k.h2_fixed = h2_inv_norm_with(params_, false, 0.0f);
        const float unit[1] = {1.0f};
        k.offset_per_variance = noise_offset_with(params_, unit, 1);
        if (runs_pilot()) {
            // noise.rs:218-224: the pilot's strength factor at h2 = 1; the main pass takes no offset.
            const float sc = params_.prefilter.strength_scale;
            k.pilot_h2_factor = 1.0f / (sc * sc);
            k.main_offset = false;
        }
        k.confidence_sad_per_sigma = conf_pass_ ? avd_sad_noise_floor(kConfBlk, 1.0f) : 0.0f;
        if (mc_) {
            // noise.rs:226-229: the window search's floor per unit sigma, the prefilter's residual
            // fraction applied; the look-ahead reads each frame along its motion (lookahead.rs).
            k.sad_per_sigma = avd_sad_noise_floor(mc_blksize(), has_reference() ? 0.0f : 1.0f);
            cfg.motion = true;
            cfg.blksize = static_cast<int>(params_.motion.search.blksize);
            cfg.overlap = static_cast<int>(params_.motion.search.overlap);
            cfg.search_radius = static_cast<int>(params_.motion.search.search_radius);
            cfg.levels = static_cast<int>(params_.motion.search.pyramid_levels);
            cfg.thsad = mc_thsad();
            cfg.ceiling = mc_ceiling_;
        }
        return noise_.allocate(cfg);
    }

    static Failure gpu_failure(const char* what, cudaError_t e) { return Failure{AVD_ERR_GPU, cuda_message(what, e)}; }

    std::optional<Failure> guard(std::optional<Failure> f) {
        if (f && f->status == AVD_ERR_GPU) poisoned_ = true;
        return f;
    }

    std::optional<Failure> check_planes(const AvdPlane* planes, const AvdSampleFormat& fmt) const {
        // engine/plane.rs:348-377 (`check_planes`); the planar engine already checked the count.
        const uint64_t need = plane_bytes(fmt, pixels());
        for (uint32_t i = 0; i < params_.channel_count(); ++i) {
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

    float bias() const { return params_.channels == Channels::Chroma ? 0.5f : 0.0f; }

    float* slot_ptr(size_t slot) const { return ring_.as<float>() + slot * frame_elems(); }

    // nlmeans/denoiser/mod.rs:484-512 (`push_planes`): a front that measures the noise reads the
    // frame in the look-ahead first; otherwise the frame goes straight into the next ring slot.
    std::optional<Failure> push_planes(const AvdPlane* planes) {
        if (measures_) return push_into_lookahead(planes);
        const size_t slot = ring_head_ % total_frames();
        if (auto f = ingest_into(planes, slot_ptr(slot))) return f;
        return enter_ring(slot);
    }

    std::optional<Failure> ingest_into(const AvdPlane* planes, float* dst) {
        const void* p0 = reinterpret_cast<const void*>(planes[0].ptr);
        const void* p1 = params_.channel_count() > 1 ? reinterpret_cast<const void*>(planes[1].ptr) : nullptr;
        cudaError_t e = launch_ingest(p0, p1, dst, static_cast<int64_t>(pixels()),
                                      static_cast<int>(params_.channel_count()), plane_format(in_), bias(), stream);
        if (e != cudaSuccess) return gpu_failure("ingest launch", e);
        return std::nullopt;
    }

    // nlmeans/denoiser/stages.rs:15-26: the per-frame stages of a frame entering ring slot `slot`.
    // noise.rs:147-165: with the pilot, the stream's first frame folds the window around frame 0
    // first, since the pilot reads the derived words and no pass has folded any yet.
    std::optional<Failure> enter_ring(size_t slot) {
        if (runs_pilot() && measures_ && frames_loaded_ == 0)
            if (auto f = noise_.fold(0, stream)) return f;
        if (auto f = run_prefilter(slot)) return f;
        if (auto f = mc_slot_written(slot, false)) return f;
        if (auto f = slot_written(slot)) return f;
        slot_frames_[slot] = static_cast<uint32_t>(real_pushes_);
        advance_ring();
        return prime_leading_edge_if_first();
    }

    // ---- the noise look-ahead (nlmeans/denoiser/lookahead.rs:182-259) ----
    size_t held() const { return measures_ ? noise_.held() : 0; }

    std::optional<Failure> push_into_lookahead(const AvdPlane* planes) {
        if (noise_.held() == NoiseFront::kFrames) {
            bool released = false;
            if (auto f = release_held_frame(&released)) return f;
        }
        if (auto f = noise_.before_ingest(stream)) return f;
        if (auto f = ingest_into(planes, noise_.slot(noise_.pushed()))) return f;
        return noise_.read_pushed(stream);
    }

    // lookahead.rs:226-259 (`release_held_frame`): the oldest held frame enters the next ring slot.
    std::optional<Failure> release_held_frame(bool* released) {
        *released = false;
        if (!measures_) return std::nullopt;
        const std::optional<size_t> frame = noise_.take_oldest();
        if (!frame) return std::nullopt;
        const size_t slot = ring_head_ % total_frames();
        cudaError_t e = cudaMemcpyAsync(slot_ptr(slot), noise_.slot(*frame), frame_elems() * sizeof(float),
                                        cudaMemcpyDeviceToDevice, stream);
        if (e != cudaSuccess) return gpu_failure("look-ahead release", e);
        *released = true;
        return enter_ring(slot);
    }

    // ring.rs:12-20.
    void advance_ring() {
        ring_head_ += 1;
        if (frames_loaded_ < total_frames()) frames_loaded_ += 1;
        real_pushes_ += 1;
    }

    // ring.rs:106-123: Repeat edges copy the first frame into the d leading slots.
    std::optional<Failure> prime_leading_edge_if_first() {
        const uint32_t d = params_.temporal_radius;
        if (d == 0 || frames_loaded_ != 1) return std::nullopt;
        for (uint32_t i = 0; i < d; ++i) {
            if (auto f = duplicate_last_frame()) return f;
            frames_loaded_ += 1;
        }
        return std::nullopt;
    }

    // ring.rs:128-180: the input slot (and a bilateral reference slot) copied; the pilot rebuilds
    // the duplicated slot's reference instead.
    std::optional<Failure> duplicate_last_frame() {
        const size_t tf = total_frames();
        const size_t last = (ring_head_ - 1) % tf;
        const size_t next = ring_head_ % tf;
        cudaError_t e = cudaMemcpyAsync(slot_ptr(next), slot_ptr(last), frame_elems() * sizeof(float),
                                        cudaMemcpyDeviceToDevice, stream);
        if (e != cudaSuccess) return gpu_failure("slot copy", e);
        if (has_reference() && !runs_pilot()) {
            e = cudaMemcpyAsync(ref_slot_ptr(next), ref_slot_ptr(last), frame_elems() * sizeof(float),
                                cudaMemcpyDeviceToDevice, stream);
            if (e != cudaSuccess) return gpu_failure("reference slot copy", e);
        }
        if (runs_pilot())
            if (auto f = run_pilot(next)) return f;
        if (auto f = mc_slot_written(next, true)) return f;
        if (auto f = slot_written(next)) return f;
        slot_frames_[next] = slot_frames_[last];
        ring_head_ += 1;
        return std::nullopt;
    }

    // ---- prefilters (nlmeans/prefilter/mod.rs, denoiser/stages.rs:29-59) ----
    bool has_reference() const { return params_.prefilter.kind != AVD_PREFILTER_NONE; }
    bool runs_pilot() const { return params_.prefilter.kind == AVD_PREFILTER_NLM_SPATIAL; }
    float* ref_slot_ptr(size_t slot) const { return ref_.as<float>() + slot * frame_elems(); }

    // stages.rs:29-59: the reference of a frame just written to ring slot `slot`.
    std::optional<Failure> run_prefilter(size_t slot) {
        if (runs_pilot()) return run_pilot(slot);
        if (params_.prefilter.kind != AVD_PREFILTER_BILATERAL) return std::nullopt;
        // prefilter/bilateral.rs:11-22, 24-61.
        const float ss = params_.prefilter.sigma_s, sr = params_.prefilter.sigma_r;
        const int radius = static_cast<int>(bilateral_radius(ss));
        cudaError_t e = launch_bilateral(slot_ptr(slot), ref_slot_ptr(slot), static_cast<int>(width_),
                                         static_cast<int>(height_), static_cast<int>(params_.channel_count()), radius,
                                         inv_two_sigma_sq(ss), inv_two_sigma_sq(sr), stream);
        if (e != cudaSuccess) return gpu_failure("bilateral prefilter launch", e);
        return std::nullopt;
    }

    // dispatch/mod.rs:598-620 (`run_nlm_spatial_pilot`): the single-frame windowed pass over the
    // noisy input of `slot` at the pilot strength with the pilot's offset table, finished into the
    // slot's reference. The reference is a float intermediate that every later distance reads, so
    // the exact finish cannot pick out samples near a change of code here: the pilot runs through
    // the exact kernel on every sample, in the reference kernels' operation order.
    std::optional<Failure> run_pilot(size_t slot) {
        NlmLaunch a{};
        a.ring = ring_.as<float>();
        a.width = static_cast<int>(width_);
        a.height = static_cast<int>(height_);
        a.channels = static_cast<int>(params_.channel_count());
        a.frame_elems = static_cast<int64_t>(frame_elems());
        a.slot_centre = static_cast<int>(slot);
        a.pairs = 0;
        a.patch_radius = static_cast<int>(params_.patch_radius);
        a.search_radius = static_cast<int>(params_.search_radius);
        a.derived = measures_ ? noise_.derived() : derived_.as<float>();
        a.h2_word = measures_ ? kDerivedPilotH2 : 3;
        a.offset_word = measures_ ? kDerivedNoiseOffset : 1;
        a.spatial_lut = measures_ ? noise_.pilot_table() : (params_.hq ? pilot_lut_.as<float>() : nullptr);
        a.wref = params_.self_weight;
        a.fast = params_.hq ? 0 : 1;
        a.out = ref_slot_ptr(slot);
        cudaError_t e = launch_nlm_exact(a, stream);
        if (e != cudaSuccess) return gpu_failure("nlm pilot launch", e);
        return std::nullopt;
    }

    // ---- motion compensation (nlmeans/dispatch/motion.rs, denoiser/stages.rs:62-209) ----
    uint32_t mc_blksize() const { return params_.motion.search.blksize; }
    int mc_step() const { return static_cast<int>(params_.motion.search.blksize - params_.motion.search.overlap); }
    float mc_thsad() const {
        // dispatch/motion.rs:75-79 (`search_thsad`).
        return avd_thsad(mc_blksize(), params_.hq ? params_.hq_params.thsad_scale : 1.0f);
    }
    // A pass that refines the luma pass's motion matches on one level (seeds.rs:184-208).
    int mc_levels() const { return reads_share_ ? 1 : static_cast<int>(params_.motion.search.pyramid_levels); }
    float* mc_search_pyramid() const { return has_reference() ? mc_ref_pyr_.as<float>() : mc_pyr_.as<float>(); }

    cudaError_t allocate_motion() {
        const int step = mc_step();
        mc_bx_ = std::max<int>((static_cast<int>(width_) + step - 1) / step, 1);
        mc_by_ = std::max<int>((static_cast<int>(height_) + step - 1) / step, 1);
        mc_mv_stride_ = static_cast<int>((2LL * mc_bx_ * mc_by_ + 7) / 8 * 8);
        mc_conf_stride_ = static_cast<int>((static_cast<int64_t>(mc_bx_) * mc_by_ + 7) / 8 * 8);
        const size_t nbrs = 2 * params_.temporal_radius, fe = frame_elems(), t = total_frames();
        const size_t pyr = static_cast<size_t>(
            pyramid_floats(static_cast<int>(width_), static_cast<int>(height_), static_cast<int>(t), mc_levels()));
        cudaError_t e;
        if ((e = mc_pyr_.alloc(pyr * sizeof(float))) != cudaSuccess) return e;
        if ((e = comp_.alloc(fe * t * sizeof(float))) != cudaSuccess) return e;
        if (has_reference()) {
            if ((e = mc_ref_pyr_.alloc(pyr * sizeof(float))) != cudaSuccess) return e;
            if ((e = comp_ref_.alloc(fe * t * sizeof(float))) != cudaSuccess) return e;
        }
        if ((e = mc_mv_.alloc(nbrs * mc_mv_stride_ * sizeof(int32_t))) != cudaSuccess) return e;
        if ((e = tm_seeds_.alloc(nbrs * mc_mv_stride_ * sizeof(int32_t))) != cudaSuccess) return e;
        if ((e = tm_field_.alloc(nbrs * mc_mv_stride_ * sizeof(int32_t))) != cudaSuccess) return e;
        if (mc_ceiling_ && !reads_share_) {
            const size_t state = escalation_state_floats(static_cast<int>(nbrs), mc_conf_stride_);
            if ((e = esc_state_.alloc(state * sizeof(float))) != cudaSuccess) return e;
            if ((e = tm_changes_.alloc(nbrs * mc_conf_stride_ * sizeof(uint32_t))) != cudaSuccess) return e;
        }
        if (mc_conf_ && (e = mc_conf_buf_.alloc(nbrs * mc_conf_stride_ * sizeof(float))) != cudaSuccess) return e;
        if (mc_chained_) {
            // motion/context.rs:209-211: 2d pair slots of two directions each.
            if ((e = pair_ring_.alloc(nbrs * 2 * mc_mv_stride_ * sizeof(int32_t))) != cudaSuccess) return e;
            if ((e = cudaMemset(pair_ring_.ptr, 0, pair_ring_.bytes)) != cudaSuccess) return e;
        }
        return cudaSuccess;
    }

    MotionLaunch mc_launch() const {
        MotionLaunch m{};
        m.pyramid = mc_search_pyramid();
        m.noise = measures_ ? noise_.derived() : derived_.as<float>();
        m.width = static_cast<int>(width_);
        m.height = static_cast<int>(height_);
        m.frame_count = static_cast<int>(total_frames());
        m.blksize = static_cast<int>(params_.motion.search.blksize);
        m.overlap = static_cast<int>(params_.motion.search.overlap);
        m.search_radius = static_cast<int>(params_.motion.search.search_radius);
        m.coarse_radius = m.search_radius;
        m.coarse_block_factor = 1;
        m.levels = mc_levels();
        m.mv_stride = mc_mv_stride_;
        m.conf_stride = mc_conf_stride_;
        m.sad_floor_word = measures_ ? kDerivedSadFloor : kFixedSadFloor;
        m.thsad = mc_thsad();
        // analyse.rs:371-380: a search (and a seeded refine below the ceiling) escalates; the
        // luma-mapped refine runs a fixed schedule.
        if (mc_ceiling_ && !reads_share_) {
            m.escalation = esc_state_.as<float>();
            m.ceiling = mc_ceiling_;
        }
        return m;
    }

    // stages.rs:62-108 and 146-209: a slot's pyramids (the input's, and the reference's under a
    // prefilter), then the pair between it and the slot before (both ways, into pair slot ring_head
    // mod 2d), or, for an edge copy, that pair slot zeroed.
    std::optional<Failure> mc_slot_written(size_t slot, bool duplicate) {
        if (!mc_) return std::nullopt;
        const int t = static_cast<int>(total_frames());
        cudaError_t e = launch_pyramid_build(ring_.as<float>(), static_cast<int>(params_.channel_count()),
                                             static_cast<int>(width_), static_cast<int>(height_), t,
                                             static_cast<int>(slot), mc_levels(), mc_pyr_.as<float>(),
                                             static_cast<int>(slot), stream);
        if (e == cudaSuccess && has_reference())
            e = launch_pyramid_build(ref_.as<float>(), static_cast<int>(params_.channel_count()),
                                     static_cast<int>(width_), static_cast<int>(height_), t, static_cast<int>(slot),
                                     mc_levels(), mc_ref_pyr_.as<float>(), static_cast<int>(slot), stream);
        if (e != cudaSuccess) return gpu_failure("motion pyramid launch", e);
        if (!mc_chained_) return std::nullopt;
        const size_t d = params_.temporal_radius;
        int32_t* pair = pair_ring_.as<int32_t>() + (ring_head_ % (2 * d)) * 2 * mc_mv_stride_;
        if (duplicate) {
            if ((e = cudaMemsetAsync(pair, 0, 2 * mc_mv_stride_ * sizeof(int32_t), stream)) != cudaSuccess)
                return gpu_failure("pair clear", e);
            return std::nullopt;
        }
        if (ring_head_ == 0) return std::nullopt;
        const size_t older = (slot + total_frames() - 1) % total_frames();
        // stages.rs:15-22, 172-180 with seeds.rs:104-134: both directions' predictions between the
        // older slot's frame and the frame entering now (its slot records it after this search), the
        // searches scored against zeroed noise words.
        if (models_)
            if (auto f = models_->compose_pair(slot_frames_[older], static_cast<uint32_t>(real_pushes_), pred_pair_.as<float>(),
                                               pred_pair_.as<float>() + kAffineWords, stream))
                return f;
        for (int dir = 0; dir < 2; ++dir) {
            MotionLaunch m = mc_launch();
            m.inline_slots[0] = static_cast<uint32_t>(dir == 0 ? slot : older);
            m.centre_slot = static_cast<int>(dir == 0 ? older : slot);
            m.neighbours = 1;
            m.mv_field = pair + dir * mc_mv_stride_;
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

    // motion/analyse.rs:175-312: the search, then one truemotion pass (field_lambda 1, the NLMeans
    // front's default) with the coarse pass's field as the seed candidates.
    std::optional<Failure> search_then_truemotion(MotionLaunch m, bool reads_floor) {
        const bool coarse = m.levels > 1 && !m.seeded;
        if (coarse) m.keep_seeds = tm_seeds_.as<int32_t>();
        // truemotion/params.rs:9-12, 79-90: two passes after a search that escalates.
        const bool two_passes = m.escalation && m.ceiling > m.search_radius;
        cudaError_t e = launch_motion_search(m, stream);
        if (e != cudaSuccess) return gpu_failure("motion search launch", e);
        TruemotionLaunch t{};
        t.pyramid = m.pyramid;
        t.slot_pixels = pyramid_slot_pixels(m.width, m.height, 0);
        t.neighbour_slots = nullptr;
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
        t.step = mc_step();
        t.blocks_x = mc_bx_;
        t.blocks_y = mc_by_;
        t.mv_stride = mc_mv_stride_;
        t.conf_stride = mc_conf_stride_;
        t.sad_field = m.sad_floor_word;
        t.reads_floor = reads_floor ? 1 : 0;
        t.refine_radius = 1;  // truemotion/params.rs:15
        // truemotion/stage.rs:52-62 with params.rs:4-33 at the default field_lambda 1.
        const float lambda = 1.0f;
        t.lambda_base = lambda * static_cast<float>(m.blksize * m.blksize) * 0.02f;
        t.lambda_noise = lambda * 1.0f;
        t.surcharge = 0.125f;
        t.fade_level = 2.0f * std::max(m.thsad, 0.0f);
        t.thsad = m.thsad;
        t.predictions = m.predictions;
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
        e = cudaMemcpyAsync(m.mv_field, t.mv_out, static_cast<size_t>(m.neighbours) * mc_mv_stride_ * sizeof(int32_t),
                            cudaMemcpyDeviceToDevice, stream);
        if (e != cudaSuccess) return gpu_failure("truemotion field copy", e);
        return std::nullopt;
    }

    // dispatch/motion.rs:427-487 then 104-229: the centre copied through, every neighbour's motion
    // estimated (Chained: the pair walk refined with confidence; Direct: the search with its
    // truemotion stage reading the window's floor), then each neighbour warped into the
    // compensated rings (compensate.rs).
    std::optional<Failure> run_motion_compensation() {
        const int d = static_cast<int>(params_.temporal_radius);
        const size_t centre = static_cast<size_t>(phys_frame(d));
        const size_t bytes = frame_elems() * sizeof(float);
        cudaError_t e = cudaSuccess;
        if (!guides_) {
            e = cudaMemcpyAsync(comp_.as<float>() + centre * frame_elems(), slot_ptr(centre), bytes,
                                cudaMemcpyDeviceToDevice, stream);
            if (e == cudaSuccess && has_reference())
                e = cudaMemcpyAsync(comp_ref_.as<float>() + centre * frame_elems(), ref_slot_ptr(centre), bytes,
                                    cudaMemcpyDeviceToDevice, stream);
            if (e != cudaSuccess) return gpu_failure("centre copy", e);
        }
        MotionLaunch m = mc_launch();
        int n = 0;
        for (int l = 0; l <= 2 * d; ++l)
            if (l != d) m.inline_slots[n++] = static_cast<uint32_t>(phys_frame(l));
        m.centre_slot = static_cast<int>(centre);
        m.neighbours = n;
        m.mv_field = mc_mv_.as<int32_t>();
        m.confidence = mc_conf_ ? mc_conf_buf_.as<float>() : nullptr;
        const uint32_t frame = slot_frames_[centre];
        const int share_slot = share_ ? static_cast<int>(frame % static_cast<uint32_t>(share_->slots)) : 0;
        if (reads_share_) {
            // dispatch/motion.rs:255-310 (`refine_luma_motion`): the luma pass's mapped vectors,
            // searched one pixel around at one level, with confidence.
            if (share_->tags[share_slot] != static_cast<int64_t>(frame)) {
                char msg[120];
                std::snprintf(msg, sizeof(msg), "the luma pass has not shared the motion of stream frame %u", frame);
                return Failure{AVD_ERR_GPU, msg};
            }
            e = cudaMemcpyAsync(mc_mv_.as<int32_t>(), share_->slot_ptr(share_slot),
                                static_cast<size_t>(n) * mc_mv_stride_ * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                                stream);
            if (e != cudaSuccess) return gpu_failure("mapped motion copy", e);
            m.search_radius = 1;  // dispatch/motion.rs:44 (MAPPED_REFINE_RADIUS)
            m.coarse_radius = 1;
            m.levels = 1;
            m.seeded = 1;
            if ((e = launch_motion_search(m, stream)) != cudaSuccess) return gpu_failure("mapped refine launch", e);
        } else if (mc_chained_) {
            e = launch_chain_compose(pair_ring_.as<int32_t>(), mc_mv_.as<int32_t>(), mc_mv_stride_, d, d,
                                     static_cast<int>(ring_head_ % (2 * d)), mc_mv_stride_, 2 * mc_mv_stride_,
                                     mc_step(), static_cast<int>(width_), static_cast<int>(height_), mc_bx_, mc_by_,
                                     stream);
            if (e != cudaSuccess) return gpu_failure("chain compose launch", e);
            m.search_radius = mc_refine_radius_;
            m.coarse_radius = mc_refine_radius_;
            m.seeded = 1;
            // dispatch/motion.rs:197-201: the window's derived noise is the escalation floor.
            m.esc_reads_floor = 1;
            if ((e = launch_motion_search(m, stream)) != cudaSuccess) return gpu_failure("seeded refine launch", e);
        } else {
            m.esc_reads_floor = 1;
            if (models_) {
                // dispatch/motion.rs:190-195 with seeds.rs:136-160: every neighbour's prediction for
                // the window's stream frames (the chained seeds already carry the camera's motion).
                uint32_t frames[2 * kMaxTemporalRadius + 1];
                for (int l = 0; l <= 2 * d; ++l) frames[l] = slot_frames_[phys_frame(l)];
                if (auto f = models_->compose_window(frames, 2 * d + 1, d, pred_window_.as<float>(), stream)) return f;
                m.predictions = pred_window_.as<float>();
            }
            if (auto f = search_then_truemotion(m, true)) return f;
        }
        if (writes_share_) {
            // dispatch/motion.rs:231-253 (`share_window_motion`).
            MapLaunch mp{};
            mp.luma = mc_mv_.as<int32_t>();
            mp.chroma = share_->slot_ptr(share_slot);
            mp.fields = n;
            mp.luma_bx = mc_bx_;
            mp.luma_by = mc_by_;
            mp.luma_step = mc_step();
            mp.luma_blksize = static_cast<int>(mc_blksize());
            mp.luma_stride = mc_mv_stride_;
            mp.chroma_bx = share_->blocks_x;
            mp.chroma_by = share_->blocks_y;
            mp.chroma_step = share_->step;
            mp.chroma_blksize = share_->blksize;
            mp.chroma_stride = share_->mv_stride;
            mp.shift_x = share_->shift_x;
            mp.shift_y = share_->shift_y;
            if ((e = launch_map_luma_fields(mp, stream)) != cudaSuccess) return gpu_failure("luma motion map launch", e);
            share_->tags[share_slot] = frame;
        }
        // dispatch/mod.rs:648-651: a front that only guides stops after the window's motion.
        if (guides_) return std::nullopt;
        WarpLaunch w{};
        w.src_ring = ring_.as<float>();
        w.dst_ring = comp_.as<float>();
        w.src_ref = has_reference() ? ref_.as<float>() : nullptr;
        w.dst_ref = has_reference() ? comp_ref_.as<float>() : nullptr;
        w.mv_field = mc_mv_.as<int32_t>();
        w.mv_stride = mc_mv_stride_;
        for (int i = 0; i < n; ++i) w.slots[i] = m.inline_slots[i];
        w.neighbours = n;
        w.frame_elems = static_cast<int64_t>(frame_elems());
        w.channels = static_cast<int>(params_.channel_count());
        w.width = static_cast<int>(width_);
        w.height = static_cast<int>(height_);
        w.step = mc_step();
        w.blocks_x = mc_bx_;
        w.blocks_y = mc_by_;
        if ((e = launch_warp(w, stream)) != cudaSuccess) return gpu_failure("warp launch", e);
        return std::nullopt;
    }

   public:
    // engine/spec.rs:350-365 and nlmeans/denoiser/seeds.rs:168-208: with motion compensation on both
    // passes, the chroma pass reads the luma pass's motion and drops its own search.
    static std::optional<Failure> link(NlmPass& luma, NlmPass& chroma, int shift_x, int shift_y) {
        if (!luma.mc_ || !chroma.mc_) return std::nullopt;
        if (luma.params_.temporal_radius != chroma.params_.temporal_radius)
            return Failure{AVD_ERR_INVALID_OPTIONS, "the luma and chroma windows differ"};
        auto share = std::make_shared<LumaMotionShare>();
        share->slots = static_cast<int>(chroma.total_frames());
        share->neighbours = static_cast<int>(2 * chroma.params_.temporal_radius);
        share->blocks_x = chroma.mc_bx_;
        share->blocks_y = chroma.mc_by_;
        share->step = chroma.mc_step();
        share->blksize = static_cast<int>(chroma.mc_blksize());
        share->mv_stride = chroma.mc_mv_stride_;
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
        chroma.mc_chained_ = false;
        return std::nullopt;
    }

   private:
    std::shared_ptr<LumaMotionShare> share_;
    bool writes_share_ = false, reads_share_ = false;
    bool guides_ = false;

    // nlmeans/denoiser/stages.rs:110-130: the confidence pyramid follows every ring slot write.
    std::optional<Failure> slot_written(size_t slot) {
        if (!conf_pass_) return std::nullopt;
        cudaError_t e = launch_pyramid_build(ring_.as<float>(), static_cast<int>(params_.channel_count()),
                                             static_cast<int>(width_), static_cast<int>(height_),
                                             static_cast<int>(total_frames()), static_cast<int>(slot), 1,
                                             pyramid_.as<float>(), static_cast<int>(slot), stream);
        if (e != cudaSuccess) return gpu_failure("confidence pyramid launch", e);
        return std::nullopt;
    }

    // nlmeans/dispatch/motion.rs:554-613 (`run_confidence_pass`): every neighbour in logical order,
    // the centre skipped, scored where each block stands.
    std::optional<Failure> run_confidence_pass() {
        const int d = static_cast<int>(params_.temporal_radius);
        MotionLaunch m{};
        m.pyramid = pyramid_.as<float>();
        m.neighbour_slots = nullptr;
        int n = 0;
        for (int l = 0; l <= 2 * d; ++l)
            if (l != d) m.inline_slots[n++] = static_cast<uint32_t>(phys_frame(l));
        m.mv_field = mv_scratch_.as<int32_t>();
        m.confidence = conf_.as<float>();
        m.noise = measures_ ? noise_.derived() : derived_.as<float>();
        m.width = static_cast<int>(width_);
        m.height = static_cast<int>(height_);
        m.frame_count = static_cast<int>(total_frames());
        m.centre_slot = phys_frame(d);
        m.neighbours = n;
        m.blksize = kConfBlk;
        m.overlap = kConfBlk - kConfStep;
        m.search_radius = 0;
        m.coarse_radius = 0;
        m.coarse_block_factor = 1;
        m.levels = 1;
        m.mv_stride = static_cast<int>(conf_bx_ * conf_by_ * 2);
        m.conf_stride = static_cast<int>(conf_bx_ * conf_by_);
        m.sad_floor_word = measures_ ? kDerivedConfidenceSadFloor : 2;
        m.thsad = thsad_;
        cudaError_t e = launch_motion_search(m, stream);
        if (e != cudaSuccess) return gpu_failure("confidence launch", e);
        return std::nullopt;
    }

    // ring.rs:182-194.
    size_t ring_start() const { return ring_head_ % total_frames(); }
    int phys_frame(int logical) const {
        const int tf = static_cast<int>(total_frames());
        int wrapped = ((logical % tf) + tf) % tf;
        return (static_cast<int>(ring_start()) + wrapped) % tf;
    }
    uint32_t centre_frame() const { return slot_frames_[phys_frame(static_cast<int>(params_.temporal_radius))]; }

    // nlmeans/denoiser/mod.rs:517-532 (`denoise_submit_gpu`).
    std::optional<Failure> denoise_submit(int* out_slot) {
        *out_slot = -1;
        if (frames_loaded_ < total_frames()) return std::nullopt;
        const int slot = next_output_slot_;
        next_output_slot_ = (slot + 1) % 2;

        cudaEvent_t start{};
        bool timed = timer_.begin(stream, &start);
        // dispatch/mod.rs:640-644: the look-ahead has read every frame the window reaches, so the fold
        // runs first and the confidence pass reads this centre's own derived words.
        if (measures_)
            if (auto f = noise_.fold(centre_frame(), stream)) return f;
        const int d = static_cast<int>(params_.temporal_radius);
        NlmLaunch a{};
        a.ring = ring_.as<float>();
        a.width = static_cast<int>(width_);
        a.height = static_cast<int>(height_);
        a.channels = static_cast<int>(params_.channel_count());
        a.frame_elems = static_cast<int64_t>(frame_elems());
        a.slot_centre = phys_frame(d);
        a.pairs = d;
        for (int k = 0; k < d; ++k) {
            const int q_k = -d + k;
            a.slot_fwd[k] = phys_frame(d + q_k);
            a.slot_bwd[k] = phys_frame(d - q_k);
        }
        a.patch_radius = static_cast<int>(params_.patch_radius);
        a.search_radius = static_cast<int>(params_.search_radius);
        a.derived = measures_ ? noise_.derived() : derived_.as<float>();
        a.h2_word = measures_ ? kDerivedH2 : 0;
        a.offset_word = measures_ ? kDerivedNoiseOffset : 1;
        a.spatial_lut = measures_ ? noise_.spatial_table() : (params_.hq ? lut_.as<float>() : nullptr);
        a.conf = nullptr;
        if (guides_) {
            if (auto f = run_motion_compensation()) return f;
            if (timed) timer_.end(stream, start);
            *out_slot = slot;
            return std::nullopt;
        }
        if (mc_) {
            if (auto f = run_motion_compensation()) return f;
            // dispatch/mod.rs:141-200: the temporal passes read the compensated rings, weighted by
            // the window search's confidence per motion block.
            a.ring = comp_.as<float>();
            if (mc_conf_) {
                a.conf = mc_conf_buf_.as<float>();
                for (int k = 0; k < d; ++k) {
                    a.conf_fwd_off[k] = static_cast<int64_t>(k) * mc_conf_stride_;
                    a.conf_bwd_off[k] = static_cast<int64_t>(2 * d - 1 - k) * mc_conf_stride_;
                }
                a.conf_step = mc_step();
                a.blocks_x = mc_bx_;
                a.blocks_y = mc_by_;
            }
        }
        if (conf_pass_) {
            if (auto f = run_confidence_pass()) return f;
            // dispatch/mod.rs:175-200: pair k (q_k = -d + k) weighs its forward frame by neighbour
            // q_k + d and its backward frame by neighbour d - 1 - q_k.
            const int stride = static_cast<int>(conf_bx_ * conf_by_);
            a.conf = conf_.as<float>();
            for (int k = 0; k < d; ++k) {
                a.conf_fwd_off[k] = k * stride;
                a.conf_bwd_off[k] = (2 * d - 1 - k) * stride;
            }
            a.conf_step = kConfStep;
            a.blocks_x = static_cast<int>(conf_bx_);
            a.blocks_y = static_cast<int>(conf_by_);
        }
        a.wref = params_.self_weight;
        a.fast = params_.hq ? 0 : 1;
        a.out = outputs_[slot].as<float>();
        a.ref_ring = has_reference() ? (mc_ ? comp_ref_.as<float>() : ref_.as<float>()) : nullptr;
        cudaError_t e;
        if (exact_all_) {
            if ((e = launch_nlm_exact(a, stream)) != cudaSuccess) return gpu_failure("exact nlm launch", e);
            if (timed) timer_.end(stream, start);
            *out_slot = slot;
            return std::nullopt;
        }
        if (window_variant_ < 0) window_variant_ = tune_window(a);
        a.variant = window_variant_;
        if (fix_.ptr) {
            // Integer outputs: the window kernel flags the pixels within the band of a change of code
            // and the exact finish recomputes them in the reference kernels' order.
            a.fix_count = fix_.as<int>();
            a.fix_list = fix_.as<int>() + 1;
            a.code_max = sample_max_value(out_);
            a.fix_band = kFixBand;
            if ((e = cudaMemsetAsync(a.fix_count, 0, sizeof(int), stream)) != cudaSuccess)
                return gpu_failure("exact-finish count", e);
        }
        if ((e = launch_nlm(a, stream)) != cudaSuccess) return gpu_failure("nlm launch", e);
        if (fix_.ptr && (e = launch_nlm_exact(a, stream)) != cudaSuccess) return gpu_failure("exact finish launch", e);
        if (timed) {
            timer_.end(stream, start);
            if (fix_.ptr) timer_.note_count(stream, a.fix_count);
        }
        *out_slot = slot;
        return std::nullopt;
    }

    // tune/driver: the window kernel's variant for this pass's shape, each timed once on this very
    // launch (without the exact-finish list) when the tuner has no choice for the shape yet.
    int tune_window(const NlmLaunch& a) {
        char key[160];
        std::snprintf(key, sizeof(key), "nlm_window c%d s%d a%d d%d fast%d conf%d lut%d %dx%d", a.channels,
                      a.patch_radius, a.search_radius, a.pairs, a.fast, a.conf ? 1 : 0, a.spatial_lut ? 1 : 0,
                      a.width, a.height);
        const int variants = a.ref_ring ? 1 : nlm_window_variants(a.channels, a.patch_radius, a.fast != 0);
        return tuned_variant(tune_, key, variants, [&](int v) {
            NlmLaunch t = a;
            t.variant = v;
            t.fix_list = nullptr;
            t.fix_count = nullptr;
            cudaEvent_t e0 = nullptr, e1 = nullptr;
            float ms = -1.0f;
            if (cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess &&
                launch_nlm(t, stream) == cudaSuccess && cudaEventRecord(e0, stream) == cudaSuccess) {
                bool ok = true;
                for (int rep = 0; rep < 3 && ok; ++rep) ok = launch_nlm(t, stream) == cudaSuccess;
                if (ok && cudaEventRecord(e1, stream) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess &&
                    cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
                    ms /= 3.0f;
                else
                    ms = -1.0f;
            }
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
            return ms;
        });
    }

    // nlmeans/denoiser/mod.rs:557-573 (`flush_step_gpu`) without look-ahead.
    // nlmeans/denoiser/mod.rs:551-573 (`flush_step_gpu`): release a held frame, else duplicate the last.
    std::optional<Failure> next_tail_frame(int* slot) {
        for (;;) {
            bool released = false;
            if (auto f = release_held_frame(&released)) return f;
            if (!released) {
                if (auto f = duplicate_last_frame()) return f;
                if (frames_loaded_ < total_frames()) frames_loaded_ += 1;
            }
            if (auto f = denoise_submit(slot)) return f;
            if (*slot >= 0) return std::nullopt;
        }
    }

    std::optional<Failure> write_out(int slot, const AvdPlane* planes) {
        if (guides_) return std::nullopt;  // a guide writes nothing
        void* p0 = reinterpret_cast<void*>(planes[0].ptr);
        void* p1 = params_.channel_count() > 1 ? reinterpret_cast<void*>(planes[1].ptr) : nullptr;
        cudaError_t e = launch_egress(outputs_[slot].as<float>(), p0, p1, static_cast<int64_t>(pixels()),
                                      static_cast<int>(params_.channel_count()), plane_format(out_), bias(), stream);
        if (e != cudaSuccess) return gpu_failure("egress launch", e);
        return std::nullopt;
    }

    // nlmeans/denoiser/mod.rs:580-590 (`reset_stream_state`) and engine.rs:138-141.
    void restart_stream() {
        ring_head_ = 0;
        frames_loaded_ = 0;
        next_output_slot_ = 0;
        real_pushes_ = 0;
        pushed_ = false;
        if (measures_) noise_.reset();
    }

    static constexpr int kDerivedSadFloor = 4, kDerivedConfidenceSadFloor = 5, kDerivedH2 = 6, kDerivedPilotH2 = 7,
                         kDerivedNoiseOffset = 8;  // derived.rs:9-31
    static constexpr int kFixedSadFloor = 4;  // the window search's floor among the fixed words

    bool mc_ = false, mc_chained_ = false, mc_conf_ = false;
    const PairModels* models_ = nullptr;  // the camera models the searches start from, or none
    DeviceBuffer pred_window_, pred_pair_;  // window predictions (2d x 6), pair predictions (2 x 6)
    int mc_refine_radius_ = 2, mc_bx_ = 1, mc_by_ = 1, mc_mv_stride_ = 2, mc_conf_stride_ = 1;
    int mc_ceiling_ = 0;  // the escalation ceiling; 0 when the search does not escalate
    DeviceBuffer mc_pyr_, mc_ref_pyr_, comp_, comp_ref_, mc_mv_, tm_seeds_, tm_field_, mc_conf_buf_, pair_ring_;
    DeviceBuffer esc_state_, tm_changes_;
    bool measures_ = false;
    NoiseFront noise_;

    NlmParams params_;
    size_t held_ = 0;
    uint32_t width_ = 0, height_ = 0;
    AvdSampleFormat in_{}, out_{};
    DeviceBuffer ring_;
    DeviceBuffer outputs_[2];
    DeviceBuffer derived_;
    DeviceBuffer lut_, pilot_lut_;
    DeviceBuffer fix_;  // integer outputs: [count, pixel list] of the exact finish
    bool exact_all_ = false;
    TuneOptions tune_;
    int window_variant_ = -1;  // the tuned window kernel variant, chosen at the first window launch
    DeviceBuffer ref_;  // the prefilter's reference ring, slot for slot beside `ring_`
    std::vector<uint32_t> slot_frames_;
    size_t ring_head_ = 0, frames_loaded_ = 0, real_pushes_ = 0;
    int next_output_slot_ = 0;
    int ready_slot_ = -1;
    size_t tail_remaining_ = 0;
    bool pushed_ = false;
    bool poisoned_ = false;
    std::optional<uint32_t> emitted_;
    DeviceTimer timer_;
};

// ---------------------------------------------------------------------------------------------
// Passthrough ring (engine/passthrough.rs): the uncleaned plane group of recent frames.
class PassthroughRing {
   public:
    std::optional<Failure> init(size_t slots, size_t planes, uint64_t bytes) {
        slots_.resize(slots);
        bytes_ = bytes;
        for (auto& s : slots_) {
            s.resize(planes);
            for (auto& b : s) {
                b = std::make_unique<DeviceBuffer>();
                cudaError_t e = b->alloc(bytes);
                if (e != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("passthrough ring", e)};
            }
        }
        return std::nullopt;
    }
    size_t slots() const { return slots_.size(); }
    cudaError_t store(uint32_t frame, const AvdPlane* planes, size_t n, cudaStream_t s) {
        auto& slot = slots_[frame % slots_.size()];
        for (size_t i = 0; i < n; ++i) {
            cudaError_t e = cudaMemcpyAsync(slot[i]->ptr, reinterpret_cast<const void*>(planes[i].ptr), bytes_,
                                            cudaMemcpyDeviceToDevice, s);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    cudaError_t load(uint32_t frame, const AvdPlane* planes, size_t n, cudaStream_t s) {
        auto& slot = slots_[frame % slots_.size()];
        for (size_t i = 0; i < n; ++i) {
            cudaError_t e = cudaMemcpyAsync(reinterpret_cast<void*>(planes[i].ptr), slot[i]->ptr, bytes_,
                                            cudaMemcpyDeviceToDevice, s);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }

   private:
    std::vector<std::vector<std::unique_ptr<DeviceBuffer>>> slots_;
    uint64_t bytes_ = 0;
};

}  // namespace

}  // namespace avd

// ---------------------------------------------------------------------------------------------
// The planar engine: engine/planar.rs:104-580.
// A second stream for a chroma pass that runs beside the luma pass of the same push, forked from
// and joined back into the engine's stream with two events; made on first use.
struct SideStream {
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;

    cudaError_t ensure() {
        cudaError_t e = cudaSuccess;
        if (!stream) e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
        if (e == cudaSuccess && !fork) e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
        if (e == cudaSuccess && !join) e = cudaEventCreateWithFlags(&join, cudaEventDisableTiming);
        return e;
    }
    ~SideStream() {
        if (stream) {
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
    }
};

struct AvdEngine {
    AvdGeometry geometry{};
    std::unique_ptr<avd::Pass> luma, chroma;
    std::unique_ptr<avd::PassthroughRing> passthrough;
    std::unique_ptr<avd::ColourMeans> colour;  // the block means the passes pool their grain per colour with
    std::unique_ptr<avd::PairModels> models;   // the camera models the luma motion pass searches from
    bool passthrough_luma = false;  // which group the ring holds
    bool luma_guides = false;       // `luma` is a chroma-only engine's luma guide, which cleans nothing
    bool poisoned = false;
    int device = 0;
    cudaStream_t stream = nullptr;
    SideStream side;  // declared after the passes: destroyed (and drained) before them
    std::string last_error;

    avd::Pass* lead() const { return luma ? luma.get() : chroma.get(); }
    // The chroma pass of a push runs beside the luma pass when it reads nothing the luma pass (or
    // the engine's colour measurement) writes in that push.
    bool overlaps_chroma() const { return luma && chroma && !luma_guides && !colour && !chroma->reads_luma(); }
};

namespace {

using avd::Failure;

thread_local std::string g_last_error;

AvdStatus fail_global(AvdStatus st, const std::string& message) {
    g_last_error = message;
    return st;
}

AvdStatus record(AvdEngine* e, AvdStatus st, const std::string& message) {
    if (e) e->last_error = st == AVD_OK ? std::string() : message;
    return st;
}

// planar.rs:253-268 (`fit_pair_model`): stream frame `frame`'s camera model from its luma plane, before
// its passes see it; a failure poisons the engine, as the ring may hold a partly written model.
std::optional<Failure> fit_pair_model(AvdEngine* e, const AvdPlane* planes, uint32_t frame) {
    if (!e->models) return std::nullopt;
    auto f = e->models->push(planes[0], frame, e->stream);
    if (f) e->poisoned = true;
    return f;
}

// planar.rs:194-217 (`measure_colour`): stream frame `frame`'s block means from all three planes,
// before its passes see it, when the passes pool colour cells.
std::optional<Failure> measure_colour(AvdEngine* e, const AvdPlane* planes, uint32_t frame) {
    if (!e->colour) return std::nullopt;
    auto f = e->colour->queue(planes, frame, e->stream);
    if (f) e->poisoned = true;
    return f;
}

AvdStatus record(AvdEngine* e, const std::optional<Failure>& f) {
    if (!f) return record(e, AVD_OK, "");
    return record(e, f->status, f->message);
}

// engine/frame.rs + planar.rs `check_planes`: all planes of the frame, each at its own size.
std::optional<Failure> check_frame_planes(const AvdGeometry& g, const AvdPlane* planes, size_t n,
                                          const AvdSampleFormat& fmt) {
    const size_t expected = avd::plane_count(g.chroma);
    if (n != expected) {
        return Failure{AVD_ERR_PLANE_MISMATCH,
                       "expected " + std::to_string(expected) + " planes, got " + std::to_string(n)};
    }
    for (size_t i = 0; i < n; ++i) {
        uint32_t w, h;
        avd::plane_dims(g, i, &w, &h);
        if (planes[i].width != w || planes[i].height != h) {
            return Failure{AVD_ERR_PLANE_MISMATCH, "plane " + std::to_string(i) + " is " +
                                                       std::to_string(planes[i].width) + "x" +
                                                       std::to_string(planes[i].height) + ", expected " +
                                                       std::to_string(w) + "x" + std::to_string(h)};
        }
        uint64_t need = avd::plane_bytes(fmt, static_cast<uint64_t>(w) * h);
        if (planes[i].bytes < need) {
            return Failure{AVD_ERR_PLANE_MISMATCH, "plane " + std::to_string(i) + " holds " +
                                                       std::to_string(planes[i].bytes) + " bytes, needs " +
                                                       std::to_string(need)};
        }
    }
    return std::nullopt;
}

// planar.rs:375-407 (`forward`): each pass in luma, chroma order; they must agree; a failure
// after one pass moved poisons the engine.
template <typename F>
std::optional<Failure> forward(AvdEngine* e, size_t* agreed_out, F&& call) {
    std::optional<size_t> agreed;
    std::optional<Failure> failure;
    avd::Pass* passes[2] = {e->luma.get(), e->chroma.get()};
    for (int i = 0; i < 2; ++i) {
        avd::Pass* p = passes[i];
        if (!p) continue;
        size_t value = 0;
        if (auto f = call(p, i == 0, &value)) {
            failure = f;
            break;
        }
        if (agreed && *agreed != value) {
            failure = Failure{AVD_ERR_GPU, "the luma pass returned " + std::to_string(*agreed) +
                                               " but the chroma pass " + std::to_string(value)};
            break;
        }
        agreed = value;
    }
    if (failure) {
        if (agreed) e->poisoned = true;
        return failure;
    }
    if (agreed_out) *agreed_out = agreed.value_or(0);
    return std::nullopt;
}

const AvdPlane* group_planes(const AvdPlane* planes, bool luma) { return luma ? planes : planes + 1; }

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int device) {
        if (cudaGetDevice(&prev) == cudaSuccess && prev != device) cudaSetDevice(device);
        else prev = -1;
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" {

AvdStatus avd_engine_create(const AvdEngineSpec* spec, const AvdTuning* tuning, AvdEngine** out) {
    if (!spec || !out) return AVD_ERR_NULL_ARG;
    const bool exact_all = tuning != nullptr && tuning->deterministic != 0;
    avd::TuneOptions tune;
    if (tuning) {
        if (tuning->mode > AVD_TUNING_OFF) return fail_global(AVD_ERR_INVALID_OPTIONS, "unknown tuning mode");
        tune.mode = static_cast<avd::TuneMode>(tuning->mode);
        if (tuning->store) tune.store = tuning->store;
    }
    *out = nullptr;
    g_last_error.clear();
    std::string message;
    AvdStatus st = avd::validate_spec(*spec, &message);
    if (st != AVD_OK) return fail_global(st, message);

    auto engine = std::make_unique<AvdEngine>();
    engine->geometry = spec->geometry;
    cudaError_t dev_err = cudaGetDevice(&engine->device);
    if (dev_err != cudaSuccess) return fail_global(AVD_ERR_GPU, avd::cuda_message("cudaGetDevice", dev_err));
    const AvdGeometry& g = spec->geometry;
    const bool nl4d = spec->kind == AVD_ENGINE_NL4D;
    const bool colour_frames = g.chroma != AVD_CHROMA_GRAY;
    if (spec->has_luma) {
        auto f = nl4d ? avd::create_nl4d_pass(spec->nl4d_luma, avd::Channels::Luma, g.width, g.height, g.input,
                                              g.output, colour_frames, &engine->luma)
                      : avd::NlmPass::create(spec->nlm_luma, avd::Channels::Luma, g.width, g.height, g.input,
                                             g.output, &engine->luma, false, exact_all, tune);
        if (f) return fail_global(f->status, f->message);
    }
    if (spec->has_chroma) {
        uint32_t cw, ch;
        avd::plane_dims(g, 1, &cw, &ch);
        auto f = nl4d ? avd::create_nl4d_pass(spec->nl4d_chroma, avd::Channels::Chroma, cw, ch, g.input, g.output,
                                              colour_frames, &engine->chroma)
                      : avd::NlmPass::create(spec->nlm_chroma, avd::Channels::Chroma, cw, ch, g.input, g.output,
                                             &engine->chroma, false, exact_all, tune);
        if (f) return fail_global(f->status, f->message);
    }
    if (!engine->luma && engine->chroma) {
        // engine/spec.rs:220-236 (`guide_pass`): a chroma-only run whose chroma pass compensates
        // motion searches luma motion with the chroma pass's settings at the luma plane's size.
        const bool moves = nl4d || (spec->nlm_chroma.motion_compensation.active &&
                                    avd::resolve_nlm_params(spec->nlm_chroma, avd::Channels::Chroma).temporal_radius > 0);
        if (moves) {
            auto f = nl4d ? avd::create_nl4d_pass(spec->nl4d_chroma, avd::Channels::Luma, g.width, g.height, g.input,
                                                  g.output, colour_frames, &engine->luma, true)
                          : avd::NlmPass::create(spec->nlm_chroma, avd::Channels::Luma, g.width, g.height, g.input,
                                                 g.output, &engine->luma, true);
            if (f) return fail_global(f->status, f->message);
            engine->luma_guides = true;
        }
    }
    if (engine->luma && engine->chroma) {
        // engine/spec.rs:350-365: the chroma pass refines the luma pass's motion, mapped through the
        // chroma subsampling.
        const int shift_x = g.chroma == AVD_CHROMA_YUV444 ? 0 : 1;
        const int shift_y = g.chroma == AVD_CHROMA_YUV420 ? 1 : 0;
        auto f = nl4d ? avd::link_nl4d_luma_motion(engine->luma.get(), engine->chroma.get(), shift_x, shift_y)
                      : avd::NlmPass::link(*static_cast<avd::NlmPass*>(engine->luma.get()),
                                           *static_cast<avd::NlmPass*>(engine->chroma.get()), shift_x, shift_y);
        if (f) return fail_global(f->status, f->message);
    }
    if (engine->luma) {
        // engine/spec.rs:426-450 (`pair_model_producer`): with a pass that searches luma motion over a
        // window, camera models fitted on the luma plane with that pass's search, in a ring covering
        // the frames the engine holds, the window and two more.
        if (auto mode = engine->luma->pair_model_mode()) {
            const size_t depth = engine->lead()->max_held_frames() + (2 * static_cast<size_t>(mode->second) + 1) + 2;
            engine->models = std::make_unique<avd::PairModels>();
            if (auto f = engine->models->allocate(g, mode->first, depth)) return fail_global(f->status, f->message);
            if (auto f = engine->luma->attach_models(engine->models.get())) return fail_global(f->status, f->message);
        }
    }
    const bool gray = g.chroma == AVD_CHROMA_GRAY;
    const bool cleans_luma = engine->luma != nullptr && !engine->luma_guides;
    {
        // engine/spec.rs:366-381 (`colour_blocks`) and planar.rs:176-192 (`attach_colour`): frames
        // with chroma whose passes pool colour cells get the block means of both grids, held for the
        // frames the passes hold; the luma pass reads the luma grid, the chroma pass the chroma grid.
        avd::Pass* luma_pass = cleans_luma ? engine->luma.get() : nullptr;
        const bool pools = (luma_pass && luma_pass->measures_colour()) ||
                           (engine->chroma && engine->chroma->measures_colour());
        if (!gray && pools) {
            size_t held = 0;
            for (avd::Pass* p : {engine->luma.get(), engine->chroma.get()})
                if (p) held = std::max(held, p->max_held_frames());
            engine->colour = std::make_unique<avd::ColourMeans>();
            if (auto f = engine->colour->allocate(g, held)) return fail_global(f->status, f->message);
            if (luma_pass)
                if (auto f = luma_pass->measure_colour(engine->colour.get(), true))
                    return fail_global(f->status, f->message);
            if (engine->chroma)
                if (auto f = engine->chroma->measure_colour(engine->colour.get(), false))
                    return fail_global(f->status, f->message);
        }
    }
    if (!gray && cleans_luma != (engine->chroma != nullptr)) {
        // planar.rs:210-220: one slot more than the cleaned pass holds frames.
        engine->passthrough = std::make_unique<avd::PassthroughRing>();
        engine->passthrough_luma = !cleans_luma;
        const size_t index = cleans_luma ? 1 : 0;
        const size_t planes = cleans_luma ? 2 : 1;
        uint32_t w, h;
        avd::plane_dims(g, index, &w, &h);
        uint64_t bytes = avd::plane_bytes(g.input, static_cast<uint64_t>(w) * h);
        if (auto f = engine->passthrough->init(engine->lead()->max_held_frames() + 1, planes, bytes))
            return fail_global(f->status, f->message);
    }
    *out = engine.release();
    return AVD_OK;
}

void avd_engine_destroy(AvdEngine* engine) {
    if (!engine) return;
    DeviceGuard dg(engine->device);
    if (engine->stream) cudaStreamSynchronize(engine->stream);
    delete engine;
}

AvdStatus avd_engine_set_stream(AvdEngine* engine, void* stream) {
    if (!engine) return AVD_ERR_NULL_ARG;
    engine->stream = static_cast<cudaStream_t>(stream);
    if (engine->luma) engine->luma->stream = engine->stream;
    if (engine->chroma) engine->chroma->stream = engine->stream;
    return AVD_OK;
}

AvdStatus avd_engine_push(AvdEngine* e, const AvdPlane* planes, size_t n, size_t* ready) {
    if (!e || !planes || !ready) return AVD_ERR_NULL_ARG;
    DeviceGuard dg(e->device);
    if (e->poisoned) return record(e, AVD_ERR_NEEDS_RESET, avd_status_message(AVD_ERR_NEEDS_RESET));
    if (auto f = check_frame_planes(e->geometry, planes, n, e->geometry.input)) return record(e, f);
    const uint32_t frame = e->lead()->next_frame();
    if (auto f = fit_pair_model(e, planes, frame)) return record(e, f);
    if (auto f = measure_colour(e, planes, frame)) return record(e, f);
    size_t value = 0;
    // The chroma pass on the side stream, forked after everything queued so far and joined back
    // before anything the caller queues next: the luma kernels' tail waves share the GPU with it.
    const bool overlap = e->overlaps_chroma() && e->side.ensure() == cudaSuccess &&
                         cudaEventRecord(e->side.fork, e->stream) == cudaSuccess &&
                         cudaStreamWaitEvent(e->side.stream, e->side.fork, 0) == cudaSuccess;
    if (overlap) e->chroma->stream = e->side.stream;
    auto f = forward(e, &value, [&](avd::Pass* p, bool luma, size_t* v) {
        return p->push(group_planes(planes, luma), v);
    });
    if (overlap) {
        e->chroma->stream = e->stream;
        cudaError_t err = cudaEventRecord(e->side.join, e->side.stream);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(e->stream, e->side.join, 0);
        if (err != cudaSuccess && !f) {
            e->poisoned = true;
            f = Failure{AVD_ERR_GPU, avd::cuda_message("side stream join", err)};
        }
    }
    if (f) return record(e, f);
    if (e->passthrough) {
        const AvdPlane* src = e->passthrough_luma ? planes : planes + 1;
        size_t np = e->passthrough_luma ? 1 : 2;
        cudaError_t err = e->passthrough->store(frame, src, np, e->stream);
        if (err != cudaSuccess) {
            e->poisoned = true;
            return record(e, AVD_ERR_GPU, avd::cuda_message("passthrough store", err));
        }
    }
    *ready = value;
    return record(e, AVD_OK, "");
}

AvdStatus avd_engine_push_context(AvdEngine* e, const AvdPlane* planes, size_t n) {
    if (!e || !planes) return AVD_ERR_NULL_ARG;
    DeviceGuard dg(e->device);
    if (e->poisoned) return record(e, AVD_ERR_NEEDS_RESET, avd_status_message(AVD_ERR_NEEDS_RESET));
    if (auto f = check_frame_planes(e->geometry, planes, n, e->geometry.input)) return record(e, f);
    const uint32_t frame = e->lead()->next_frame();
    if (auto f = fit_pair_model(e, planes, frame)) return record(e, f);
    if (auto f = measure_colour(e, planes, frame)) return record(e, f);
    auto f = forward(e, nullptr, [&](avd::Pass* p, bool luma, size_t* v) {
        *v = 0;
        return p->push_context(group_planes(planes, luma));
    });
    if (f) return record(e, f);
    if (e->passthrough) {
        const AvdPlane* src = e->passthrough_luma ? planes : planes + 1;
        size_t np = e->passthrough_luma ? 1 : 2;
        cudaError_t err = e->passthrough->store(frame, src, np, e->stream);
        if (err != cudaSuccess) {
            e->poisoned = true;
            return record(e, AVD_ERR_GPU, avd::cuda_message("passthrough store", err));
        }
    }
    return record(e, AVD_OK, "");
}

AvdStatus avd_engine_emit_into(AvdEngine* e, const AvdPlane* planes, size_t n) {
    if (!e || !planes) return AVD_ERR_NULL_ARG;
    DeviceGuard dg(e->device);
    if (e->poisoned) return record(e, AVD_ERR_NEEDS_RESET, avd_status_message(AVD_ERR_NEEDS_RESET));
    if (auto f = check_frame_planes(e->geometry, planes, n, e->geometry.output)) return record(e, f);
    auto f = forward(e, nullptr, [&](avd::Pass* p, bool luma, size_t* v) {
        *v = 0;
        return p->emit_into(group_planes(planes, luma));
    });
    if (f) return record(e, f);
    if (e->passthrough) {
        auto frame = e->lead()->emitted_frame();
        const AvdPlane* dst = e->passthrough_luma ? planes : planes + 1;
        size_t np = e->passthrough_luma ? 1 : 2;
        cudaError_t err = e->passthrough->load(frame.value_or(0), dst, np, e->stream);
        if (err != cudaSuccess) {
            e->poisoned = true;
            return record(e, AVD_ERR_GPU, avd::cuda_message("passthrough load", err));
        }
    }
    return record(e, AVD_OK, "");
}

AvdStatus avd_engine_finish(AvdEngine* e, size_t* tail) {
    if (!e || !tail) return AVD_ERR_NULL_ARG;
    DeviceGuard dg(e->device);
    if (e->poisoned) return record(e, AVD_ERR_NEEDS_RESET, avd_status_message(AVD_ERR_NEEDS_RESET));
    size_t value = 0;
    auto f = forward(e, &value, [&](avd::Pass* p, bool, size_t* v) { return p->finish(v); });
    if (f) return record(e, f);
    *tail = value;
    return record(e, AVD_OK, "");
}

AvdStatus avd_engine_reset(AvdEngine* e) {
    if (!e) return AVD_ERR_NULL_ARG;
    if (e->luma) e->luma->reset();
    if (e->chroma) e->chroma->reset();
    if (e->colour) e->colour->clear();
    if (e->models) e->models->reset();
    e->poisoned = false;
    return record(e, AVD_OK, "");
}

AvdStatus avd_engine_models(AvdEngine* e, float* out, uint32_t capacity, uint32_t* depth) {
    if (!e || !depth) return AVD_ERR_NULL_ARG;
    DeviceGuard dg(e->device);
    *depth = e->models ? static_cast<uint32_t>(e->models->depth()) : 0u;
    if (!e->models || !out) return record(e, AVD_OK, "");
    const size_t words = e->models->depth() * avd::kModelWords;
    if (capacity < words) return record(e, AVD_ERR_INVALID_OPTIONS, "camera models: buffer below depth * 5 words");
    cudaError_t err = cudaStreamSynchronize(e->stream);
    if (err == cudaSuccess) err = cudaMemcpy(out, e->models->ring(), words * sizeof(float), cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) return record(e, AVD_ERR_GPU, avd::cuda_message("camera models read", err));
    return record(e, AVD_OK, "");
}

AvdStatus avd_engine_window_span(const AvdEngine* e, AvdWindowSpan* out) {
    if (!e || !out) return AVD_ERR_NULL_ARG;
    *out = e->lead()->window_span();
    return AVD_OK;
}

AvdStatus avd_engine_max_held_frames(const AvdEngine* e, size_t* out) {
    if (!e || !out) return AVD_ERR_NULL_ARG;
    *out = e->lead()->max_held_frames();
    return AVD_OK;
}

AvdStatus avd_engine_timing(AvdEngine* e, AvdPassTimings* out) {
    if (!e || !out) return AVD_ERR_NULL_ARG;
    DeviceGuard dg(e->device);
    std::memset(out, 0, sizeof(*out));
    if (e->luma) {
        out->has_luma = 1;
        out->luma = e->luma->timing();
    }
    if (e->chroma) {
        out->has_chroma = 1;
        out->chroma = e->chroma->timing();
    }
    return AVD_OK;
}

AvdStatus avd_engine_sample_device_time(AvdEngine* e, uint32_t every) {
    if (!e) return AVD_ERR_NULL_ARG;
    if (e->luma) e->luma->sample_device_time(every);
    if (e->chroma) e->chroma->sample_device_time(every);
    return AVD_OK;
}

const char* avd_engine_last_error(const AvdEngine* e) { return e ? e->last_error.c_str() : ""; }

const char* avd_last_error(void) { return g_last_error.c_str(); }

AvdStatus avd_engine_fail_for_test(AvdEngine* e) {
    if (!e) return AVD_ERR_NULL_ARG;
    auto f = e->lead()->fail_for_test();
    return record(e, f);
}

}  // extern "C"

void avd_set_last_error(const std::string& m) { g_last_error = m; }
