// Pieces shared by the engine's passes: the error a call carries out, owned device buffers, the
// per-pass device timer and the interface every plane-group pass implements.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <algorithm>
#include <optional>
#include <string>
#include <utility>
#include <vector>

#include "avd_internal.h"
#include "kernels.h"

namespace avd {

// Error carried out of a call: a status plus its message.
struct Failure {
    AvdStatus status;
    std::string message;
};

struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer() {
        if (ptr) cudaFree(ptr);
    }
    cudaError_t alloc(size_t n) {
        bytes = n;
        return cudaMalloc(&ptr, n ? n : 4);
    }
    template <typename T>
    T* as() const {
        return static_cast<T*>(ptr);
    }
};

inline std::string cuda_message(const char* what, cudaError_t e) {
    return std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
}

inline PlaneFormat plane_format(const AvdSampleFormat& f) {
    PlaneFormat p;
    p.kind = static_cast<int>(f.kind);
    p.samples_per_word = static_cast<int>(samples_per_word(f));
    p.max_value = sample_max_value(f);
    return p;
}

// Timing of one pass: CUDA events around sampled frames (engine/timing.rs:22-70).
struct DeviceTimer {
    uint32_t every = 0;
    uint64_t frame_counter = 0;
    double total = 0.0;
    uint64_t frames = 0;
    uint64_t exact_samples = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
    // The pass's core launches (the NL4D group search and filter) inside sampled frames.
    bool sampling = false;
    double core_total = 0.0;
    uint64_t core_launches = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> core_pending;
    // Pinned host words the sampled frames' exact-finish counts are copied into (one per pending
    // frame, up to kCountSlots between collections).
    static constexpr size_t kCountSlots = 256;
    int* counts = nullptr;
    size_t counted = 0;

    ~DeviceTimer() {
        for (auto* list : {&pending, &core_pending})
            for (auto& p : *list) {
                cudaEventDestroy(p.first);
                cudaEventDestroy(p.second);
            }
        if (counts) cudaFreeHost(counts);
    }
    // Queues a copy of a sampled frame's exact-finish count (after its exact launch, on `s`).
    void note_count(cudaStream_t s, const int* device_count) {
        if (!counts && cudaHostAlloc(reinterpret_cast<void**>(&counts), kCountSlots * sizeof(int),
                                     cudaHostAllocDefault) != cudaSuccess) {
            counts = nullptr;
            return;
        }
        if (counted < kCountSlots &&
            cudaMemcpyAsync(counts + counted, device_count, sizeof(int), cudaMemcpyDeviceToHost, s) == cudaSuccess)
            counted += 1;
    }
    bool begin(cudaStream_t s, cudaEvent_t* start) {
        uint64_t n = frame_counter++;
        sampling = every != 0 && n % every == 0;
        if (!sampling) return false;
        cudaEventCreate(start);
        cudaEventRecord(*start, s);
        return true;
    }
    void end(cudaStream_t s, cudaEvent_t start) {
        cudaEvent_t stop;
        cudaEventCreate(&stop);
        cudaEventRecord(stop, s);
        pending.emplace_back(start, stop);
        sampling = false;
    }
    // Events around one core launch of a sampled frame (no-ops otherwise).
    void core_begin(cudaStream_t s, cudaEvent_t* start) {
        if (!sampling) return;
        cudaEventCreate(start);
        cudaEventRecord(*start, s);
    }
    void core_end(cudaStream_t s, cudaEvent_t start) {
        if (!sampling) return;
        cudaEvent_t stop;
        cudaEventCreate(&stop);
        cudaEventRecord(stop, s);
        core_pending.emplace_back(start, stop);
    }
    AvdEngineTiming collect() {
        for (auto& p : pending) {
            float ms = 0.0f;
            if (cudaEventSynchronize(p.second) == cudaSuccess && cudaEventElapsedTime(&ms, p.first, p.second) == cudaSuccess) {
                total += ms * 1e-3;
                frames += 1;
            }
            cudaEventDestroy(p.first);
            cudaEventDestroy(p.second);
        }
        pending.clear();
        for (auto& p : core_pending) {
            float ms = 0.0f;
            if (cudaEventSynchronize(p.second) == cudaSuccess && cudaEventElapsedTime(&ms, p.first, p.second) == cudaSuccess) {
                core_total += ms * 1e-3;
                core_launches += 1;
            }
            cudaEventDestroy(p.first);
            cudaEventDestroy(p.second);
        }
        core_pending.clear();
        if (counted) {
            cudaDeviceSynchronize();
            for (size_t i = 0; i < counted; ++i) exact_samples += static_cast<uint64_t>(counts[i]);
            counted = 0;
        }
        AvdEngineTiming t;
        t.device_time = total;
        t.frames = frames;
        t.exact_samples = exact_samples;
        t.core_time = core_total;
        t.core_launches = core_launches;
        return t;
    }
};

// ---------------------------------------------------------------------------------------------
// The block means of the newest frames on both 16x16 noise grids (noise/colour.rs:176-330,
// `ColourBlocks`; colour.cu). The engine measures each pushed frame's mean luma, Cb and Cr from all
// three planes before its passes see the frame, so the luma pass reads the chroma of its blocks and
// the chroma pass the luma of its blocks. Stream frame f keeps slot f % slots, tagged with f, so a
// read never returns another frame's means.
class ColourMeans {
   public:
    std::optional<Failure> allocate(const AvdGeometry& g, size_t held_frames);
    std::optional<Failure> queue(const AvdPlane* planes, uint32_t frame, cudaStream_t s);
    // Stream frame `frame`'s means (3 floats per block) on the luma or the chroma grid, or null
    // when its slot holds another frame.
    const float* held(bool luma_grid, uint32_t frame) const;
    void clear();
    // The factor from a normalised sample to the 8-bit scale (colour.rs:338-361).
    float grain_scale() const;

   private:
    AvdGeometry geometry_{};
    size_t slots_ = 0, luma_blocks_ = 0, chroma_blocks_ = 0;
    std::vector<int64_t> tags_;
    DeviceBuffer luma_, chroma_;
};

// The colour parts of one geometry and input format (colour.rs:338-361).
float colour_grain_scale(const AvdSampleFormat& f);
float colour_eight_bit_scale(const AvdSampleFormat& f);

// ---------------------------------------------------------------------------------------------
// The camera models (motion/global/producer.rs `PairModelProducer`, nlmeans/denoiser/seeds.rs
// `ModelSeeds`): one similarity per adjacent pair of pushed luma frames, fitted before the passes
// see the frame, and composed into the predictions the luma motion pass searches from. Stream frame
// f's model (the pair f - 1 -> f) keeps ring slot f % depth; the ring covers the frames the passes
// hold and their window, so a window never reads a slot a newer frame took.
struct PairModelMode {
    int blksize = 16, overlap = 8, search_radius = 4, ceiling = 0, levels = 2;
};

class PairModels {
   public:
    std::optional<Failure> allocate(const AvdGeometry& g, const PairModelMode& mode, size_t depth);
    // producer.rs:327-372 (`push`): fits the pair from stream frame `frame - 1` to `frame` from the
    // luma plane; a frame that does not follow the last one pushed starts a run and writes identity.
    std::optional<Failure> push(const AvdPlane& luma, uint32_t frame, cudaStream_t s);
    void reset() { running_ = false; }
    // seeds.rs:136-160: the prediction of every neighbour of a window of stream frames (positions
    // before `centre` lie behind it), 6 floats each, into `out`.
    std::optional<Failure> compose_window(const uint32_t* window_frames, int count, int centre, float* out,
                                          cudaStream_t s) const;
    // seeds.rs:104-134: the pair's predictions older -> newer (when `older_to_newer` is set) and newer
    // -> older; a pair that does not step one frame predicts no motion.
    std::optional<Failure> compose_pair(uint32_t older, uint32_t newer, float* older_to_newer, float* newer_to_older,
                                        cudaStream_t s) const;
    // Zeroed noise words: a pair search with predictions keeps its seed only on exact ties.
    const float* zero_noise() const { return zero_noise_.as<float>(); }
    const float* ring() const { return models_.as<float>(); }
    size_t depth() const { return depth_; }

   private:
    uint32_t slot(uint32_t frame) const { return static_cast<uint32_t>(frame % depth_); }
    std::optional<Failure> match(bool deep, int older, int newer, cudaStream_t s);

    AvdGeometry geometry_{};
    PairModelMode mode_{};
    size_t depth_ = 0;
    int blocks_x_ = 0, blocks_y_ = 0, mv_stride_ = 0, conf_stride_ = 0;
    bool running_ = false;
    uint32_t run_first_ = 0, run_last_ = 0;
    DeviceBuffer models_, luma_, rows_, high_, pyramid_, field_, sad_, predictions_, seeds_, tm_field_, changes_,
        escalation_, scratch_, zero_noise_;
};

// ---------------------------------------------------------------------------------------------
// A pass over one plane group.
class Pass {
   public:
    virtual ~Pass() = default;
    virtual std::optional<Failure> push(const AvdPlane* planes, size_t* ready) = 0;
    virtual std::optional<Failure> push_context(const AvdPlane* planes) = 0;
    virtual std::optional<Failure> emit_into(const AvdPlane* planes) = 0;
    virtual std::optional<Failure> finish(size_t* tail) = 0;
    virtual void reset() = 0;
    virtual size_t max_held_frames() const = 0;
    virtual AvdWindowSpan window_span() const = 0;
    virtual uint32_t next_frame() const = 0;
    virtual std::optional<uint32_t> emitted_frame() const = 0;
    virtual AvdEngineTiming timing() = 0;
    virtual void sample_device_time(uint32_t every) = 0;
    virtual std::optional<Failure> fail_for_test() = 0;
    // Whether the pass pools its measured grain into colour cells (nl4d/engine.rs:405-411), and the
    // block means it does so with, on the luma or the chroma grid (engine/planar.rs:176-192).
    // engine/spec.rs:426-450 (`pair_model_producer`): the search of a pass that estimates luma
    // motion over a window, which the camera models fit with, and its temporal radius.
    virtual std::optional<std::pair<PairModelMode, int>> pair_model_mode() const { return std::nullopt; }
    // nlmeans/denoiser/seeds.rs:162-208 (`set_shared_motion`): the pass's own searches start from the
    // camera models too (a pass that refines luma motion runs no search and takes none).
    virtual std::optional<Failure> attach_models(const PairModels*) { return std::nullopt; }
    virtual bool measures_colour() const { return false; }
    virtual std::optional<Failure> measure_colour(const ColourMeans*, bool) { return std::nullopt; }
    // Whether the pass reads anything the luma pass of the same push writes (the shared luma
    // motion); a chroma pass that does not may run beside the luma pass on a second stream.
    virtual bool reads_luma() const { return false; }
    cudaStream_t stream = nullptr;
};

// The noise look-ahead of a front that measures the noise (noise_front.cpp).
struct NoiseFrontConfig {
    uint32_t width = 0, height = 0, channels = 1, temporal_radius = 0;
    uint32_t table_radius = 0;  // the NLM offset tables' search radius, 0 for none
    FoldCoefficients coefficients;
    bool motion = false;  // read each frame along the motion to the frame before it
    int blksize = 16, overlap = 8, search_radius = 4, levels = 2;
    float thsad = 0.0f;
    int ceiling = 0;  // the search's escalation ceiling (lookahead.rs:505-515); 0: no escalation
    // Each record carries the luma quarter fields and each reading the noise curve
    // (noise/state.rs:297, `wants_curve`; the NL4D luma noise map).
    bool luma_fields = false;
};

class NoiseFront {
   public:
    static constexpr size_t kFrames = 8;  // nlmeans/denoiser/lookahead.rs:30
    NoiseFront() = default;
    NoiseFront(const NoiseFront&) = delete;
    NoiseFront& operator=(const NoiseFront&) = delete;
    ~NoiseFront();
    std::optional<Failure> allocate(const NoiseFrontConfig& cfg);
    // lookahead.rs:310-316 and seeds.rs:104-134: the look-ahead's pair searches also search around
    // the camera models' pair predictions, keeping their seed only on exact ties.
    std::optional<Failure> attach_models(const PairModels* models);
    // Orders a write into a look-ahead slot on `main` after the reads queued on the side stream.
    std::optional<Failure> before_ingest(cudaStream_t main);
    // The look-ahead slot of stream frame `frame`.
    float* slot(size_t frame) const;
    size_t held() const { return pushed_ - released_; }
    size_t pushed() const { return pushed_; }
    // Reads stream frame pushed(), which the caller has just ingested into slot(pushed()) on `main`.
    // The reads run on the front's own high-priority stream, overlapping the pass's work on `main`.
    std::optional<Failure> read_pushed(cudaStream_t main);
    // The oldest held stream frame, now released, or none when nothing is held.
    std::optional<size_t> take_oldest();
    // Folds the window around stream frame `centre` into the derived words and tables, on `main`
    // after the reads.
    std::optional<Failure> fold(uint32_t centre, cudaStream_t main);
    float* derived() const { return derived_.as<float>(); }
    // The stream state's 16 curve ratios (noise/fold.rs:47-72), read while the curve flag is set.
    const float* curve_ratios() const { return state_.as<float>() + 16; }
    float* spatial_table() const { return spatial_.as<float>(); }
    float* pilot_table() const { return pilot_.as<float>(); }
    // Pools each reading's blocks into colour cells with the block means `means` holds (on the luma
    // grid with `luma_grid`) and fits the grain model at each fold (noise/colour.rs:733-827).
    std::optional<Failure> measure_colour(const ColourMeans* means, bool luma_grid);
    // The last fold's log gain tables, 976 per channel, or null without colour.
    const float* colour_gains() const { return colour_ ? colour_gains_.as<float>() : nullptr; }
    void reset();

   private:
    std::optional<Failure> search(size_t centre_frame, size_t neighbour_frame, int direction, cudaStream_t s);
    std::optional<Failure> read_against(size_t frame, std::optional<size_t> prev, int direction, cudaStream_t s);
    NoiseFrontConfig cfg_;
    cudaStream_t side_ = nullptr;
    cudaEvent_t ingested_ = nullptr, read_done_ = nullptr, snapshot_ = nullptr;
    // One event per history slot, recorded after the reads of the frame in it, so a fold waits only
    // for the frames of its window and the newest reads overlap the passes.
    std::vector<cudaEvent_t> frame_read_;
    bool reads_queued_ = false, snapshot_pending_ = false;
    // The derived words the look-ahead's searches read: a copy taken as each push's reads start, so
    // they read the previous push's fold whatever the pass's fold on the main stream writes meanwhile.
    DeviceBuffer search_words_;
    const PairModels* models_ = nullptr;
    DeviceBuffer pair_predictions_;  // older -> newer, then newer -> older, 6 floats each
    size_t capacity_ = 0, pushed_ = 0, released_ = 0, recorded_ = 0;
    int step_ = 8, blocks_x_ = 1, blocks_y_ = 1, mv_stride_ = 2, conf_stride_ = 1;
    DeviceBuffer lookahead_, partials_, records_, scratch_, history_records_, history_results_, settings_, state_,
        derived_, spatial_, pilot_, pyramid_, pair_, escalation_;
    const ColourMeans* colour_ = nullptr;
    bool colour_luma_ = true;
    size_t colour_words_ = 0;  // int32 words of one frame's cell sums
    DeviceBuffer colour_cells_, colour_window_, colour_scratch_, colour_table_, colour_gains_;
};

// NL4D pass over one plane group (nl4d_pass.cpp).
// `colour_frames` is set for frames with chroma planes, whose measured passes scale their thresholds
// by the colour grain gains (noise/colour.rs:204-286). With `guides_only` the pass is a chroma-only
// engine's luma guide: it runs the motion machinery on the luma plane for the chroma pass to read,
// and no filter (engine/spec.rs:220-236).
std::optional<Failure> create_nl4d_pass(const AvdNl4dOptions& options, Channels channels, uint32_t width,
                                        uint32_t height, const AvdSampleFormat& in, const AvdSampleFormat& out,
                                        bool colour_frames, std::unique_ptr<Pass>* result,
                                        bool guides_only = false);

// The luma pass's window motion mapped onto the chroma pass's block grid, shared by the two passes
// of one engine (motion/luma_ring.rs, motion/chroma_map.rs): one slot of 2d chroma fields per
// window, keyed by the window's centre stream frame. The chroma pass allocates it at link time with
// its own block grid; the luma pass writes it after each window search and the chroma pass refines
// the mapped vectors instead of searching its own.
struct LumaMotionShare {
    DeviceBuffer fields;
    std::vector<int64_t> tags;  // the stream frame each slot holds, -1 for none
    int slots = 0, neighbours = 0, blocks_x = 1, blocks_y = 1, step = 8, blksize = 16, mv_stride = 2;
    int shift_x = 0, shift_y = 0;
    int32_t* slot_ptr(int slot) const { return fields.as<int32_t>() + static_cast<int64_t>(slot) * neighbours * mv_stride; }
    void clear() { std::fill(tags.begin(), tags.end(), -1); }
};

// Links an NL4D engine's luma and chroma passes: the chroma pass reads the luma pass's mapped
// window motion (engine/spec.rs:350-365 `luma_motion_ring`, nlmeans/denoiser/seeds.rs:168-208).
// `shift_x`/`shift_y` are the chroma subsampling as powers of two.
std::optional<Failure> link_nl4d_luma_motion(Pass* luma, Pass* chroma, int shift_x, int shift_y);

}  // namespace avd
