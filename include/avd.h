/*
 * avd.h - C ABI of the B200 denoising engine (NLMeans, NLMeans-HQ, NL4D and the noise estimator).
 *
 * Every entry point mirrors one item of av-denoise-core's public Rust API. The citation beside each
 * names the reference interface it replaces, by its path inside the av-denoise project.
 *
 * Conventions
 *  - Plain C types only: pointers, sizes and PODs. Device buffers are raw CUDA device addresses
 *    (`uint64_t`), borrowed for the duration of one call, exactly like the reference's
 *    `DevicePlane<'a>` (av-denoise-core/src/engine/plane.rs:54-86).
 *  - `Option<T>` fields become a `has_x` flag plus the value.
 *  - Every call returns an `AvdStatus`; statuses map 1:1 onto `Error`
 *    (av-denoise-core/src/error.rs:3-19), plus `AVD_ERR_NULL_ARG` for a null pointer argument.
 *  - A failed state-changing call poisons the engine until `avd_engine_reset`, exactly as the
 *    reference engine does (av-denoise-core/src/engine/mod.rs:167).
 *  - An engine is `Send` but not `Sync`: one thread at a time may call into one engine.
 */
#ifndef AVD_H
#define AVD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AVD_ABI_VERSION 6u

#if defined(__GNUC__)
#define AVD_API __attribute__((visibility("default")))
#else
#define AVD_API
#endif

/* ---- status -------------------------------------------------------------------------------- */

/* av-denoise-core/src/error.rs:3-19 (`Error` variants, same order). */
typedef enum AvdStatus {
    AVD_OK = 0,
    AVD_ERR_INVALID_OPTIONS = 1,
    AVD_ERR_INVALID_GEOMETRY = 2,
    AVD_ERR_PLANE_MISMATCH = 3,
    AVD_ERR_OUTPUTS_PENDING = 4,
    AVD_ERR_NOTHING_TO_EMIT = 5,
    AVD_ERR_CONTEXT_AFTER_PUSH = 6,
    AVD_ERR_NEEDS_RESET = 7,
    AVD_ERR_GPU = 8, /* Error::Gpu: any CUDA failure, which poisons the engine */
    AVD_ERR_NULL_ARG = 9,
    /* av-denoise/src/host/mod.rs:37-57 (`DenoiserError`) for the host denoiser below: */
    AVD_ERR_QUEUE_FULL = 10, /* QueueFull: MAX_PENDING frames wait to be collected; not poisoning */
    AVD_ERR_POISONED = 11    /* Poisoned: an earlier call failed; reset the stream */
} AvdStatus;

/* ---- geometry ------------------------------------------------------------------------------ */

/* av-denoise-core/src/engine/plane.rs:8-17 (`SampleFormat`). */
typedef enum AvdSampleKind { AVD_SAMPLE_U8 = 0, AVD_SAMPLE_U16 = 1, AVD_SAMPLE_F32 = 2 } AvdSampleKind;

typedef struct AvdSampleFormat {
    uint32_t kind;  /* AvdSampleKind */
    uint32_t depth; /* significant bits for AVD_SAMPLE_U16, in 9..=16; ignored otherwise */
} AvdSampleFormat;

/* av-denoise-core/src/engine/frame.rs:10-20 (`ChromaLayout`). */
typedef enum AvdChromaLayout {
    AVD_CHROMA_GRAY = 0,
    AVD_CHROMA_YUV420 = 1,
    AVD_CHROMA_YUV422 = 2,
    AVD_CHROMA_YUV444 = 3
} AvdChromaLayout;

/* av-denoise-core/src/engine/frame.rs:54-66 (`ChromaSiting`): carried, never changes output. */
typedef enum AvdChromaSiting {
    AVD_SITING_LEFT = 0,
    AVD_SITING_CENTER = 1,
    AVD_SITING_TOP_LEFT = 2,
    AVD_SITING_UNKNOWN = 3
} AvdChromaSiting;

/* av-denoise-core/src/engine/frame.rs:73-81 (`Geometry`). */
typedef struct AvdGeometry {
    uint32_t width;
    uint32_t height;
    uint32_t chroma; /* AvdChromaLayout */
    uint32_t chroma_siting; /* AvdChromaSiting */
    AvdSampleFormat input;
    AvdSampleFormat output;
} AvdGeometry;

/* av-denoise-core/src/engine/plane.rs:54-86 (`DevicePlane`): a packed plane, stride = width,
 * `bytes` >= SampleFormat::plane_bytes(width * height) (whole 32-bit words). */
typedef struct AvdPlane {
    uint64_t ptr; /* CUDA device address */
    uint64_t bytes;
    uint32_t width;
    uint32_t height;
} AvdPlane;

/* ---- NLMeans options ----------------------------------------------------------------------- */

/* av-denoise-core/src/options.rs:151-165 (`Preset`). */
typedef enum AvdPreset {
    AVD_PRESET_VERYFAST = 0,
    AVD_PRESET_FAST = 1,
    AVD_PRESET_BASE = 2,
    AVD_PRESET_SLOW = 3,
    AVD_PRESET_VERYSLOW = 4
} AvdPreset;

/* av-denoise-core/src/nlmeans/prefilter/mod.rs:15-26 (`PrefilterMode`). */
typedef enum AvdPrefilterKind {
    AVD_PREFILTER_NONE = 0,
    AVD_PREFILTER_BILATERAL = 1,
    AVD_PREFILTER_NLM_SPATIAL = 2
} AvdPrefilterKind;

typedef struct AvdPrefilter {
    uint32_t kind; /* AvdPrefilterKind */
    float sigma_s; /* Bilateral */
    float sigma_r; /* Bilateral */
    float strength_scale; /* NlmSpatial */
} AvdPrefilter;

/* av-denoise-core/src/motion/search.rs:94-113 (`MotionEstimation`). */
typedef enum AvdEstimationKind {
    AVD_ESTIMATION_AUTO = 0,
    AVD_ESTIMATION_DIRECT = 1,
    AVD_ESTIMATION_CHAINED = 2
} AvdEstimationKind;

/* av-denoise-core/src/motion/search.rs:5-53 (`MotionSearch`), also the payload of
 * `MotionCompensationMode::Mvtools` (search.rs:58-89). */
typedef struct AvdMotionSearch {
    uint32_t blksize;
    uint32_t overlap;
    uint32_t search_radius;
    uint32_t max_search_escalation;
    uint32_t pyramid_levels;
    uint32_t estimation; /* AvdEstimationKind */
    uint32_t refine_radius; /* Chained only */
} AvdMotionSearch;

/* av-denoise-core/src/motion/search.rs:58-89 (`MotionCompensationMode`). */
typedef struct AvdMotionCompensation {
    uint32_t active; /* 0 = None, 1 = Mvtools { search } */
    AvdMotionSearch search;
} AvdMotionCompensation;

/* av-denoise-core/src/nlmeans/options.rs:94-101 (`NlmTuning`). */
typedef struct AvdNlmTuning {
    uint32_t has_search_radius;
    uint32_t search_radius;
    uint32_t has_patch_radius;
    uint32_t patch_radius;
    uint32_t has_strength;
    float strength;
    uint32_t has_self_weight;
    float self_weight;
} AvdNlmTuning;

/* av-denoise-core/src/nlmeans/options.rs:84-92 (`DenoisingMode`). */
typedef struct AvdDenoisingMode {
    uint32_t temporal; /* 0 = Spacial, 1 = Temporal { radius } */
    uint32_t radius;
} AvdDenoisingMode;

/* av-denoise-core/src/nlmeans/params.rs:113-158 (`HqParams`). */
typedef struct AvdHqParams {
    uint32_t auto_strength;
    uint32_t noise_floor;
    uint32_t has_sigma_override;
    float sigma_override;
    uint32_t temporal_confidence;
    float thsad_scale;
    float sigma_scale;
} AvdHqParams;

/* av-denoise-core/src/nlmeans/options.rs:4-46 (`NlmeansOptions`, `NlmeansHqOptions`,
 * `NlmeansAlgorithm`). `variant` 0 = Fast(options), 1 = Hq(options + hq). */
typedef struct AvdNlmeansAlgorithm {
    uint32_t variant;
    AvdPrefilter prefilter;
    AvdMotionCompensation motion_compensation;
    AvdNlmTuning tuning;
    AvdDenoisingMode mode;
    AvdHqParams hq;
} AvdNlmeansAlgorithm;

/* ---- NL4D options -------------------------------------------------------------------------- */

/* av-denoise-core/src/nl4d/options.rs:11-92 (`Nl4dOptions`). */
typedef struct AvdNl4dOptions {
    AvdMotionSearch motion;
    uint32_t has_sigma;
    float sigma;
    float sigma_scale;
    float thsad_scale;
    uint32_t refine;
    uint32_t spatial_radius;
    uint32_t has_lambda_ht;
    float lambda_ht;
    float lambda_ht_scale;
    float c_min;
    float kaiser_beta;
    float field_lambda;
    uint32_t noise_map;
    uint32_t pooled_threshold;
    uint32_t grain_data; /* accepted and validated; AV1 grain measurement is not built */
    uint32_t temporal_radius;
    /* Nonzero adds the empirical Wiener stage after the threshold (an extension the reference does
     * not have; off by default, which is the reference's filter). */
    uint32_t wiener;
} AvdNl4dOptions;

/* ---- engine spec --------------------------------------------------------------------------- */

/* av-denoise-core/src/engine/spec.rs:146-157 (`EngineSpec`). */
typedef enum AvdEngineKind { AVD_ENGINE_NLMEANS = 0, AVD_ENGINE_NL4D = 1 } AvdEngineKind;

typedef struct AvdEngineSpec {
    uint32_t kind; /* AvdEngineKind */
    uint32_t has_luma;
    uint32_t has_chroma;
    AvdNlmeansAlgorithm nlm_luma; /* kind == NLMEANS */
    AvdNlmeansAlgorithm nlm_chroma;
    AvdNl4dOptions nl4d_luma; /* kind == NL4D */
    AvdNl4dOptions nl4d_chroma;
    AvdGeometry geometry;
} AvdEngineSpec;

/* av-denoise-core/src/tune/config.rs:8-75 (`TuningMode`, `TuningConfig`). `deterministic` ("picks
 * only bit-identical candidates and the baseline profile"): every NLMeans sample is computed by the
 * exact kernel in the operation order of the reference's baseline (direct row-major patch sums), so
 * float outputs too are bit-identical to the CPU restatement; slower. Off (the default), integer
 * outputs still match it: the fast window kernel flags the samples near a change of code and the
 * exact kernel recomputes only those. The NLM pilot prefilter's reference always runs exactly.
 *
 * `mode` picks each launch site's variant (same results, different launch shapes) per frame shape:
 * AUTO (the default) uses the remembered or stored choice and times every variant once on the
 * site's first launch for a shape without one; CACHED uses stored choices only, else the baseline;
 * OFF runs every baseline. `store` is the directory of the results file
 * (`av-denoise-b200-tune.jsonl`, one JSON object per device and shape); null keeps results for
 * this process only. A null AvdTuning means all defaults. */
typedef enum AvdTuningMode { AVD_TUNING_AUTO = 0, AVD_TUNING_CACHED = 1, AVD_TUNING_OFF = 2 } AvdTuningMode;
typedef struct AvdTuning {
    uint32_t deterministic;
    uint32_t mode;     /* AvdTuningMode */
    const char* store; /* directory of the per-shape results, or null */
} AvdTuning;

/* The tuner's choice for one launch-site key among `variants` under AvdTuning's `mode` and `store`,
 * with variant v timed as `times_ms[v]` instead of a launch (tune/store.rs, driver/mod.rs): the
 * store's tests drive it without a GPU. avd_tune_forget drops the results this process remembers. */
AVD_API int avd_tune_variant_for_test(uint32_t mode, const char* store, const char* key, uint32_t variants,
                                      const float* times_ms);
AVD_API void avd_tune_forget(void);

/* av-denoise-core/src/engine/mod.rs:40-62 (`WindowSpan`, `EdgePadding`). */
typedef struct AvdWindowSpan {
    uint64_t behind;
    uint64_t ahead;
    uint32_t edges; /* 0 = Repeat, 1 = Shifted */
    uint32_t reserved;
} AvdWindowSpan;

/* av-denoise-core/src/engine/timing.rs (`EngineTiming`) and engine/mod.rs:113-120
 * (`PassTimings`). Times in seconds of device time, gathered while sampling is on. */
typedef struct AvdEngineTiming {
    double device_time;
    uint64_t frames;
    /* No field in the reference: over the same sampled frames, the samples (pixels) the exact finish
     * recomputed in the reference kernels' order (NLMeans with integer outputs; 0 otherwise). */
    uint64_t exact_samples;
    /* No field in the reference: over the same sampled frames, the device time of the pass's core
     * launches (NL4D: the group search and the group filter) and how many there were. */
    double core_time;
    uint64_t core_launches;
} AvdEngineTiming;

typedef struct AvdPassTimings {
    uint32_t has_luma;
    uint32_t has_chroma;
    AvdEngineTiming luma;
    AvdEngineTiming chroma;
} AvdPassTimings;

typedef struct AvdEngine AvdEngine;

/* ---- library-level helpers (host only, no GPU) ----------------------------------------------- */

/* ABI version of the loaded library. */
AVD_API uint32_t avd_abi_version(void);

/* The message of the calling thread's last failed call that has no engine to keep it
 * (`avd_engine_create`, `avd_spec_validate`); empty after a success. */
AVD_API const char* avd_last_error(void);

/* av-denoise-core/src/error.rs:3-19: the fixed text of a status. */
AVD_API const char* avd_status_message(AvdStatus status);

/* Default-filled option structs, matching the reference's `Default` impls:
 * nlmeans/options.rs:5-29 + params.rs:147-158 (NLMeans), nl4d/options.rs:68-92 (NL4D),
 * motion/search.rs:33-44 (MotionSearch), engine/frame.rs:73-81 (Geometry, caller sets sizes). */
AVD_API void avd_default_nlmeans(AvdNlmeansAlgorithm* out);
AVD_API void avd_default_nl4d(AvdNl4dOptions* out);
AVD_API void avd_default_motion_search(AvdMotionSearch* out);

/* Presets: av-denoise-core/src/nlmeans/options.rs:58-82 and options.rs:170-175.
 * `avd_nlmeans_variant_for` returns 0 = Fast, 1 = Hq. `avd_search_escalation_for` returns 0 for
 * `None`. */
AVD_API uint32_t avd_nlmeans_variant_for(uint32_t preset);
AVD_API uint32_t avd_nlmeans_temporal_radius_for(uint32_t preset);
AVD_API uint32_t avd_nlmeans_search_radius_for(uint32_t preset);
AVD_API uint32_t avd_search_escalation_for(uint32_t preset);

/* av-denoise-core/src/nlmeans/params.rs:27-33 (`hq_default_strength`); channels 1 = luma,
 * 2 = chroma. */
AVD_API float avd_hq_default_strength(uint32_t channels, uint32_t temporal_radius);

/* av-denoise-core/src/engine/spec.rs:291-345 (`EngineSpec::validate`) plus the per-pass
 * parameter checks the reference runs at build time (nlmeans/params.rs:276-428,
 * nl4d/params.rs:119-197, nl4d/options.rs:127-185). Writes the message of a failure into `msg`
 * (may be NULL). Runs on the host only. */
AVD_API AvdStatus avd_spec_validate(const AvdEngineSpec* spec, char* msg, size_t msg_len);

/* av-denoise-core/src/engine/spec.rs:260-281 (`EngineSpec::max_held_frames`,
 * `EngineSpec::window_span`) for a spec, without building an engine. */
AVD_API AvdStatus avd_spec_window_span(const AvdEngineSpec* spec, AvdWindowSpan* out);

/* ---- engine -------------------------------------------------------------------------------- */

/* av-denoise-core/src/tune/setup.rs:79-91 (`build_engine`). Validates first, touching no GPU
 * state on failure. `tuning` may be NULL. The engine runs on the current CUDA device. */
AVD_API AvdStatus avd_engine_create(const AvdEngineSpec* spec, const AvdTuning* tuning, AvdEngine** out);

AVD_API void avd_engine_destroy(AvdEngine* engine);

/* Sets the CUDA stream (`cudaStream_t`) every later call queues its work on; 0 = legacy default.
 * The reference's equivalent is the CubeCL client's queue. */
AVD_API AvdStatus avd_engine_set_stream(AvdEngine* engine, void* stream);

/* av-denoise-core/src/engine/mod.rs:170 (`Engine::push`). `planes` holds every plane of the
 * frame, luma first; `*ready` receives how many frames are ready to emit (0 or 1). */
AVD_API AvdStatus avd_engine_push(AvdEngine* engine, const AvdPlane* planes, size_t n_planes, size_t* ready);

/* av-denoise-core/src/engine/mod.rs:185 (`Engine::push_context`). */
AVD_API AvdStatus avd_engine_push_context(AvdEngine* engine, const AvdPlane* planes, size_t n_planes);

/* av-denoise-core/src/engine/mod.rs:188 (`Engine::emit_into`). */
AVD_API AvdStatus avd_engine_emit_into(AvdEngine* engine, const AvdPlane* planes, size_t n_planes);

/* av-denoise-core/src/engine/mod.rs:191 (`Engine::finish`). */
AVD_API AvdStatus avd_engine_finish(AvdEngine* engine, size_t* tail);

/* av-denoise-core/src/engine/mod.rs:194 (`Engine::reset`). */
AVD_API AvdStatus avd_engine_reset(AvdEngine* engine);

/* av-denoise-core/src/engine/mod.rs:196 (`Engine::window_span`). */
AVD_API AvdStatus avd_engine_window_span(const AvdEngine* engine, AvdWindowSpan* out);

/* av-denoise-core/src/engine/mod.rs:199 (`Engine::max_held_frames`). */
AVD_API AvdStatus avd_engine_max_held_frames(const AvdEngine* engine, size_t* out);

/* av-denoise-core/src/engine/mod.rs:207 (`Engine::timing`). */
AVD_API AvdStatus avd_engine_timing(AvdEngine* engine, AvdPassTimings* out);

/* av-denoise-core/src/engine/mod.rs:210 (`Engine::sample_device_time`). */
AVD_API AvdStatus avd_engine_sample_device_time(AvdEngine* engine, uint32_t every);

/* The message of the engine's last failed call (empty when none). */
AVD_API const char* avd_engine_last_error(const AvdEngine* engine);

/* Test hook mirroring `fail_through_guard_for_test` (av-denoise-core/src/nlmeans/engine.rs:194-199):
 * forces a GPU-class failure through the poison guard, with no GPU work. */
AVD_API AvdStatus avd_engine_fail_for_test(AvdEngine* engine);

/* ---- host denoiser ------------------------------------------------------------------------ */

/* av-denoise/src/host/mod.rs:111-420 (`HostDenoiser`): an engine fed from host memory. Frames go
 * in as wire planes (width x height samples: 1 byte for U8, 2 little-endian bytes for U16, 4 for
 * F32, each plane at its own size), are staged in pinned memory and uploaded on a copy stream that
 * overlaps the engine's stream; denoised frames are read back on a third stream into pinned
 * memory, at most MAX_PENDING = 2 in flight (mod.rs:27-33). The denoiser owns its streams and
 * buffers. */
typedef struct AvdHost AvdHost;

/* `HostDenoiser::create` without the accelerator choice: the CUDA device current at the call. */
AVD_API AvdStatus avd_host_create(const AvdEngineSpec* spec, const AvdTuning* tuning, AvdHost** out);
AVD_API void avd_host_destroy(AvdHost* host);

/* The wire byte length of plane `index` (`plane_lengths`, mod.rs:124). */
AVD_API uint64_t avd_host_plane_bytes(const AvdHost* host, size_t index);

/* mod.rs:256-290 (`push`): uploads one frame and starts denoising every frame it completes.
 * AVD_ERR_QUEUE_FULL once 2 frames wait in flight (the call changes nothing); a rejected plane
 * (AVD_ERR_PLANE_MISMATCH) leaves the denoiser usable; any other failure poisons it. */
AVD_API AvdStatus avd_host_push(AvdHost* host, const void* const* planes, const uint64_t* bytes, size_t n);

/* mod.rs:302-322 (`push_priming`): uploads one frame as context only. */
AVD_API AvdStatus avd_host_push_priming(AvdHost* host, const void* const* planes, const uint64_t* bytes, size_t n);

/* mod.rs:324-343 (`recv`): blocks until the oldest frame in flight lands and copies its planes into
 * `out` (avd_host_plane_bytes each); `*got` is 0 when nothing was in flight. */
AVD_API AvdStatus avd_host_recv(AvdHost* host, void* const* out, size_t n, int* got);

/* mod.rs:345-373 (`flush`): drains the frames in flight and the temporal tail, handing each to
 * `sink` in order; the denoiser is ready for a fresh stream afterwards. */
typedef void (*AvdHostSink)(void* user, const void* const* planes, size_t n);
AVD_API AvdStatus avd_host_flush(AvdHost* host, AvdHostSink sink, void* user);

/* mod.rs:375-381 (`reset_stream`): drops the frames in flight and clears any poison. */
AVD_API void avd_host_reset(AvdHost* host);

/* The message of the host denoiser's last failed call; with a null host, of the last failed create. */
AVD_API const char* avd_host_last_error(const AvdHost* host);

/* av-denoise/src/host/timing.rs:20-56 (`PlanarTiming`): where the denoiser's time went since it
 * was built. `blocked` is host time waiting for readbacks to land, `submit` the rest of the time
 * spent inside its calls (the flush sink's time excluded); each denoised plane group's device time
 * is scaled from its sampled frames to every emitted frame, or -1 when nothing was sampled. */
typedef struct AvdHostTiming {
    double blocked;
    double submit;
    uint64_t frames;
    uint32_t has_luma;
    uint32_t has_chroma;
    double luma_device_busy;
    double chroma_device_busy;
} AvdHostTiming;

/* mod.rs:383-398 (`timing`; waits for device spans in flight) and `sample_device_time`. */
AVD_API AvdStatus avd_host_timing(AvdHost* host, AvdHostTiming* out);
AVD_API void avd_host_sample_device_time(AvdHost* host, uint32_t every);

/* Marks the stream failed, as a failure inside a call would, so that tests can exercise the
 * Poisoned path without a device fault (av-denoise/src/host/mod.rs:392-395, `poison_for_test`). */
AVD_API void avd_host_poison_for_test(AvdHost* host);

/* ---- NL4D kernel-level entry points ------------------------------------------------------- */

/* The arguments of one NL4D collaborative-filter pass over device buffers, as the reference's
 * `collab_fused` launch takes them (av-denoise-core/src/collab/kernels/fused/mod.rs:170-234). */
typedef struct AvdCollabPass {
    uint64_t ring;            /* f32 frames, `slots` x height x width x channels, interleaved */
    uint64_t mv_field;        /* i32 (dx, dy) per motion block per neighbour, `mv_stride` apart */
    uint64_t confidence;      /* f32 per motion block per neighbour, `conf_stride` apart */
    uint64_t neighbour_slots; /* u32 ring slot of each neighbour index */
    uint64_t noise;           /* f32 derived words */
    uint64_t noise_curve;     /* 16 f32 luma curve ratios */
    uint64_t dct_profile;     /* 8 f32 per-frequency variance multipliers */
    uint64_t kaiser;          /* 8 f32 aggregation taps */
    uint64_t accum;           /* i32, slots x height x width x channels, accumulated into */
    uint64_t wsum;            /* i32, slots x height x width, accumulated into */
    uint64_t group_weight;    /* f32 per reference patch, written */
    uint64_t members;         /* scratch of avd_collab_member_bytes(width, height) bytes */
    uint32_t width, height, channels, centre_slot;
    uint32_t sigma_word, weight_scale_word, curve_valid_word; /* indices into `noise` */
    uint32_t radius, refine, spatial_radius, k_max;
    uint32_t mv_stride, conf_stride, blk_step, blksize, blocks_x, blocks_y;
    uint32_t pooled;
    float c_min, lambda_ht, accum_scale, pool_ratio;
    /* Nonzero adds the empirical Wiener stage after the threshold: each kept coefficient z of noise
     * variance v is scaled by z^2 / (z^2 + v) and the group weight counts g^2 v. An extension: the
     * reference's filter stops at the threshold (fused/mod.rs:112-134). */
    uint32_t wiener;
} AvdCollabPass;

/* The gradients of one pass's adjoint. A and W are the accumulators in real units
 * (accum / accum_scale and wsum / (5 accum_scale)); the normalised frame is A / W. */
typedef struct AvdCollabAdjoint {
    uint64_t grad_accum;      /* f32 dL/dA, laid out as `accum` */
    uint64_t grad_wsum;       /* f32 dL/dW, laid out as `wsum` */
    uint64_t grad_ring;       /* f32 dL/d(ring), laid out as `ring`, added into */
    uint64_t grad_sigma_refs; /* f32 per reference patch and channel, its share of dL/d(sigma_c), written */
} AvdCollabAdjoint;

/* av-denoise-core/src/collab/kernels/fused/mod.rs:170 (`collab_fused`): one pass, queued on
 * `stream`. Adds into `accum`/`wsum` (integer adds: the result does not depend on scheduling). */
AVD_API AvdStatus avd_collab_pass(const AvdCollabPass* pass, void* stream);

/* The scratch bytes one collab pass over a width x height plane needs between its group search
 * and its filter (the reference's split search profile hands the same member words over,
 * av-denoise-core/src/collab/kernels/fused/split.rs). */
AVD_API uint64_t avd_collab_member_bytes(uint32_t width, uint32_t height);

/* Reference patches of one pass over a width x height plane (the rows of `grad_sigma_refs`). */
AVD_API uint64_t avd_collab_refs(uint32_t width, uint32_t height);

/* The adjoint of the pass `pass` describes, queued on `stream` after that pass (it reads the
 * member words the pass's search left in `members`). Holds the groups and every keep decision
 * fixed and reads the pass as A and W above: adds dL/d(ring) and writes each reference patch's
 * share of dL/d(sigma) (sigma from the `noise` words; the weight-scale word read as proportional to
 * sigma_0^2, as the engine derives it). An extension with no counterpart in the reference. */
AVD_API AvdStatus avd_collab_adjoint(const AvdCollabPass* pass, const AvdCollabAdjoint* adjoint, void* stream);

/* av-denoise-core/src/collab/kernels/transforms.rs:196-221 (`dct_noise_profile`). */
AVD_API void avd_dct_noise_profile(float rho, float* out8);

/* av-denoise-core/src/collab/kernels/aggregate.rs:114-132 (`kaiser_window`). */
AVD_API void avd_kaiser_window(float beta, float* out8);

/* av-denoise-core/src/collab/kernels/aggregate.rs:33-54 (`cross_frame_accum_scale`). */
AVD_API float avd_cross_frame_accum_scale(uint32_t spatial_radius, uint32_t temporal_radius);

/* ---- motion search kernel-level entry points ---------------------------------------------- */

/* The floats a luma pyramid of `levels` levels over `frame_count` slots holds
 * (av-denoise-core/src/motion/pyramid.rs:16-20, `pyramid_pixels_per_frame` x frames). */
AVD_API uint64_t avd_motion_pyramid_floats(uint32_t width, uint32_t height, uint32_t frame_count, uint32_t levels);

/* av-denoise-core/src/motion/pyramid.rs:82-107 (`run_pyramid_build`): lane 0 of ring slot
 * `ring_slot` (f32, `channels` interleaved) becomes level 0 of pyramid slot `pyramid_slot`, and each
 * further level averages 2x2 pixels of the one below. Queued on `stream`. */
AVD_API AvdStatus avd_motion_pyramid_build(uint64_t ring, uint32_t channels, uint32_t width, uint32_t height,
                                           uint32_t frame_count, uint32_t ring_slot, uint32_t levels,
                                           uint64_t pyramid, uint32_t pyramid_slot, void* stream);

/* One block-matching motion search over a built pyramid, as `run_analyse` runs it before its
 * truemotion stage (av-denoise-core/src/motion/analyse.rs:170-266), and as `run_confidence` runs it
 * with `search_radius` 0 and one level (motion/confidence.rs:39-66). */
typedef struct AvdMotionPass {
    uint64_t pyramid;         /* f32, avd_motion_pyramid_floats(width, height, frame_count, levels) */
    uint64_t neighbour_slots; /* u32 pyramid slot of each neighbour */
    uint64_t mv_field;        /* i32 (dx, dy) per block per neighbour, `mv_stride` apart; written */
    uint64_t confidence;      /* f32 per block per neighbour, `conf_stride` apart; 0 = not written */
    uint64_t noise;           /* f32 words; the SAD floor is word `sad_floor_word` */
    uint32_t width, height, frame_count, centre_slot, neighbours;
    uint32_t blksize, overlap, search_radius, levels;
    uint32_t mv_stride, conf_stride, sad_floor_word;
    float thsad; /* av-denoise-core/src/motion/confidence.rs:27-30; must be > 0 with confidence */
    uint32_t seeded; /* 1: `mv_field` already holds each block's seed and the search skips the coarse
                      * pass, as `run_seeded_refine` does (motion/analyse.rs:273-316) */
    uint64_t keep_seeds; /* i32 like `mv_field`: the field after the coarse pass, the truemotion stage's
                          * seed candidates (analyse.rs:268-277); 0 = not kept */
    uint64_t escalation; /* f32 scratch of avd_escalation_state_floats(neighbours, conf_stride) values;
                          * with ceiling > search_radius the blocks that fail the first pass search again
                          * `ceiling` around their first window (motion/escalate.rs:19-57, analyse.rs:
                          * 234-262); 0 = no escalation */
    uint32_t ceiling;         /* motion/context.rs:55-71: max_search_escalation; at most 8 */
    uint32_t esc_reads_floor; /* 1: a positive noise word `sad_floor_word` is the escalation floor; else it
                               * is measured from the first pass's SADs (escalate.rs:168-257) */
    uint64_t predictions; /* f32, 6 words per neighbour (m00 m01 m10 m11 tx ty): the camera model's
                           * prediction, a second search window at every level when it moves anything
                           * and lies outside the first, winning by more than 1/8 of noise word
                           * `sad_floor_word` (motion/kernels/candidates.rs, block_match.rs:98-265);
                           * 0 = no camera model (`noise` is then optional) */
    uint64_t sad;         /* f32, 2 * neighbours * conf_stride: each block's winning SAD, then its window's
                           * mean SAD (analyse.rs:41-60); 0 = not written */
    uint32_t coarse_radius;       /* motion/context.rs:34-37: the coarse pass's radius, 1..=8 or 12;
                                   * 0 = search_radius */
    uint32_t coarse_block_factor; /* context.rs:38-40: coarse blocks this many times wider; 0 or 1 = 1 */
} AvdMotionPass;

/* The f32 values the escalation state of a search over `neighbours` neighbours holds: four
 * sections of neighbours * conf_stride and the SAD floor (motion/analyse.rs:85-95). */
AVD_API uint64_t avd_escalation_state_floats(uint32_t neighbours, uint32_t conf_stride);

AVD_API AvdStatus avd_motion_search(const AvdMotionPass* pass, void* stream);

/* One pass of the truemotion stage that ends a search (av-denoise-core/src/motion/truemotion/
 * stage.rs:29-145 with kernels/truemotion/mod.rs:560-763): every block of every neighbour picks its
 * vector in `mv_in` again from its own vector, its 3x3 lower median, its four adjacent blocks'
 * vectors, zero, with `predictions` the camera model's point, and with `seeds` its own and its four
 * diagonal blocks' seeds, at cost SAD + lambda * |v - median|_1 (+ SAD / 8 off the median), with
 * lambda = field_lambda * blksize^2 * 0.02 + field_lambda * floor faded by the median's excess SAD
 * over 2 * thsad, then the ring of radius 1 around a new winner. The floor is noise word
 * `sad_field` when `reads_floor` and positive, else 0. Writes `mv_out` (a buffer apart from
 * `mv_in`) and, when set, `confidence` scored against noise word `sad_field`. Queued on `stream`. */
typedef struct AvdTruemotionPass {
    uint64_t pyramid;         /* f32 pyramid; level 0 is read */
    uint64_t neighbour_slots; /* u32 pyramid slot of each neighbour */
    uint64_t mv_in;           /* i32 (dx, dy) per block per neighbour, `mv_stride` apart */
    uint64_t seeds;           /* i32 like `mv_in`, the coarse pass's field; 0 = no seed candidates */
    uint64_t mv_out;          /* i32 like `mv_in`; written */
    uint64_t confidence;      /* f32 per block per neighbour, `conf_stride` apart; 0 = not written */
    uint64_t noise;           /* f32 words */
    uint32_t width, height, frame_count, centre_slot, neighbours;
    uint32_t blksize, overlap, mv_stride, conf_stride, sad_field, reads_floor;
    float field_lambda; /* > 0 */
    float thsad;
    uint64_t predictions; /* f32, 6 words per neighbour; 0 = no camera-model candidate */
    uint64_t sad;         /* f32 per block per neighbour, `conf_stride` apart: each block's winning SAD;
                           * 0 = not written */
} AvdTruemotionPass;

/* ---- the camera model (av-denoise-core/src/motion/global, motion/kernels/global.rs) -------------
 * A pair model is 5 f32 words (a, b, tx, ty, valid) mapping a luma position of the older frame into
 * the newer one: x' = a x - b y + tx, y' = b x + a y + ty (global/model.rs:6-10). */

/* global/fit.rs:196-250 (`run_model_fit`): fits one direction of a pair field into ring slot `slot`
 * of `models`, starting from ring slot `prior` when it is valid and would be accepted (-1: none).
 * `sad` (0 = none) holds each block's winning SAD and, with `has_contrast`, its window mean SAD and its
 * mean sample, `means_offset` values apart. `scratch` holds avd_model_fit_scratch_floats(blocks) f32;
 * its first 8 words end as the fit's state. */
typedef struct AvdModelFit {
    uint64_t field;   /* i32 (dx, dy) per block: one direction of a pair field */
    uint64_t sad;
    uint32_t has_contrast, means_offset, older_to_newer;
    uint32_t width, height, blksize, overlap;
    int32_t prior;
    uint64_t models;
    uint32_t slot;
    uint64_t scratch;
} AvdModelFit;

AVD_API uint64_t avd_model_fit_scratch_floats(uint32_t blocks);
AVD_API AvdStatus avd_model_fit(const AvdModelFit* fit, void* stream);

/* global/compose.rs:66-101 (`run_compose_models`) with kernels/global.rs:18-119: one prediction per
 * neighbour from the ring `models` and the device gap table `gaps` (`max_steps` ring slots per
 * neighbour from the centre outward, 0xFFFFFFFF for none); the first `past_neighbours` lie behind the
 * centre. `out` takes 6 f32 per neighbour. */
AVD_API AvdStatus avd_compose_models(uint64_t models, uint64_t gaps, uint64_t out, uint32_t neighbours,
                                     uint32_t max_steps, uint32_t past_neighbours, void* stream);

/* motion/kernels/global.rs:121-155 (`mc_block_means`): each block's mean sample of an f32 plane. */
AVD_API AvdStatus avd_block_means(uint64_t plane, uint64_t out, uint32_t width, uint32_t height, uint32_t blksize,
                                  uint32_t overlap, void* stream);

/* motion/kernels/pyramid.rs:66-132 (`mc_box_rows`, `mc_high_pass_cols`): an f32 plane minus its
 * (2 radius + 1)^2 box mean into `out`; `rows` is a plane of scratch. */
/* engine/spec.rs:403-415 (`build_with_models`): the engine's camera-model ring copied to `out` (depth
 * slots of 5 f32 words: a, b, tx, ty, valid; stream frame f's pair model in slot f % depth) after the
 * queued work; `*depth` is 0 when the engine fits no models (out may then be null). */
AVD_API AvdStatus avd_engine_models(AvdEngine* engine, float* out, uint32_t capacity, uint32_t* depth);

AVD_API AvdStatus avd_high_pass(uint64_t plane, uint64_t rows, uint64_t out, uint32_t width, uint32_t height,
                                uint32_t radius, void* stream);

AVD_API AvdStatus avd_truemotion_pass(const AvdTruemotionPass* pass, void* stream);

/* av-denoise-core/src/nlmeans/dispatch/motion.rs:619-690 (`run_chain_compose`) with
 * motion/kernels/chain.rs:20-72: every neighbour's seed of a pass centred on logical `centre` of a
 * 2d+1 window, walked through the pair ring from the centre (neighbour n is logical n, or n + 1 past
 * the centre). The pair between logical g and g+1 is in slot (head_mod + g) mod 2d; each slot holds
 * the older-to-newer field, then the newer-to-older field, `dir_stride` i32 apart. Writes
 * `mv_field` (2d neighbours, `mv_stride` apart). Queued on `stream`. */
AVD_API AvdStatus avd_chain_compose(uint64_t pair_ring, uint64_t mv_field, uint32_t mv_stride, uint32_t centre,
                                    uint32_t temporal_radius, uint32_t head_mod, uint32_t dir_stride, uint32_t width,
                                    uint32_t height, uint32_t blksize, uint32_t overlap, void* stream);

/* av-denoise-core/src/motion/confidence.rs:17-21 (`sad_noise_floor`). */
AVD_API float avd_sad_noise_floor(uint32_t blksize, float sigma);

/* av-denoise-core/src/motion/confidence.rs:27-30 (`thsad`). */
AVD_API float avd_thsad(uint32_t blksize, float thsad_scale);

/* ---- noise estimator kernel-level entry points --------------------------------------------- */

/* The floats of one frame's Immerkær partials: 2 lanes per 32x8 block
 * (av-denoise-core/src/noise/spatial.rs:44-47, `partials_len`). */
AVD_API uint64_t avd_immerkaer_partials_len(uint32_t width, uint32_t height);

/* The Immerkær spatial estimate of one f32 frame (`channels` 1 or 2 interleaved, as a ring slot holds
 * it): av-denoise-core/src/noise/spatial.rs:98-138 (`run_noise_estimate`: `nlm_noise_partial` into
 * `partials`, `nlm_noise_reduce` into `results`, 2 floats) and the reading's per-channel lower
 * quartile of the block sigmas (noise/kernels/sample.rs:181-203, 660-682) into `sigma_low`
 * (2 floats, 0 for an unused channel). `results` and `sigma_low` may be 0 to skip them. Queued on
 * `stream`. */
AVD_API AvdStatus avd_immerkaer(uint64_t frame, uint32_t channels, uint32_t width, uint32_t height, uint64_t partials,
                                uint64_t results, uint64_t sigma_low, void* stream);

/* The floats of one frame's temporal residual records: 3 * channels + 26 per 16x16 block
 * (av-denoise-core/src/noise/temporal.rs:98-123), and of the reading's per-block scratch. */
AVD_API uint64_t avd_noise_records_floats(uint32_t width, uint32_t height, uint32_t channels);
AVD_API uint64_t avd_noise_scratch_floats(uint32_t width, uint32_t height);

/* The temporal residual records of f32 frame `next` against `prev` (kernels/stats.rs:141-620,
 * `nlm_temporal_noise_stats` without motion compensation); with `luma_fields` each record also
 * carries its four 8x8 quarters' residual sums, luma sum, minimum, maximum and flatness
 * (stats.rs:466-606), else those lanes read 0. `prev` = 0 zeroes the records, as a stream's first
 * frame reads (noise/slot.rs:40-60). */
AVD_API AvdStatus avd_noise_temporal_stats(uint64_t next, uint64_t prev, uint32_t channels, uint32_t width,
                                           uint32_t height, uint32_t luma_fields, uint64_t records, void* stream);

/* The records of `next` against `prev` along a motion field (kernels/stats.rs:224-330, the compensated
 * variant): `mv_field` holds an int32 (dx, dy) per block of an mv_blocks_x x mv_blocks_y grid at
 * `mv_step`; each 16x16 block follows the vector of the motion block covering its origin when its
 * channel-0 residual variance along it is at most half the zero-vector variance, and a followed block
 * that leaves the frame writes an all-zero record. The moved lane records each followed block. */
AVD_API AvdStatus avd_noise_compensated_stats(uint64_t next, uint64_t prev, uint32_t channels, uint32_t width,
                                              uint32_t height, uint64_t mv_field, uint32_t mv_blocks_x,
                                              uint32_t mv_blocks_y, uint32_t mv_step, uint32_t luma_fields,
                                              uint64_t records, void* stream);

/* One frame's reading, AVD_NOISE_READING_WORDS floats (noise/reading.rs:7-33), from its records
 * (0 without temporal stats: the reading is then the Immerkaer words alone) through
 * kernels/sample.rs:143-803. With `curve` (records taken with the luma fields) the reading also
 * holds the noise curve: its flag, the static quarters' median sigma, the populated bin count and
 * 16 ratios (kernels/curve.rs:37-133, sample.rs:717-803). Words 0 and 1 must already hold the
 * frame's Immerkaer lower quartiles (`sigma_low` of avd_immerkaer); the call writes the rest.
 * `scratch` holds avd_noise_scratch_floats floats. */
#define AVD_NOISE_READING_WORDS 30
#define AVD_NOISE_STATE_WORDS 32
#define AVD_NOISE_DERIVED_WORDS 11
#define AVD_NOISE_FOLD_WORDS 16
AVD_API AvdStatus avd_noise_reading(uint64_t records, uint32_t channels, uint32_t width, uint32_t height,
                                    uint32_t curve, uint64_t scratch, uint64_t reading, void* stream);

/* The colour grain gains (av-denoise-core/src/noise/colour.rs, noise/kernels/colour.rs,
 * noise/kernels/colour_fit.rs). A cell table holds 976 values per plane: 16 brightness bins, each
 * one neutral cell and 5 saturation levels of 12 hue sectors. A frame's cell sums hold
 * avd_colour_records records of 69 int32 words (count, fixed-point log grain, luma, Cb and Cr sums,
 * a 64-bin log-grain histogram): the planes' cells, then 16 luma calibration records (luma) or one
 * record per chroma plane. */
AVD_API uint64_t avd_colour_records(uint32_t planes, uint32_t luma);
/* The mean luma, Cb and Cr (8-bit scale, chroma centred on 0) of every 16x16 block of the luma and
 * the chroma noise grids of one frame of `geometry` (kernels/colour.rs:187-340,
 * `noise_colour_means`), 3 floats per block of each grid. */
AVD_API AvdStatus avd_colour_means(uint64_t luma, uint64_t cb, uint64_t cr, const AvdGeometry* geometry,
                                   uint64_t luma_means, uint64_t chroma_means, void* stream);
/* One frame's cell sums, zeroed first, from its temporal records and its block means on the records'
 * grid (kernels/colour.rs:342-430, `noise_colour_accumulate`); `luma` pools the luma calibration
 * records. `grain_scale` turns a normalised residual sigma into codes on the 8-bit scale. */
AVD_API AvdStatus avd_colour_accumulate(uint64_t records, uint64_t means, uint32_t width, uint32_t height,
                                        uint32_t channels, uint32_t luma, float grain_scale, uint64_t cells,
                                        void* stream);
/* The decoded sums of frames first..=last of a ring of `capacity` frames' cell sums (frame f in slot
 * f % capacity, `words` int32 words each; kernels/colour.rs:441-470, `noise_colour_window`). */
AVD_API AvdStatus avd_colour_window(uint64_t ring, uint32_t capacity, uint32_t first, uint32_t last, uint32_t words,
                                    uint64_t window, void* stream);
/* Both fits of the window's sums and the log gain tables (noise/colour.rs:630-680, `ColourFit::queue`):
 * `planes` tables of 976 log grains into `table` and of 976 log gains into `gains`. A luma fit
 * (`luma`) reads the 16 curve ratios `curve` while the derived words' curve flag (word 3 of
 * `derived`) is set. `scratch` holds avd_colour_fit_scratch_floats floats. */
AVD_API uint64_t avd_colour_fit_scratch_floats(uint32_t planes);
AVD_API AvdStatus avd_colour_fit(uint64_t window, uint32_t planes, uint32_t luma, uint64_t curve, uint64_t derived,
                                 uint64_t scratch, uint64_t table, uint64_t gains, void* stream);
/* A table's value and its exponential (the gain) at each of `n` (luma, cb, cr) colours
 * (colour_fit.rs:196-262, `colour_table_value`, `colour_gain`). */
AVD_API AvdStatus avd_colour_lookup(uint64_t table, uint64_t colours, uint32_t n, uint64_t values, uint64_t gains,
                                    void* stream);

/* The fold settings words for a plane of width x height (noise/fold.rs:118-146, `fold_words`):
 * sigma_scale, whether the consumer applies the curve, the weight-scale gain and floor, the h2
 * coefficient (`h2_auto` 0 for a fixed strength `h2_fixed`), the pilot factor, the noise-offset
 * coefficient and whether the main pass subtracts it, and the two SAD-floor coefficients. */
AVD_API void avd_noise_fold_words(uint32_t width, uint32_t height, float sigma_scale, uint32_t curve_applies,
                                  float weight_g_max, float weight_floor, uint32_t h2_auto,
                                  float h2_per_inverse_variance, float h2_fixed, float pilot_h2_factor,
                                  float offset_per_variance, uint32_t main_offset, float sad_per_sigma,
                                  float confidence_sad_per_sigma, float* out16);

/* One window fold over history frames first..=last, frame f in slot f % capacity of `records`
 * (READING_WORDS each) and `results` (the two Immerkaer abs totals each): kernels/window.rs:414-498
 * (`noise_window_fold`). Writes the stream state (STATE_WORDS), the derived words
 * (DERIVED_WORDS: sigma[2], weight scale, curve flag, SAD floor, confidence SAD floor, h2, pilot h2,
 * noise offset, input noise offset, rho) and, with table_radius > 0, both (2r+1)^2 offset tables. */
AVD_API AvdStatus avd_noise_fold(uint64_t records, uint64_t results, uint32_t capacity, uint32_t first,
                                 uint32_t last, uint64_t settings, uint32_t channels, uint32_t table_radius,
                                 uint64_t state, uint64_t derived, uint64_t spatial_table, uint64_t pilot_table,
                                 void* stream);

/* ---- adjoint -------------------------------------------------------------------------------- */

/* No Rust item in the reference: the adjoint the hot-path contract adds to the boundary
 * (`avd_nlm_backward`, dL/d(frames) and dL/d(h)). It differentiates one output frame of the windowed
 * NLMeans path (av-denoise-core/src/nlmeans/kernels/fused.rs:138-530, accumulate.rs:152-202): the
 * window of 2d+1 normalised f32 frames (oldest first, `channels` interleaved, contiguous), the
 * search radius a, the patch radius s, the strength (h2 = 255^2 / (3 strength^2 (2s+1)^2), as
 * nlmeans/params.rs:229-233), the self weight, and the noise offsets of the pair and spatial
 * offsets (both 0 for the fast variant; NLMeans-HQ with a pinned sigma passes its noise offset in
 * both). Weights are recomputed, never stored; the max weight passes its gradient to the first offset
 * that reaches it. Scratch: avd_nlm_backward_scratch_bytes(width, height) bytes. Shared memory bounds
 * the window: the staged frames and gradient tiles, 2 (2d+1) (32 + 2(a+s)) (8 + 2(a+s)) channels
 * floats, must stay within 200 KiB, else AVD_ERR_INVALID_OPTIONS. `grad_window` and `grad_strength` are overwritten; queued on `stream`. */
typedef struct AvdNlmBackward {
    uint64_t window;        /* f32, (2d+1) x height x width x channels */
    uint64_t grad_out;      /* f32, height x width x channels: dL/d(output) */
    uint64_t grad_window;   /* f32 like `window`: dL/d(frames), written */
    uint64_t grad_strength; /* f32[1]: dL/d(strength), written */
    uint64_t scratch;
    uint32_t width, height, channels, temporal_radius, search_radius, patch_radius;
    float strength, self_weight, pair_offset, spatial_offset;
} AvdNlmBackward;

AVD_API uint64_t avd_nlm_backward_scratch_bytes(uint32_t width, uint32_t height);

/* The forward the adjoint differentiates, at kernel level: one output frame of the windowed NLMeans
 * path (the engine's launch, nlmeans/dispatch/mod.rs:627-679) from the same `AvdNlmBackward` fields
 * (`window`, the radii, strength, self weight and offsets) into `grad_out`, which here receives the
 * f32 output frame; `grad_window` and `grad_strength` are unused. `scratch` needs
 * avd_nlm_window_scratch_bytes(search_radius) bytes. Queued on `stream`; allocates nothing. */
AVD_API uint64_t avd_nlm_window_scratch_bytes(uint32_t search_radius);
AVD_API AvdStatus avd_nlm_window(const AvdNlmBackward* args, void* stream);

/* No Rust item in the reference (its `f32::exp`, helpers.rs:70-73, is lowered inside CubeCL): the
 * exponential of the exact NLMeans finish and the bilateral prefilter (exp_mirror.cuh) over `n`
 * device floats `x` into `out`, queued on `stream`; exposed so tests compare it with the CPU
 * restatement bit for bit. */
AVD_API AvdStatus avd_exp_mirror(uint64_t x, uint64_t out, uint64_t n, void* stream);
AVD_API AvdStatus avd_nlm_backward(const AvdNlmBackward* args, void* stream);

/* ---- batched launch ------------------------------------------------------------------------- */

/* No Rust item in the reference: the batched launch the hot-path contract adds to the boundary
 * (`avd_batch_submit`). Many clips of uneven resolution, window and strength, one denoised frame
 * per job, in one persistent launch over a tile work queue. A job is one output frame: `frames`
 * holds the clip's `n_frames` normalised f32 frames (height x width x channels each, contiguous),
 * the window is frames clamp(centre - d + k), k in 0..=2d (the engine's repeat edges), and the
 * result goes to `out`. Each job carries its own strength (h2 = 255^2 / (3 strength^2 (2s+1)^2)) and
 * noise offsets (0 and 0 for the fast variant; NLMeans-HQ with a pinned sigma passes its offset in
 * both). The batch shares channels, search radius, patch radius and self weight. */
typedef struct AvdBatchJob {
    uint64_t frames;
    uint64_t out;
    uint32_t n_frames, centre, temporal_radius, width, height;
    float strength, pair_offset, spatial_offset;
} AvdBatchJob;

/* The scratch one batch of `n_jobs` jobs needs (job table, tile prefix, strength words). */
AVD_API uint64_t avd_batch_scratch_bytes(size_t n_jobs, uint32_t search_radius);

/* Queues the batch on `stream`: one copy of its table into `scratch`, then one launch. */
AVD_API AvdStatus avd_batch_submit(const AvdBatchJob* jobs, size_t n_jobs, uint32_t channels, uint32_t search_radius,
                                   uint32_t patch_radius, float self_weight, uint64_t scratch, void* stream);

/* No counterpart in the reference (it ingests one frame per launch). The word planes of many frames
 * of mixed size and bit depth normalised into f32 frames by one launch, so a batch of clips of 8-,
 * 10- and 12-bit sources feeds avd_batch_submit without a launch per frame. Each item: `channels`
 * planes (plane1 for the second channel), samples of `bits` bits (8: four to a 32-bit word; 9..16:
 * two), normalised by 2^bits - 1 exactly as the engine's ingest does (a correctly rounded
 * division), interleaved into `frame` (width x height x channels f32). */
typedef struct AvdBatchIngest {
    uint64_t plane0, plane1, frame;
    uint32_t width, height, channels, bits;
} AvdBatchIngest;

/* The scratch one batched ingest of `n_items` items needs (its item table and word prefix). */
AVD_API uint64_t avd_batch_ingest_scratch_bytes(size_t n_items);

/* Queues the ingest on `stream`: one copy of its table into `scratch`, then one launch. */
AVD_API AvdStatus avd_batch_ingest(const AvdBatchIngest* items, size_t n_items, uint64_t scratch, void* stream);

/* ---- allocation-free entry point ----------------------------------------------------------- */

/* No counterpart in the reference. One fast-variant NLMeans output frame for callers that cannot
 * allocate device memory (a plugin inside another application's CUDA context, a real-time path
 * that must not enter the allocator mid-stream, a sandbox without the allocation calls). It makes
 * no cudaMalloc or cudaFree and calls no allocating library routine: its scratch lives in one
 * file-scope device array of 32 MiB that every GPU loading this library holds until exit, and
 * sizes that need more than that fail with AVD_ERR_INVALID_GEOMETRY (message in avd_last_error).
 *
 * `window` holds the (2 * temporal_radius + 1) input frames, oldest first, each as `channels`
 * planes (1 = luma, 2 = the U and V planes); the centre frame is the one denoised, exactly as the
 * engine denoises it with that window. `out` receives `channels` planes. Work is queued on
 * `stream` (a cudaStream_t; NULL = legacy default) with no host synchronisation.
 *
 * The first call in each CUDA context on a device (the primary context, a caller's own context, or
 * the new primary context after cudaDeviceReset) looks up the array's device address with that
 * device current, so make it before any stream capture. Every call shares the array and leaves its
 * contents behind; each call writes every scratch word it reads (it clears the count of samples
 * its exact finish recomputes), but calls whose GPU work overlaps race. */
AVD_API AvdStatus avd_nlm_frame_static(const AvdNlmeansAlgorithm* algorithm, uint32_t channels, uint32_t width,
                                       uint32_t height, AvdSampleFormat input, AvdSampleFormat output,
                                       const AvdPlane* window, size_t n_window, const AvdPlane* out, size_t n_out,
                                       void* stream);

#ifdef __cplusplus
}
#endif

#endif /* AVD_H */
