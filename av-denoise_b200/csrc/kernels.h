// Launch interfaces of the CUDA kernels (host-callable, no CUDA types beyond cudaStream_t).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace avd {

constexpr int kMaxPairs = 8;

// Sample layout of a caller plane: u8/u16 packed into 32-bit words, or f32.
struct PlaneFormat {
    int kind;  // AvdSampleKind
    int samples_per_word;
    float max_value;
};

// av-denoise-core/src/engine/kernels.rs:25-90 (`ingest_words`, `ingest_f32`): planes -> one
// interleaved f32 ring slot.
// One frame of a batched ingest: `channels` word planes (plane1 for the second channel) of
// `pixels` samples packed `samples_per_word` to a 32-bit word, normalised by `max_value` into the
// interleaved f32 frame `dst`.
struct BatchIngestItem {
    const uint32_t* plane0;
    const uint32_t* plane1;
    float* dst;
    int64_t pixels;
    int channels, samples_per_word;
    float max_value;
};
// Every item's words in one launch; `word_prefix[i]` is the first global word of item i
// (word_prefix[n] the total), both tables in device memory.
cudaError_t launch_batch_ingest(const BatchIngestItem* items, const int64_t* word_prefix, int n, int64_t total_words,
                                cudaStream_t stream);

cudaError_t launch_ingest(const void* plane0, const void* plane1, float* slot, int64_t pixels, int channels,
                          PlaneFormat fmt, float bias, cudaStream_t stream);

// av-denoise-core/src/engine/kernels.rs:103-184 (`egress_words`, `egress_f32`): an interleaved f32
// frame -> caller planes, zeroing the word padding.
cudaError_t launch_egress(const float* frame, void* plane0, void* plane1, int64_t pixels, int channels,
                          PlaneFormat fmt, float bias, cudaStream_t stream);

// One NLM output frame: every temporal pair pass, the single-frame pass and the finish, in one
// launch.
struct NlmLaunch {
    const float* ring;  // f32 ring, `slots` frames of width*height*channels
    int width, height, channels;
    int64_t frame_elems;  // width*height*channels
    int slot_centre;
    int pairs;  // temporal radius d
    int slot_fwd[kMaxPairs];  // pair k (q_k = -d + k): frame centre + q_k
    int slot_bwd[kMaxPairs];  // frame centre - q_k
    int patch_radius, search_radius;
    const float* derived;  // device words; h2 at `h2_word`, pair noise offset at `offset_word`
    int h2_word, offset_word;
    const float* spatial_lut;  // (2a+1)^2 single-pass offsets, or null for zeros
    const float* conf;  // per-block confidence, or null
    int64_t conf_fwd_off[kMaxPairs], conf_bwd_off[kMaxPairs];
    int conf_step, blocks_x, blocks_y;
    float wref;
    int fast;  // 1: no noise offsets and no confidence, so one strength weighs every lane
    float* out;  // width*height*channels
    const float* ref_ring;  // a prefilter's reference ring (same slots as `ring`) the distances
                            // compare, or null to compare `ring` itself
    // Samples near a rounding boundary (nlm_exact.cu). With `fix_count` set, the window kernel
    // appends to `fix_list` (and counts in `*fix_count`) every pixel with a result that, quantised
    // as the egress quantises it (clamped to [0, 1], times `code_max`, plus 0.5), lies within
    // code_max * (fix_band + kFixBandPerH2 * h2) codes of an integer; `launch_nlm_exact` then
    // recomputes those pixels in the FP32 mirror's operation order. The list holds at most
    // width*height entries.
    int* fix_list;
    int* fix_count;
    float code_max, fix_band;
    // The window kernel's launch variant (0: the baseline), one of nlm_window_variants(): the same
    // code built for a different number of resident CTAs per SM, so a variant trades registers for
    // occupancy and changes how many waves a frame's tiles take, never the results.
    int variant;
};

cudaError_t launch_nlm(const NlmLaunch& args, cudaStream_t stream);
int nlm_window_variants(int channels, int patch_radius, bool fast);

// The exact finish (nlm_exact.cu): every pixel of `args.fix_list[0 .. *args.fix_count)` (every pixel
// of the frame when `fix_list` is null) recomputed in the order and rounding of the FP32 mirror of
// the reference kernels (row-major patch sums, separately rounded operations, the mirror's own
// exponential) and written to `args.out`. The kernel reads the count on the device.
cudaError_t launch_nlm_exact(const NlmLaunch& args, cudaStream_t stream);
// The FP32 mirror's exponential of `n` floats on the device (its comparison with the oracle).
cudaError_t launch_exp_mirror(const float* x, float* out, int64_t n, cudaStream_t stream);
// The band the window kernel flags around each rounding boundary, in normalised units:
// kFixBand + kFixBandPerH2 * h2. The window kernel's float result differs from the mirror's by the
// box sums' and the MUFU exponential's rounding, which the strength h2 amplifies. Measured over
// strengths 1..16, patch radii 1..3, luma, chroma and NLMeans-HQ: the 99.99th percentile of the
// difference lies inside the band everywhere (6e-7 against 2.07e-6 at the 1080p luma workload's
// h2 of 13.5; 3.4e-6 against 1.4e-5 at h2 2408), the largest difference inside it where h2 is
// below 30. A sample is missed only where a difference past the band meets a value that close to a
// boundary: a few in ten million.
constexpr float kFixBand = 2e-6f;
constexpr float kFixBandPerH2 = 5e-9f;
// The same launch with `args.ref_ring` set (prefilter.cu).
cudaError_t launch_nlm_ref(const NlmLaunch& args, cudaStream_t stream);

// The bilateral prefilter (nlmeans/kernels/bilateral.rs:16-107) of one frame `in` into `out`
// (both width*height*channels f32): kernel radius `radius`, with the spatial and range factors
// 1 / (2 sigma^2) of prefilter/bilateral.rs:20-22.
cudaError_t launch_bilateral(const float* in, float* out, int width, int height, int channels, int radius,
                             float inv_two_sigma_s_sq, float inv_two_sigma_r_sq, cudaStream_t stream);

// A batch of NLM launches (device array `jobs`, all with `channels`, `patch_radius` and `fast`) as one
// persistent launch: `prefix` holds njobs + 1 running tile counts, `counter` one zeroed int.
int nlm_tile_rows(int channels, int patch_radius);
int nlm_tile_cols();
cudaError_t launch_nlm_batch(const NlmLaunch* jobs, const int* prefix, int njobs, int* counter, int channels,
                             int patch_radius, bool fast, int max_search_radius, int max_pairs, cudaStream_t stream);

// One NL4D collaborative-filter pass (collab/kernels/fused/mod.rs:170): every reference patch of
// the centre slot, scattered into the per-slot fixed-point accumulators.
struct CollabLaunch {
    const float* ring;  // slots of width*height*channels f32
    int width, height, channels, centre_slot;
    int64_t frame_elems;
    const int32_t* mv_field;        // per neighbour: blocks x (dx, dy)
    const float* confidence;        // per neighbour: blocks
    const uint32_t* neighbour_slots;  // ring slot of each neighbour index
    const float* noise;             // derived words
    int sigma_word, weight_scale_word, curve_valid_word;
    const float* noise_curve;       // 16 ratios
    const float* dct_profile;       // 8
    const float* kaiser;            // 8
    int32_t* accum;                 // slots x pixels x channels
    int32_t* wsum;                  // slots x pixels
    float* group_weight;            // refs
    uint32_t* members;              // scratch: collab_member_words(width, height) words
    float c_min, lambda_ht, accum_scale, pool_ratio;
    int pooled;
    int radius, refine, spatial_radius, k_max;
    int mv_stride, conf_stride, blk_step, blksize, blocks_x, blocks_y;
    // The colour grain gains (collab/kernels/fused/colour.rs): one log gain table of 976 cells per
    // channel, the centre frame's block means (3 floats per block of this plane's 16x16 grid,
    // colour_blocks_x across) and the factor from a sample to the 8-bit scale; read with colour_on.
    const float* colour_gains;
    const float* colour_means;
    float colour_scale;
    int colour_on, colour_blocks_x;
    // The empirical Wiener stage after the threshold (an extension the reference does not have):
    // each kept coefficient z of noise variance v scaled by z^2 / (z^2 + v).
    int wiener;
};

cudaError_t launch_collab(const CollabLaunch& args, cudaStream_t stream);

// The adjoint of one collab pass (collab.cu: collab_adjoint_kernel), run after the pass with the
// same arguments and the member words its search left in `members`. A and W are the accumulators
// in real units (accum / accum_scale, wsum / (5 accum_scale)).
struct CollabAdjointLaunch {
    const float* grad_accum;  // dL/dA, laid out as the accumulators (slots x pixels x channels)
    const float* grad_wsum;   // dL/dW, slots x pixels
    float* grad_ring;         // dL/d(ring), laid out as the ring, added into
    float* grad_sigma_refs;   // each reference patch's share of dL/d(sigma_c), refs x channels, written
};
cudaError_t launch_collab_adjoint(const CollabLaunch& args, const CollabAdjointLaunch& adjoint, cudaStream_t stream);
// The scratch words between the search and filter launches: 9 per reference patch.
size_t collab_member_words(int width, int height);

// collab/kernels/aggregate.rs:240-290 (`collab_normalise`): one region's accum * 5 / wsum (accum
// itself where wsum is 0) into `out`, then the region zeroed.
cudaError_t launch_collab_normalise(int32_t* accum, int32_t* wsum, float* out, int64_t pixels, int channels,
                                    cudaStream_t stream);

// Block-matching motion search (motion.cu). The pyramid must already hold every slot it reads.
struct MotionLaunch {
    static constexpr int kMaxInlineSlots = 16;
    const float* pyramid;
    const uint32_t* neighbour_slots;  // device table, or null to read `inline_slots`
    uint32_t inline_slots[kMaxInlineSlots];
    int32_t* mv_field;
    float* confidence;  // may be null: no confidence is written
    const float* noise;
    int width, height, frame_count, centre_slot, neighbours;
    int blksize, overlap, search_radius, coarse_radius, coarse_block_factor, levels;
    int mv_stride, conf_stride, sad_floor_word;
    float thsad;
    int seeded;  // 1: the field already holds every block's seed; no coarse pass
    int32_t* keep_seeds;  // non-null: the field after the coarse pass is copied here (the truemotion
                          // stage's seed candidates)
    // Search escalation (motion/escalate.rs): with `escalation` (escalation_state_floats of scratch)
    // and ceiling > search_radius, the blocks that fail the first pass search again `ceiling` around
    // their first window's centre. The floor is the noise word when `esc_reads_floor` and positive,
    // else measured from the first pass's SADs; `thsad` must be positive.
    float* escalation;
    int ceiling, esc_reads_floor;
    // The camera model (motion/kernels/candidates.rs): with `predictions` (6 words per neighbour,
    // `noise` required) every pass also searches around the neighbour's prediction, that window
    // winning by more than 1/8 of noise word `sad_floor_word` (scaled to the coarse block on the
    // coarse level). With `sad`, the fine pass writes each block's winning SAD and then, neighbours *
    // conf_stride values on, its window's mean SAD; escalation replaces an improved block's SAD.
    const float* predictions;
    float* sad;
};

size_t escalation_state_floats(int neighbours, int conf_stride);

int64_t pyramid_slot_pixels(int width, int height, int level);
void pyramid_level_dims(int width, int height, int level, int* w, int* h);
int64_t pyramid_level_base(int width, int height, int frame_count, int level);
int64_t pyramid_floats(int width, int height, int frame_count, int levels);
cudaError_t launch_pyramid_build(const float* ring, int channels, int width, int height, int frame_count,
                                 int ring_slot, int levels, float* pyramid, int pyramid_slot, cudaStream_t stream);
cudaError_t launch_motion_search(const MotionLaunch& args, cudaStream_t stream);

// One truemotion pass (truemotion.cu, motion/truemotion/kernels/truemotion/mod.rs:560-763) over the
// field `mv_in` into `mv_out` (a separate buffer), with `seeds` (or null) as extra candidates and
// the confidence written when `confidence` is set. lambda_base = field_lambda * blksize^2 * 0.02,
// lambda_noise = field_lambda, fade_level = 2 * thsad (truemotion/stage.rs:52-62).
struct TruemotionLaunch {
    static constexpr int kMaxInlineSlots = 16;
    const float* pyramid;  // level 0: slot s starts s * slot_pixels values in
    int64_t slot_pixels;
    const uint32_t* neighbour_slots;  // device table, or null to read `inline_slots`
    uint32_t inline_slots[kMaxInlineSlots];
    const int32_t* mv_in;
    const int32_t* seeds;
    int32_t* mv_out;
    float* confidence;
    const float* noise;
    int width, height, centre_slot, neighbours, blksize, step, blocks_x, blocks_y, mv_stride, conf_stride;
    int sad_field, reads_floor, refine_radius;
    float lambda_base, lambda_noise, surcharge, fade_level, thsad;
    // truemotion/kernels/truemotion/mod.rs:483-520: with `changes_in`, a block whose 3x3
    // neighbourhood changed nothing last pass copies its own vector (its confidence stands);
    // `changes_out` flags the blocks whose pick left their own vector (conf layout).
    const uint32_t* changes_in;
    uint32_t* changes_out;
    // mod.rs:878-900: with `predictions` (6 words per neighbour) the camera model's prediction at the
    // block is a candidate when the model moves anything; with `sad`, every rescored block writes
    // its winning SAD there (conf layout).
    const float* predictions;
    float* sad;
};
cudaError_t launch_truemotion(const TruemotionLaunch& args, cudaStream_t stream);

// ---- the camera model (camera.cu; av-denoise-core/src/motion/global, kernels/global.rs) ------------

constexpr int kAffineWords = 6;  // a prediction: m00 m01 m10 m11 tx ty
constexpr int kModelWords = 5;   // a pair model: a b tx ty valid (global/model.rs:6-10)
//
// A pair model is 5 f32 words (a, b, tx, ty, valid) mapping a luma position of the older frame into
// the newer one, x' = a x - b y + tx, y' = b x + a y + ty; a prediction is 6 words (m00 m01 m10 m11
// tx ty) per neighbour.

// global/fit.rs:196-250 (`run_model_fit`): fits one direction of a pair field into ring slot `slot`
// of `models`, from ring slot `prior` when it is at least 0. `sad` (or null) holds the winning SADs,
// then, with `has_contrast`, the window means and the block means, `means_offset` values apart.
// `scratch` holds model_fit_scratch_floats(blocks) floats: the 8 state words first.
struct ModelFitLaunch {
    const int32_t* field;
    const float* sad;
    bool has_contrast;
    int means_offset;
    bool older_to_newer;
    int width, height, blksize, step;
    int prior;
    float* models;
    int slot;
    float* scratch;
};
size_t model_fit_scratch_floats(int blocks);
cudaError_t launch_model_fit(const ModelFitLaunch& args, cudaStream_t stream);
// global.rs:18-119 (`mc_compose_models`): `gaps` holds `max_steps` ring slots (or 0xFFFFFFFF) per
// neighbour, from the centre outward; the first `past_neighbours` neighbours lie behind the centre.
cudaError_t launch_compose_models(const float* models, const uint32_t* gaps, float* out, int neighbours,
                                  int max_steps, int past_neighbours, cudaStream_t stream);
// The same with a host gap table of neighbours * max_steps entries (at most kMaxInlineGaps), passed
// to the kernel by value.
constexpr int kMaxInlineGaps = 256;
cudaError_t launch_compose_inline(const float* models, const uint32_t* host_gaps, float* out, int neighbours,
                                  int max_steps, int past_neighbours, cudaStream_t stream);
// global.rs:121-155 (`mc_block_means`) on the block grid of blksize / step.
cudaError_t launch_block_means(const float* plane, float* out, int width, int height, int blksize, int step,
                               cudaStream_t stream);
// pyramid.rs:66-132: `out` = `plane` minus its (2 radius + 1)^2 box mean; `rows` is scratch.
cudaError_t launch_high_pass(const float* plane, float* rows, float* out, int width, int height, int radius,
                             cudaStream_t stream);
// global.rs:157-172 (`mc_model_identity`).
cudaError_t launch_model_identity(float* models, int slot, cudaStream_t stream);

// motion/kernels/compensate.rs (`mc_warp`) for every neighbour of a window in one launch: ring slot
// slots[n] of `src_ring` (and `src_ref`, when set) warped along neighbour n's field into the same
// slot of `dst_ring` (and `dst_ref`).
struct WarpLaunch {
    static constexpr int kMaxSlots = 16;
    const float* src_ring;
    float* dst_ring;
    const float* src_ref;
    float* dst_ref;
    const int32_t* mv_field;
    int mv_stride;
    uint32_t slots[kMaxSlots];
    int neighbours;
    int64_t frame_elems;
    int channels, width, height, step, blocks_x, blocks_y;
};
cudaError_t launch_warp(const WarpLaunch& args, cudaStream_t stream);

// motion/kernels/chroma_map.rs (`mc_map_luma_fields`): `fields` luma motion fields mapped onto the
// chroma block grid, each chroma block the per-component lower median of the luma blocks inside the
// area it covers (clamped to the luma grid), divided by the subsampling and rounded half away from
// zero.
struct MapLaunch {
    const int32_t* luma;
    int32_t* chroma;
    int fields;
    int luma_bx, luma_by, luma_step, luma_blksize, luma_stride;
    int chroma_bx, chroma_by, chroma_step, chroma_blksize, chroma_stride;
    int shift_x, shift_y;
};
cudaError_t launch_map_luma_fields(const MapLaunch& args, cudaStream_t stream);

// motion/kernels/chain.rs (`mc_chain_compose`): every neighbour's seed as the walk of pair vectors
// from the centre. Neighbour n is logical position n (n < centre) or n + 1 of a 2d+1 window; the pair
// between logical g and g+1 sits in pair slot (head_mod + g) mod 2d, direction 0 older-to-newer and
// 1 newer-to-older, `dir_stride` values apart, `slot_stride` per slot.
cudaError_t launch_chain_compose(const int32_t* pair_ring, int32_t* mv_field, int mv_stride, int centre, int d,
                                 int head_mod, int dir_stride, int slot_stride, int step, int width, int height,
                                 int blocks_x, int blocks_y, cudaStream_t stream);

// Immerkær spatial noise estimate (immerkaer.cu) of one f32 frame (`channels` interleaved):
// per 32x8 block partials (2 lanes each), optional frame totals (2 floats) and optional per-channel
// lower quartile of the block sigmas (2 floats; unused channels 0). `scale` is sqrt(pi / 2) in f32.
size_t immerkaer_partials_len(int width, int height);
// Automatic noise estimate (noise_estimate.cu).
size_t noise_scratch_floats(int width, int height);
size_t noise_records_floats(int width, int height, int channels);
// With `mv_field` (null for none) each block reads `prev` along its motion block's vector; with
// `luma_fields` each record also carries its four 8x8 quarters' fields, from which a reading with
// `curve` builds the noise curve.
cudaError_t launch_temporal_stats(const float* next, const float* prev, int channels, int width, int height,
                                  const int32_t* mv_field, int mv_blocks_x, int mv_blocks_y, int mv_step,
                                  bool luma_fields, float* records, cudaStream_t s);
cudaError_t launch_noise_reading(const float* records, int channels, int width, int height, float* scratch,
                                 uint32_t min_accepted, bool curve, float* reading, cudaStream_t s);
cudaError_t launch_noise_fold(const float* records, const float* results, int capacity, int first, int last,
                              const float* settings, int channels, int table_radius, float* state, float* derived,
                              float* spatial, float* pilot, cudaStream_t s);
cudaError_t launch_immerkaer(const float* frame, int channels, int width, int height, float scale, float* partials,
                             float* results, float* sigma_low, cudaStream_t stream);

// The colour grain gains (colour.cu). A cell table holds 976 values per plane: 16 brightness bins of
// one neutral cell and 5 saturation levels of 12 hue sectors. A frame's cell sums hold
// colour_records(planes, luma) records of kColourCellWords int32 words: the planes' cells, then 16
// luma calibration records or one record per chroma plane.
constexpr int kColourCells = 976;
constexpr int kColourCellWords = 69;
constexpr int kColourFitPlaneWords = 22;
constexpr int kColourDerivedCurveWord = 3;  // the derived words' curve flag
size_t colour_records(int planes, bool luma);

// noise/kernels/colour.rs:187-340: the mean luma, Cb and Cr (8-bit scale, chroma centred on 0) of
// every 16x16 block of the luma and of the chroma noise grid, from the three input planes.
struct ColourMeansLaunch {
    const uint32_t *luma, *cb, *cr;  // word-packed planes
    int width, height, shift_x, shift_y;
    int samples_per_word;            // 4 (8-bit), 2 (9..16-bit) or 1 (f32)
    bool is_float;
    float eight_bit_scale, chroma_bias;
    float *luma_means, *chroma_means;  // 3 floats per block of each grid
};
cudaError_t launch_colour_means(const ColourMeansLaunch& args, cudaStream_t s);
// noise/kernels/colour.rs:342-430: one frame's cell sums (zeroed first) from its temporal records
// and its block means on the records' grid; `luma` pools the luma calibration records.
cudaError_t launch_colour_accumulate(const float* records, const float* means, int width, int height, int channels,
                                     bool luma, float grain_scale, int32_t* cells, cudaStream_t s);
// noise/kernels/colour.rs:441-470: the decoded sums of frames first..last (frame f in ring slot
// f % capacity, `words` int32 words per slot).
cudaError_t launch_colour_window(const int32_t* ring, int capacity, int first, int last, int words, float* window,
                                 cudaStream_t s);
// noise/colour.rs:630-680 (`ColourFit::queue`): both fits and the log gain tables of the window's sums.
struct ColourFitLaunch {
    const float* window;
    int planes;
    bool luma;                 // luma: mean levels, calibration against the curve; chroma: medians
    const float* curve;        // 16 luma curve ratios (luma only)
    const float* derived;      // the fold's derived words: the curve flag
    float *levels, *ceilings, *fit_cells, *fit_planes, *bases;  // scratch (colour_fit_scratch_floats)
    float *table, *gains;      // planes x 976 each
};
// The scratch floats of one fit: levels (2 per cell), ceilings (1), cell records (5), plane headers
// and the lift's 2 x 976 queries per plane.
inline size_t colour_fit_scratch_floats(int planes) {
    return static_cast<size_t>(planes) * (kColourCells * 8 + kColourFitPlaneWords + 2 * kColourCells);
}
cudaError_t launch_colour_fit(const ColourFitLaunch& args, cudaStream_t s);
// colour_fit.rs:196-262: a table's value and its gain at each of `n` (luma, cb, cr) colours.
cudaError_t launch_colour_lookup(const float* table, const float* colours, int n, float* values, float* gains,
                                 cudaStream_t s);

// Adjoint of one windowed NLMeans frame (nlm_backward.cu).
struct NlmBackwardLaunch {
    const float* window;    // (2d+1) frames of width*height*channels f32, oldest first
    const float* grad_out;  // width*height*channels
    float* grad_window;     // like window; overwritten
    float* grad_strength;   // 1 float; overwritten
    float* scratch;         // nlm_backward_scratch_floats(width, height)
    int width, height, channels, temporal_radius, search_radius, patch_radius;
    float strength, h2, wref, pair_offset, spatial_offset;
};
size_t nlm_backward_scratch_floats(int width, int height);
size_t nlm_backward_smem_bytes(int channels, int temporal_radius, int search_radius, int patch_radius);
cudaError_t launch_nlm_backward(const NlmBackwardLaunch& args, cudaStream_t stream);
// Words for a kernel-level NLM launch: h2 at 0, the pair offset at 1, the (2a+1)^2 spatial offset
// table (flat, 0 at the centre) from word 8.
cudaError_t launch_window_words(float* words, float h2, float pair_offset, float spatial_offset, int a,
                                cudaStream_t stream);

}  // namespace avd
