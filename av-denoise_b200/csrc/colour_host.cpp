// Host side of the colour grain gains: the engine's block-means ring (noise/colour.rs:176-330,
// `ColourBlocks`), the sample scales (colour.rs:338-361) and the C entry points of the colour kernels.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>

#include "avd_internal.h"
#include "engine_parts.h"
#include "kernels.h"

namespace avd {

namespace {
constexpr size_t kSlotMargin = 2;  // colour.rs:172-175: a compensated stream reads its first frame again

size_t grid_blocks(uint32_t w, uint32_t h) { return static_cast<size_t>((w + 15) / 16) * ((h + 15) / 16); }

int shift_x_of(const AvdGeometry& g) { return g.chroma == AVD_CHROMA_YUV444 ? 0 : 1; }
int shift_y_of(const AvdGeometry& g) { return g.chroma == AVD_CHROMA_YUV420 ? 1 : 0; }
}  // namespace

// colour.rs:344-361 (`eight_bit_scale`): a high bit-depth code divides by its extra bits; a float
// sample is normalised, so it scales by 255.
float colour_eight_bit_scale(const AvdSampleFormat& f) {
    switch (f.kind) {
        case AVD_SAMPLE_U8: return 1.0f;
        case AVD_SAMPLE_U16: return 1.0f / static_cast<float>(1u << (f.depth - 8));
        default: return 255.0f;
    }
}

// colour.rs:338-342 (`grain_scale`).
float colour_grain_scale(const AvdSampleFormat& f) { return sample_max_value(f) * colour_eight_bit_scale(f); }

std::optional<Failure> ColourMeans::allocate(const AvdGeometry& g, size_t held_frames) {
    geometry_ = g;
    slots_ = held_frames + kSlotMargin;
    uint32_t cw, ch;
    plane_dims(g, 1, &cw, &ch);
    luma_blocks_ = grid_blocks(g.width, g.height);
    chroma_blocks_ = grid_blocks(cw, ch);
    tags_.assign(slots_, -1);
    cudaError_t e;
    if ((e = luma_.alloc(slots_ * luma_blocks_ * 3 * sizeof(float))) != cudaSuccess ||
        (e = chroma_.alloc(slots_ * chroma_blocks_ * 3 * sizeof(float))) != cudaSuccess)
        return Failure{AVD_ERR_GPU, cuda_message("colour block means", e)};
    return std::nullopt;
}

std::optional<Failure> ColourMeans::queue(const AvdPlane* planes, uint32_t frame, cudaStream_t s) {
    const size_t slot = frame % slots_;
    ColourMeansLaunch a{};
    a.luma = reinterpret_cast<const uint32_t*>(planes[0].ptr);
    a.cb = reinterpret_cast<const uint32_t*>(planes[1].ptr);
    a.cr = reinterpret_cast<const uint32_t*>(planes[2].ptr);
    a.width = static_cast<int>(geometry_.width);
    a.height = static_cast<int>(geometry_.height);
    a.shift_x = shift_x_of(geometry_);
    a.shift_y = shift_y_of(geometry_);
    a.samples_per_word = static_cast<int>(samples_per_word(geometry_.input));
    a.is_float = geometry_.input.kind == AVD_SAMPLE_F32;
    a.eight_bit_scale = colour_eight_bit_scale(geometry_.input);
    a.chroma_bias = a.is_float ? 0.5f : 0.0f;  // colour.rs:363-371: float chroma sits in -0.5..0.5
    a.luma_means = luma_.as<float>() + slot * luma_blocks_ * 3;
    a.chroma_means = chroma_.as<float>() + slot * chroma_blocks_ * 3;
    cudaError_t e = launch_colour_means(a, s);
    if (e != cudaSuccess) return Failure{AVD_ERR_GPU, cuda_message("colour block means launch", e)};
    tags_[slot] = frame;
    return std::nullopt;
}

const float* ColourMeans::held(bool luma_grid, uint32_t frame) const {
    const size_t slot = frame % slots_;
    if (tags_[slot] != static_cast<int64_t>(frame)) return nullptr;
    return luma_grid ? luma_.as<float>() + slot * luma_blocks_ * 3 : chroma_.as<float>() + slot * chroma_blocks_ * 3;
}

void ColourMeans::clear() { std::fill(tags_.begin(), tags_.end(), -1); }

float ColourMeans::grain_scale() const { return colour_grain_scale(geometry_.input); }

}  // namespace avd

// ---- C entry points (include/avd.h) -------------------------------------------------------------

void avd_set_last_error(const std::string& m);

namespace {
AvdStatus fail(AvdStatus st, const std::string& m) {
    avd_set_last_error(m);
    return st;
}
AvdStatus gpu(const char* what, cudaError_t e) {
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, avd::cuda_message(what, e));
    return AVD_OK;
}
}  // namespace

uint64_t avd_colour_records(uint32_t planes, uint32_t luma) { return avd::colour_records(static_cast<int>(planes), luma != 0); }

uint64_t avd_colour_fit_scratch_floats(uint32_t planes) {
    return avd::colour_fit_scratch_floats(static_cast<int>(planes));
}

AvdStatus avd_colour_means(uint64_t luma, uint64_t cb, uint64_t cr, const AvdGeometry* geometry, uint64_t luma_means,
                           uint64_t chroma_means, void* stream) {
    if (!geometry || !luma || !cb || !cr || !luma_means || !chroma_means)
        return fail(AVD_ERR_NULL_ARG, "colour means: null argument");
    const AvdGeometry& g = *geometry;
    if (g.chroma == AVD_CHROMA_GRAY || g.width == 0 || g.height == 0)
        return fail(AVD_ERR_INVALID_GEOMETRY, "colour means: frames with chroma planes are needed");
    avd::ColourMeansLaunch a{};
    a.luma = reinterpret_cast<const uint32_t*>(luma);
    a.cb = reinterpret_cast<const uint32_t*>(cb);
    a.cr = reinterpret_cast<const uint32_t*>(cr);
    a.width = static_cast<int>(g.width);
    a.height = static_cast<int>(g.height);
    a.shift_x = avd::shift_x_of(g);
    a.shift_y = avd::shift_y_of(g);
    a.samples_per_word = static_cast<int>(avd::samples_per_word(g.input));
    a.is_float = g.input.kind == AVD_SAMPLE_F32;
    a.eight_bit_scale = avd::colour_eight_bit_scale(g.input);
    a.chroma_bias = a.is_float ? 0.5f : 0.0f;
    a.luma_means = reinterpret_cast<float*>(luma_means);
    a.chroma_means = reinterpret_cast<float*>(chroma_means);
    return gpu("colour means launch", avd::launch_colour_means(a, static_cast<cudaStream_t>(stream)));
}

AvdStatus avd_colour_accumulate(uint64_t records, uint64_t means, uint32_t width, uint32_t height, uint32_t channels,
                                uint32_t luma, float grain_scale, uint64_t cells, void* stream) {
    if (!records || !means || !cells) return fail(AVD_ERR_NULL_ARG, "colour cells: null buffer");
    if (channels < 1 || channels > 2 || width == 0 || height == 0)
        return fail(AVD_ERR_INVALID_GEOMETRY, "colour cells: bad geometry");
    return gpu("colour cells launch",
               avd::launch_colour_accumulate(reinterpret_cast<const float*>(records),
                                             reinterpret_cast<const float*>(means), static_cast<int>(width),
                                             static_cast<int>(height), static_cast<int>(channels), luma != 0,
                                             grain_scale, reinterpret_cast<int32_t*>(cells),
                                             static_cast<cudaStream_t>(stream)));
}

AvdStatus avd_colour_window(uint64_t ring, uint32_t capacity, uint32_t first, uint32_t last, uint32_t words,
                            uint64_t window, void* stream) {
    if (!ring || !window) return fail(AVD_ERR_NULL_ARG, "colour window: null buffer");
    if (capacity == 0 || last < first || last - first + 1 > capacity || words == 0)
        return fail(AVD_ERR_INVALID_OPTIONS, "colour window: bad bounds");
    return gpu("colour window launch",
               avd::launch_colour_window(reinterpret_cast<const int32_t*>(ring), static_cast<int>(capacity),
                                         static_cast<int>(first), static_cast<int>(last), static_cast<int>(words),
                                         reinterpret_cast<float*>(window), static_cast<cudaStream_t>(stream)));
}

AvdStatus avd_colour_fit(uint64_t window, uint32_t planes, uint32_t luma, uint64_t curve, uint64_t derived,
                         uint64_t scratch, uint64_t table, uint64_t gains, void* stream) {
    if (!window || !derived || !scratch || !table || !gains || (luma && !curve))
        return fail(AVD_ERR_NULL_ARG, "colour fit: null buffer");
    if (planes < 1 || planes > 2) return fail(AVD_ERR_INVALID_OPTIONS, "colour fit: 1 or 2 planes");
    avd::ColourFitLaunch a{};
    const int p = static_cast<int>(planes);
    float* s = reinterpret_cast<float*>(scratch);
    a.window = reinterpret_cast<const float*>(window);
    a.planes = p;
    a.luma = luma != 0;
    a.curve = reinterpret_cast<const float*>(curve);
    a.derived = reinterpret_cast<const float*>(derived);
    a.levels = s;
    a.ceilings = a.levels + 2 * p * avd::kColourCells;
    a.fit_cells = a.ceilings + p * avd::kColourCells;
    a.fit_planes = a.fit_cells + 5 * p * avd::kColourCells;
    a.bases = a.fit_planes + p * avd::kColourFitPlaneWords;
    a.table = reinterpret_cast<float*>(table);
    a.gains = reinterpret_cast<float*>(gains);
    return gpu("colour fit launch", avd::launch_colour_fit(a, static_cast<cudaStream_t>(stream)));
}

AvdStatus avd_colour_lookup(uint64_t table, uint64_t colours, uint32_t n, uint64_t values, uint64_t gains,
                            void* stream) {
    if (!table || !colours || !values || !gains) return fail(AVD_ERR_NULL_ARG, "colour lookup: null buffer");
    if (n == 0) return AVD_OK;
    return gpu("colour lookup launch",
               avd::launch_colour_lookup(reinterpret_cast<const float*>(table), reinterpret_cast<const float*>(colours),
                                         static_cast<int>(n), reinterpret_cast<float*>(values),
                                         reinterpret_cast<float*>(gains), static_cast<cudaStream_t>(stream)));
}
