// Host side of the automatic noise estimate: the kernel-level C ABI over noise_estimate.cu and the
// host helpers the engine shares with it (noise/temporal.rs:83-100 `min_static_blocks`,
// noise/fold.rs:118-146 `fold_words`).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "avd_internal.h"
#include "kernels.h"

void avd_set_last_error(const std::string& m);

namespace avd {

// The fewest accepted blocks out of `total` whose static fraction reaches 0.05, with the f32
// division the reading's gate uses.
uint32_t min_static_blocks(uint32_t total) {
    const float t = static_cast<float>(total);
    auto reaches = [&](uint32_t a) { return static_cast<float>(a) / t >= 0.05f; };
    uint32_t a = std::min<uint32_t>(static_cast<uint32_t>(0.05f * t), total);
    while (a > 0 && reaches(a - 1)) --a;
    while (a < total && !reaches(a)) ++a;
    return a;
}

float immerkaer_sigma_scale() {
    const volatile float half_pi = 1.57079632679489661923f;
    return std::sqrt(static_cast<float>(half_pi));
}

void noise_fold_words(uint32_t width, uint32_t height, const FoldCoefficients& k, float* words) {
    std::fill(words, words + 16, 0.0f);
    const float interior = static_cast<float>(width - 2) * static_cast<float>(height - 2);
    const float divisor = 6.0f * interior;
    words[0] = k.sigma_scale;
    words[1] = k.curve_applies ? 1.0f : 0.0f;
    words[2] = k.weight_g_max;
    words[3] = k.weight_floor;
    words[4] = k.h2_auto ? 1.0f : 0.0f;
    words[5] = k.h2_auto ? k.h2_per_inverse_variance : 0.0f;
    words[6] = k.h2_fixed;
    words[7] = k.pilot_h2_factor;
    words[8] = k.offset_per_variance;
    words[9] = k.main_offset ? 1.0f : 0.0f;
    words[10] = k.sad_per_sigma;
    words[11] = k.confidence_sad_per_sigma;
    words[12] = immerkaer_sigma_scale() / divisor;
    // noise/correlation.rs:7-8: the correlation table's three segment widths, as reciprocals.
    const float rho[4] = {0.0f, 0.3f, 0.5f, 0.65f};
    for (int i = 0; i < 3; ++i) words[13 + i] = 1.0f / (rho[i + 1] - rho[i]);
}

}  // namespace avd

namespace {
AvdStatus fail(AvdStatus s, const std::string& m) {
    avd_set_last_error(m);
    return s;
}
}  // namespace

extern "C" {

uint64_t avd_noise_records_floats(uint32_t width, uint32_t height, uint32_t channels) {
    return avd::noise_records_floats(static_cast<int>(width), static_cast<int>(height), static_cast<int>(channels));
}

uint64_t avd_noise_scratch_floats(uint32_t width, uint32_t height) {
    return avd::noise_scratch_floats(static_cast<int>(width), static_cast<int>(height));
}

AvdStatus avd_noise_temporal_stats(uint64_t next, uint64_t prev, uint32_t channels, uint32_t width, uint32_t height,
                                   uint32_t luma_fields, uint64_t records, void* stream) {
    if (!next || !records) return fail(AVD_ERR_NULL_ARG, "noise temporal stats: null buffer");
    if (channels < 1 || channels > 2 || width == 0 || height == 0)
        return fail(AVD_ERR_INVALID_GEOMETRY, "noise temporal stats: bad geometry");
    cudaError_t e = avd::launch_temporal_stats(reinterpret_cast<const float*>(next), reinterpret_cast<const float*>(prev),
                                               static_cast<int>(channels), static_cast<int>(width),
                                               static_cast<int>(height), nullptr, 0, 0, 0, luma_fields != 0,
                                               reinterpret_cast<float*>(records), static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, std::string("noise temporal stats launch: ") + cudaGetErrorString(e));
    return AVD_OK;
}

AvdStatus avd_noise_compensated_stats(uint64_t next, uint64_t prev, uint32_t channels, uint32_t width, uint32_t height,
                                      uint64_t mv_field, uint32_t mv_blocks_x, uint32_t mv_blocks_y, uint32_t mv_step,
                                      uint32_t luma_fields, uint64_t records, void* stream) {
    if (!next || !prev || !records || !mv_field) return fail(AVD_ERR_NULL_ARG, "noise compensated stats: null buffer");
    if (channels < 1 || channels > 2 || width == 0 || height == 0 || mv_blocks_x == 0 || mv_blocks_y == 0 ||
        mv_step == 0)
        return fail(AVD_ERR_INVALID_GEOMETRY, "noise compensated stats: bad geometry");
    cudaError_t e = avd::launch_temporal_stats(
        reinterpret_cast<const float*>(next), reinterpret_cast<const float*>(prev), static_cast<int>(channels),
        static_cast<int>(width), static_cast<int>(height), reinterpret_cast<const int32_t*>(mv_field),
        static_cast<int>(mv_blocks_x), static_cast<int>(mv_blocks_y), static_cast<int>(mv_step), luma_fields != 0,
        reinterpret_cast<float*>(records), static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess)
        return fail(AVD_ERR_GPU, std::string("noise compensated stats launch: ") + cudaGetErrorString(e));
    return AVD_OK;
}

AvdStatus avd_noise_reading(uint64_t records, uint32_t channels, uint32_t width, uint32_t height, uint32_t curve,
                            uint64_t scratch, uint64_t reading, void* stream) {
    if (!reading || (records && !scratch)) return fail(AVD_ERR_NULL_ARG, "noise reading: null buffer");
    if (channels < 1 || channels > 2 || width == 0 || height == 0)
        return fail(AVD_ERR_INVALID_GEOMETRY, "noise reading: bad geometry");
    const uint32_t blocks = ((width + 15) / 16) * ((height + 15) / 16);
    cudaError_t e = avd::launch_noise_reading(reinterpret_cast<const float*>(records), static_cast<int>(channels),
                                              static_cast<int>(width), static_cast<int>(height),
                                              reinterpret_cast<float*>(scratch), avd::min_static_blocks(blocks),
                                              curve != 0, reinterpret_cast<float*>(reading),
                                              static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, std::string("noise reading launch: ") + cudaGetErrorString(e));
    return AVD_OK;
}

void avd_noise_fold_words(uint32_t width, uint32_t height, float sigma_scale, uint32_t curve_applies,
                          float weight_g_max, float weight_floor, uint32_t h2_auto, float h2_per_inverse_variance,
                          float h2_fixed, float pilot_h2_factor, float offset_per_variance, uint32_t main_offset,
                          float sad_per_sigma, float confidence_sad_per_sigma, float* out16) {
    if (!out16) return;
    avd::FoldCoefficients k{};
    k.sigma_scale = sigma_scale;
    k.curve_applies = curve_applies != 0;
    k.weight_g_max = weight_g_max;
    k.weight_floor = weight_floor;
    k.h2_auto = h2_auto != 0;
    k.h2_per_inverse_variance = h2_per_inverse_variance;
    k.h2_fixed = h2_fixed;
    k.pilot_h2_factor = pilot_h2_factor;
    k.offset_per_variance = offset_per_variance;
    k.main_offset = main_offset != 0;
    k.sad_per_sigma = sad_per_sigma;
    k.confidence_sad_per_sigma = confidence_sad_per_sigma;
    avd::noise_fold_words(width, height, k, out16);
}

AvdStatus avd_noise_fold(uint64_t records, uint64_t results, uint32_t capacity, uint32_t first, uint32_t last,
                         uint64_t settings, uint32_t channels, uint32_t table_radius, uint64_t state, uint64_t derived,
                         uint64_t spatial_table, uint64_t pilot_table, void* stream) {
    if (!records || !results || !settings || !state || !derived || (table_radius && (!spatial_table || !pilot_table)))
        return fail(AVD_ERR_NULL_ARG, "noise fold: null buffer");
    if (last < first || last - first + 1 > 17 || last - first + 1 > capacity || channels < 1 || channels > 2 ||
        table_radius > 8)
        return fail(AVD_ERR_INVALID_OPTIONS, "noise fold: bad window");
    cudaError_t e = avd::launch_noise_fold(
        reinterpret_cast<const float*>(records), reinterpret_cast<const float*>(results), static_cast<int>(capacity),
        static_cast<int>(first), static_cast<int>(last), reinterpret_cast<const float*>(settings),
        static_cast<int>(channels), static_cast<int>(table_radius), reinterpret_cast<float*>(state),
        reinterpret_cast<float*>(derived), reinterpret_cast<float*>(spatial_table), reinterpret_cast<float*>(pilot_table),
        static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, std::string("noise fold launch: ") + cudaGetErrorString(e));
    return AVD_OK;
}

}  // extern "C"
