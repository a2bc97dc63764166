// Host side of the batched NLMeans entry point: many clips' frames of uneven size, window and
// strength denoised by one persistent launch. The job table, tile prefix and strength words go to
// the caller's scratch in one copy; the kernel then takes tiles from one counter
// (nlm.cu, `nlm_batch_kernel`).

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "avd_internal.h"
#include "kernels.h"

void avd_set_last_error(const std::string& m);

namespace {

AvdStatus fail(AvdStatus s, const std::string& m) {
    avd_set_last_error(m);
    return s;
}

size_t align16(size_t n) { return (n + 15) / 16 * 16; }

struct Layout {
    size_t prefix, jobs, words, total, words_per_job;
};

Layout layout_for(size_t n, uint32_t search_radius) {
    Layout l{};
    const size_t side = 2 * static_cast<size_t>(search_radius) + 1;
    l.words_per_job = 8 + side * side;
    l.prefix = 16;
    l.jobs = align16(l.prefix + (n + 1) * sizeof(int));
    l.words = align16(l.jobs + n * sizeof(avd::NlmLaunch));
    l.total = align16(l.words + n * l.words_per_job * sizeof(float));
    return l;
}

}  // namespace

extern "C" {

uint64_t avd_batch_scratch_bytes(size_t n_jobs, uint32_t search_radius) {
    return layout_for(n_jobs, search_radius).total;
}

AvdStatus avd_batch_submit(const AvdBatchJob* jobs, size_t n_jobs, uint32_t channels, uint32_t search_radius,
                           uint32_t patch_radius, float self_weight, uint64_t scratch, void* stream) {
    if (!jobs || !scratch) return fail(AVD_ERR_NULL_ARG, "batch: null jobs or scratch");
    if (n_jobs == 0) return AVD_OK;
    if (channels < 1 || channels > 2) return fail(AVD_ERR_INVALID_OPTIONS, "batch: channels must be 1 or 2");
    if (search_radius > avd::kMaxSearchRadius || patch_radius > avd::kMaxPatchRadius)
        return fail(AVD_ERR_INVALID_OPTIONS, "batch: radius past the NLMeans limits");
    const Layout L = layout_for(n_jobs, search_radius);
    std::vector<unsigned char> host(L.total, 0);
    int* prefix = reinterpret_cast<int*>(host.data() + L.prefix);
    auto* launches = reinterpret_cast<avd::NlmLaunch*>(host.data() + L.jobs);
    float* words = reinterpret_cast<float*>(host.data() + L.words);
    const auto dev_base = static_cast<uintptr_t>(scratch);
    const int side = 2 * static_cast<int>(search_radius) + 1;
    const int ty = avd::nlm_tile_rows(static_cast<int>(channels), static_cast<int>(patch_radius));
    const int tx = avd::nlm_tile_cols();
    bool fast = true;
    for (size_t j = 0; j < n_jobs; ++j) fast = fast && jobs[j].pair_offset == 0.0f && jobs[j].spatial_offset == 0.0f;
    int tiles = 0, max_pairs = 0;
    const float area = static_cast<float>((2 * patch_radius + 1) * (2 * patch_radius + 1));
    for (size_t j = 0; j < n_jobs; ++j) {
        const AvdBatchJob& b = jobs[j];
        if (!b.frames || !b.out) return fail(AVD_ERR_NULL_ARG, "batch: a job has a null buffer");
        if (b.width < avd::kMinFrameDim || b.height < avd::kMinFrameDim || b.n_frames == 0 || b.centre >= b.n_frames)
            return fail(AVD_ERR_INVALID_GEOMETRY, "batch: job " + std::to_string(j) + " has a bad geometry");
        if (b.temporal_radius > avd::kMaxTemporalRadius)
            return fail(AVD_ERR_INVALID_OPTIONS, "batch: job " + std::to_string(j) + " has a temporal radius past 8");
        if (!(b.strength > 0.0f))
            return fail(AVD_ERR_INVALID_OPTIONS, "batch: job " + std::to_string(j) + " needs a positive strength");
        prefix[j] = tiles;
        tiles += ((static_cast<int>(b.width) + tx - 1) / tx) * ((static_cast<int>(b.height) + ty - 1) / ty);
        float* w = words + j * L.words_per_job;
        // nlmeans/params.rs:229-233 in the forward's f32 order; the flat spatial table is 0 at q = 0.
        w[0] = (255.0f * 255.0f) / ((3.0f * b.strength * b.strength) * area);
        w[1] = b.pair_offset;
        for (int i = 0; i < side * side; ++i) w[8 + i] = i == (side * side) / 2 ? 0.0f : b.spatial_offset;
        avd::NlmLaunch& a = launches[j];
        std::memset(&a, 0, sizeof(a));
        const int d = static_cast<int>(b.temporal_radius), n = static_cast<int>(b.n_frames), c = static_cast<int>(b.centre);
        a.ring = reinterpret_cast<const float*>(b.frames);
        a.width = static_cast<int>(b.width);
        a.height = static_cast<int>(b.height);
        a.channels = static_cast<int>(channels);
        a.frame_elems = static_cast<int64_t>(b.width) * b.height * channels;
        // Repeat edges (nlmeans/denoiser/ring.rs:103-146): window frame k is clamp(c - d + k).
        a.slot_centre = c;
        a.pairs = d;
        for (int k = 0; k < d; ++k) {
            a.slot_fwd[k] = std::min(std::max(c - d + k, 0), n - 1);
            a.slot_bwd[k] = std::min(std::max(c + d - k, 0), n - 1);
        }
        a.patch_radius = static_cast<int>(patch_radius);
        a.search_radius = static_cast<int>(search_radius);
        a.derived = reinterpret_cast<const float*>(dev_base + L.words + j * L.words_per_job * sizeof(float));
        a.h2_word = 0;
        a.offset_word = 1;
        a.spatial_lut = fast ? nullptr : a.derived + 8;
        a.conf = nullptr;
        a.wref = self_weight;
        a.fast = fast ? 1 : 0;
        a.out = reinterpret_cast<float*>(b.out);
        max_pairs = std::max(max_pairs, d);
    }
    prefix[n_jobs] = tiles;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(reinterpret_cast<void*>(scratch), host.data(), L.total, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, std::string("batch upload: ") + cudaGetErrorString(e));
    e = avd::launch_nlm_batch(reinterpret_cast<const avd::NlmLaunch*>(dev_base + L.jobs),
                              reinterpret_cast<const int*>(dev_base + L.prefix), static_cast<int>(n_jobs),
                              reinterpret_cast<int*>(dev_base), static_cast<int>(channels),
                              static_cast<int>(patch_radius), fast, static_cast<int>(search_radius), max_pairs, s);
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, std::string("batch launch: ") + cudaGetErrorString(e));
    // The staging copy above is pageable: cudaMemcpyAsync has consumed `host` before returning.
    return AVD_OK;
}

namespace {

struct IngestLayout {
    size_t items, prefix, total;
};

IngestLayout ingest_layout(size_t n) {
    IngestLayout l{};
    l.items = 0;
    l.prefix = align16(n * sizeof(avd::BatchIngestItem));
    l.total = align16(l.prefix + (n + 1) * sizeof(int64_t));
    return l;
}

}  // namespace

uint64_t avd_batch_ingest_scratch_bytes(size_t n_items) { return ingest_layout(n_items).total; }

AvdStatus avd_batch_ingest(const AvdBatchIngest* items, size_t n_items, uint64_t scratch, void* stream) {
    if (!items || !scratch) return fail(AVD_ERR_NULL_ARG, "batch ingest: null items or scratch");
    if (n_items == 0) return AVD_OK;
    if (n_items > static_cast<size_t>(1) << 30) return fail(AVD_ERR_INVALID_OPTIONS, "batch ingest: too many items");
    const IngestLayout L = ingest_layout(n_items);
    std::vector<unsigned char> host(L.total, 0);
    auto* table = reinterpret_cast<avd::BatchIngestItem*>(host.data() + L.items);
    auto* prefix = reinterpret_cast<int64_t*>(host.data() + L.prefix);
    int64_t words = 0;
    for (size_t i = 0; i < n_items; ++i) {
        const AvdBatchIngest& b = items[i];
        if (!b.plane0 || !b.frame || (b.channels == 2 && !b.plane1))
            return fail(AVD_ERR_NULL_ARG, "batch ingest: item " + std::to_string(i) + " has a null buffer");
        if (b.channels < 1 || b.channels > 2 || b.width == 0 || b.height == 0)
            return fail(AVD_ERR_INVALID_GEOMETRY, "batch ingest: item " + std::to_string(i) + " has a bad geometry");
        if (b.bits < 8 || b.bits > 16)
            return fail(AVD_ERR_INVALID_OPTIONS, "batch ingest: item " + std::to_string(i) + " has bits outside 8..16");
        avd::BatchIngestItem& t = table[i];
        t.plane0 = reinterpret_cast<const uint32_t*>(b.plane0);
        t.plane1 = reinterpret_cast<const uint32_t*>(b.plane1);
        t.dst = reinterpret_cast<float*>(b.frame);
        t.pixels = static_cast<int64_t>(b.width) * b.height;
        t.channels = static_cast<int>(b.channels);
        t.samples_per_word = b.bits == 8 ? 4 : 2;
        t.max_value = static_cast<float>((1u << b.bits) - 1u);
        prefix[i] = words;
        words += (t.pixels + t.samples_per_word - 1) / t.samples_per_word;
    }
    prefix[n_items] = words;
    auto s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(reinterpret_cast<void*>(scratch), host.data(), L.total, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        auto* dev = reinterpret_cast<unsigned char*>(scratch);
        e = avd::launch_batch_ingest(reinterpret_cast<const avd::BatchIngestItem*>(dev + L.items),
                                     reinterpret_cast<const int64_t*>(dev + L.prefix), static_cast<int>(n_items), words,
                                     s);
    }
    // The staging copy above is pageable: cudaMemcpyAsync has consumed `host` before returning.
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, std::string("batch ingest: ") + cudaGetErrorString(e));
    return AVD_OK;
}

}  // extern "C"
