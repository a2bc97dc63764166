// One NLMeans frame with no device allocation, for callers that cannot call cudaMalloc.
//
// Some hosts of this library cannot allocate device memory on their own terms: a plugin
// running inside another application's CUDA context whose allocations that application owns, a
// real-time video path that must never hit the driver's allocator mid-stream, or a sandbox that
// forbids the allocation calls outright. `avd_nlm_frame_static` serves them: the caller passes
// the window's input planes and the output planes, and the engine's scratch (the normalised f32
// frames, the f32 result and the strength words) lives in one file-scope device array of fixed
// size, which every GPU that loads the library holds until the process exits.
//
// The array is shared by every call on a device and keeps the last call's contents. Every word a
// call reads is first written by the same call (the frames by the ingest, the result by the
// window kernel, the strength words by a one-thread kernel), except the count of samples the exact
// finish recomputes, which each call clears first; two calls whose GPU work overlaps (two streams,
// or two host threads) race on the array.
//
// The array's address for host code comes from cudaGetSymbolAddress, taken with the device
// current on the first call made in each CUDA context on that device (the process's primary
// context, an application's own context, or the new primary context after a cudaDeviceReset: a
// context is told apart by its driver-issued id, which is never reused); make that first call
// before any stream capture.

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>

#include "avd_internal.h"
#include "kernels.h"

void avd_set_last_error(const std::string& m);

namespace avd {

namespace {

// 32 MiB: the frames, result, 64 strength words and (integer outputs) the exact finish's count and
// pixel list of one call must fit.
constexpr size_t kStaticScratchBytes = size_t(32) << 20;
constexpr size_t kStaticScratchFloats = kStaticScratchBytes / sizeof(float);
constexpr size_t kWordsFloats = 64;
constexpr int kMaxDevices = 64;

__device__ __align__(256) float g_nlm_scratch[kStaticScratchFloats];

std::mutex g_setup_mutex;
struct SetupRecord {
    unsigned long long context_id;  // the CUDA context the address was taken in (0: none yet)
    float* ptr;
};
SetupRecord g_setup[kMaxDevices] = {};

// cuCtxGetCurrent and cuCtxGetId, reached through the runtime so the library needs no link to the
// driver library; resolved once.
using CtxGetCurrentFn = int (*)(void**);
using CtxGetIdFn = int (*)(void*, unsigned long long*);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

__global__ void write_strength_words(float* words, float h2, float offset) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        words[0] = h2;
        words[1] = offset;
    }
}

AvdStatus fail(AvdStatus st, const std::string& m) {
    avd_set_last_error(m);
    return st;
}

// The id of the calling thread's current CUDA context (0 when none is bound yet). Caller holds
// g_setup_mutex.
cudaError_t current_context_id(unsigned long long* id) {
    if (g_ctx_get_current == nullptr || g_ctx_get_id == nullptr) {
        void* f0 = nullptr;
        void* f1 = nullptr;
        cudaDriverEntryPointQueryResult q0{}, q1{};
        cudaError_t e = cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f0, 12000, cudaEnableDefault, &q0);
        if (e == cudaSuccess) e = cudaGetDriverEntryPointByVersion("cuCtxGetId", &f1, 12000, cudaEnableDefault, &q1);
        if (e != cudaSuccess) return e;
        if (q0 != cudaDriverEntryPointSuccess || q1 != cudaDriverEntryPointSuccess || !f0 || !f1)
            return cudaErrorSymbolNotFound;
        g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f0);
        g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f1);
    }
    void* ctx = nullptr;
    if (g_ctx_get_current(&ctx) != 0) return cudaErrorDeviceUninitialized;
    *id = 0;
    if (ctx != nullptr && g_ctx_get_id(ctx, id) != 0) return cudaErrorDeviceUninitialized;
    return cudaSuccess;
}

// The device address of the scratch array in the current context of the current device, taken
// once per device and context.
cudaError_t scratch_for_current_device(float** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    unsigned long long id = 0;
    if ((e = current_context_id(&id)) != cudaSuccess) return e;
    SetupRecord& rec = g_setup[dev];
    if (rec.ptr == nullptr || id == 0 || rec.context_id != id) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_nlm_scratch);  // binds the primary context when none was
        if (e != cudaSuccess) return e;
        if ((e = current_context_id(&id)) != cudaSuccess) return e;
        rec.ptr = static_cast<float*>(ptr);
        rec.context_id = id;
    }
    *out = rec.ptr;
    return cudaSuccess;
}

PlaneFormat plane_format_of(const AvdSampleFormat& f) {
    PlaneFormat p;
    p.kind = static_cast<int>(f.kind);
    p.samples_per_word = static_cast<int>(samples_per_word(f));
    p.max_value = sample_max_value(f);
    return p;
}

}  // namespace

}  // namespace avd

using namespace avd;

extern "C" AvdStatus avd_nlm_frame_static(const AvdNlmeansAlgorithm* algorithm, uint32_t channels, uint32_t width,
                                          uint32_t height, AvdSampleFormat input, AvdSampleFormat output,
                                          const AvdPlane* window, size_t n_window, const AvdPlane* out,
                                          size_t n_out, void* stream) {
    if (!algorithm || !window || !out) return AVD_ERR_NULL_ARG;
    avd_set_last_error("");
    if (channels != 1 && channels != 2) return fail(AVD_ERR_INVALID_OPTIONS, "channels must be 1 (luma) or 2 (chroma)");
    if (algorithm->variant != 0)
        return fail(AVD_ERR_INVALID_OPTIONS, "the allocation-free entry point runs the fast NLMeans variant only");
    for (const AvdSampleFormat* f : {&input, &output}) {
        if (f->kind > AVD_SAMPLE_F32 || (f->kind == AVD_SAMPLE_U16 && (f->depth < 9 || f->depth > 16)))
            return fail(AVD_ERR_INVALID_GEOMETRY, "unsupported sample format");
    }
    if (width < kMinFrameDim || height < kMinFrameDim)
        return fail(AVD_ERR_INVALID_GEOMETRY, "frame dimensions are below the supported minimum of 3x3");
    const Channels ch = channels == 1 ? Channels::Luma : Channels::Chroma;
    const NlmParams p = resolve_nlm_params(*algorithm, ch);
    std::string bad = validate_nlm_params(p);
    if (!bad.empty()) return fail(AVD_ERR_INVALID_OPTIONS, bad);
    if (p.prefilter.kind != AVD_PREFILTER_NONE || (p.motion.active && p.temporal_radius > 0))
        return fail(AVD_ERR_INVALID_OPTIONS, "the allocation-free entry point runs without prefilter or motion");

    const uint32_t frames = p.total_frames();
    if (n_window != static_cast<size_t>(frames) * channels)
        return fail(AVD_ERR_PLANE_MISMATCH, "the window needs (2 * temporal_radius + 1) * channels planes");
    if (n_out != channels) return fail(AVD_ERR_PLANE_MISMATCH, "the output needs `channels` planes");
    const uint64_t pixels = static_cast<uint64_t>(width) * height;
    const uint64_t frame_elems = pixels * channels;
    const bool integer_out = output.kind != AVD_SAMPLE_F32;
    const uint64_t need = kWordsFloats + frame_elems * (frames + 1) + (integer_out ? pixels + 1 : 0);
    if (need > kStaticScratchFloats) {
        char m[256];
        std::snprintf(m, sizeof(m),
                      "a %ux%u frame with %u channel(s) and a %u-frame window needs %llu bytes of scratch, "
                      "past the fixed %zu-byte array of the allocation-free entry point",
                      width, height, channels, frames, (unsigned long long)(need * sizeof(float)),
                      kStaticScratchBytes);
        return fail(AVD_ERR_INVALID_GEOMETRY, m);
    }
    const uint64_t in_bytes = plane_bytes(input, pixels), out_bytes = plane_bytes(output, pixels);
    for (size_t i = 0; i < n_window; ++i)
        if (window[i].width != width || window[i].height != height || window[i].bytes < in_bytes || !window[i].ptr)
            return fail(AVD_ERR_PLANE_MISMATCH, "a window plane does not match the frame size");
    for (size_t i = 0; i < n_out; ++i)
        if (out[i].width != width || out[i].height != height || out[i].bytes < out_bytes || !out[i].ptr)
            return fail(AVD_ERR_PLANE_MISMATCH, "an output plane does not match the frame size");

    float* scratch = nullptr;
    cudaError_t e = scratch_for_current_device(&scratch);
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float* words = scratch;
    float* ring = scratch + kWordsFloats;
    float* result = ring + frame_elems * frames;
    const float bias = (ch == Channels::Chroma) ? 0.5f : 0.0f;

    write_strength_words<<<1, 32, 0, s>>>(words, h2_inv_norm_with(p, false, 0.0f), 0.0f);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(AVD_ERR_GPU, cudaGetErrorString(e));
    for (uint32_t f = 0; f < frames; ++f) {
        const void* p0 = reinterpret_cast<const void*>(window[f * channels].ptr);
        const void* p1 = reinterpret_cast<const void*>(window[f * channels + channels - 1].ptr);
        e = launch_ingest(p0, p1, ring + f * frame_elems, static_cast<int64_t>(pixels), static_cast<int>(channels),
                          plane_format_of(input), bias, s);
        if (e != cudaSuccess) return fail(AVD_ERR_GPU, cudaGetErrorString(e));
    }
    const int d = static_cast<int>(p.temporal_radius);
    NlmLaunch a{};
    a.ring = ring;
    a.width = static_cast<int>(width);
    a.height = static_cast<int>(height);
    a.channels = static_cast<int>(channels);
    a.frame_elems = static_cast<int64_t>(frame_elems);
    a.slot_centre = d;
    a.pairs = d;
    for (int k = 0; k < d; ++k) {
        a.slot_fwd[k] = k;          // centre + q_k with q_k = -d + k
        a.slot_bwd[k] = 2 * d - k;  // centre - q_k
    }
    a.patch_radius = static_cast<int>(p.patch_radius);
    a.search_radius = static_cast<int>(p.search_radius);
    a.derived = words;
    a.h2_word = 0;
    a.offset_word = 1;
    a.wref = p.self_weight;
    a.fast = 1;
    a.out = result;
    if (integer_out) {
        // The exact finish of the samples near a change of code, as the engine runs it; the count
        // is the one word of the array that must start at zero, so every call clears it.
        a.fix_count = reinterpret_cast<int*>(result + frame_elems);
        a.fix_list = a.fix_count + 1;
        a.code_max = sample_max_value(output);
        a.fix_band = kFixBand;
        if ((e = cudaMemsetAsync(a.fix_count, 0, sizeof(int), s)) != cudaSuccess)
            return fail(AVD_ERR_GPU, cudaGetErrorString(e));
    }
    if ((e = launch_nlm(a, s)) != cudaSuccess) return fail(AVD_ERR_GPU, cudaGetErrorString(e));
    if (integer_out && (e = launch_nlm_exact(a, s)) != cudaSuccess) return fail(AVD_ERR_GPU, cudaGetErrorString(e));
    void* o0 = reinterpret_cast<void*>(out[0].ptr);
    void* o1 = reinterpret_cast<void*>(out[channels - 1].ptr);
    e = launch_egress(result, o0, o1, static_cast<int64_t>(pixels), static_cast<int>(channels),
                      plane_format_of(output), bias, s);
    if (e != cudaSuccess) return fail(AVD_ERR_GPU, cudaGetErrorString(e));
    return AVD_OK;
}
