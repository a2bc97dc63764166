// The host denoiser: an engine fed from host memory (av-denoise/src/host/mod.rs:111-420), built on
// the engine's own C ABI as the reference builds `HostDenoiser` on the `Engine` trait.
//
// Each frame's wire planes are copied into one of two pinned input sets and uploaded on a copy
// stream into that set's device planes, so the upload of frame n+1 overlaps the engine's work on
// frame n; the engine's stream waits for the upload, and the set is reused only after the engine
// has ingested it (events both ways). Denoised frames are emitted into one of two device output
// sets and read back into pinned memory on a third stream, so the readback of frame n overlaps the
// engine's work on frame n+1; `recv` waits on that readback's event. At most two frames are in
// flight (MAX_PENDING = OUTPUT_SETS = 2, mod.rs:27-33).

#include <cuda_runtime.h>

#include <chrono>
#include <cstring>
#include <deque>
#include <string>
#include <vector>

#include "avd_internal.h"

namespace {

constexpr size_t kMaxPending = 2;
constexpr size_t kSets = 2;

struct InputSet {
    std::vector<void*> dev;
    unsigned char* pinned = nullptr;
    cudaEvent_t uploaded = nullptr, consumed = nullptr;
    bool used = false;
};

struct OutputSet {
    std::vector<void*> dev;
    unsigned char* pinned = nullptr;
    cudaEvent_t emitted = nullptr, landed = nullptr;
    bool used = false;
};

}  // namespace

struct AvdHost {
    AvdEngine* engine = nullptr;
    AvdGeometry geometry{};
    size_t planes = 0;
    std::vector<uint32_t> width, height;
    std::vector<uint64_t> wire_in, wire_out, dev_in, dev_out;  // bytes per plane
    uint64_t pinned_in = 0, pinned_out = 0;                     // bytes per set
    cudaStream_t compute = nullptr, copy = nullptr, readback = nullptr;
    InputSet in[kSets];
    OutputSet out[kSets];
    size_t next_in = 0, next_out = 0;
    std::deque<size_t> pending;
    bool poisoned = false;
    std::string error;
    int device = 0;
    double call_time = 0, output_wait = 0, sink_time = 0;  // seconds (mod.rs:131-137)
    uint64_t frames_emitted = 0;

    ~AvdHost() {
        if (compute) cudaStreamSynchronize(compute);
        if (copy) cudaStreamSynchronize(copy);
        if (readback) cudaStreamSynchronize(readback);
        if (engine) avd_engine_destroy(engine);
        for (auto& s : in) {
            for (void* p : s.dev) cudaFree(p);
            if (s.pinned) cudaFreeHost(s.pinned);
            if (s.uploaded) cudaEventDestroy(s.uploaded);
            if (s.consumed) cudaEventDestroy(s.consumed);
        }
        for (auto& s : out) {
            for (void* p : s.dev) cudaFree(p);
            if (s.pinned) cudaFreeHost(s.pinned);
            if (s.emitted) cudaEventDestroy(s.emitted);
            if (s.landed) cudaEventDestroy(s.landed);
        }
        if (compute) cudaStreamDestroy(compute);
        if (copy) cudaStreamDestroy(copy);
        if (readback) cudaStreamDestroy(readback);
    }
};

namespace {

thread_local std::string g_host_error;

AvdStatus fail(AvdHost* h, AvdStatus s, const std::string& m, bool poison) {
    if (h) {
        h->error = m;
        if (poison) h->poisoned = true;
    } else {
        g_host_error = m;
    }
    return s;
}

AvdStatus cuda_fail(AvdHost* h, const char* what, cudaError_t e) {
    return fail(h, AVD_ERR_GPU, std::string(what) + ": " + cudaGetErrorString(e), true);
}

// An engine call's failure, with the engine's own message. Everything but a context frame sent
// after a push may leave the stream part-advanced, so it poisons (mod.rs:60-75).
AvdStatus engine_fail(AvdHost* h, AvdStatus s) {
    const char* m = avd_engine_last_error(h->engine);
    return fail(h, s, m && *m ? m : avd_status_message(s), s != AVD_ERR_CONTEXT_AFTER_PUSH);
}

double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Adds the time from construction to destruction to `*acc` (`clocked`, mod.rs:398-405).
struct Clock {
    double* acc;
    double t0;
    explicit Clock(double* a) : acc(a), t0(now()) {}
    ~Clock() { *acc += now() - t0; }
};

struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(int d) {
        if (cudaGetDevice(&prev) == cudaSuccess && prev != d) cudaSetDevice(d);
        else prev = -1;
    }
    ~DeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

std::vector<AvdPlane> set_planes(const AvdHost* h, const std::vector<void*>& dev, const std::vector<uint64_t>& bytes) {
    std::vector<AvdPlane> p(h->planes);
    for (size_t i = 0; i < h->planes; ++i) p[i] = AvdPlane{reinterpret_cast<uint64_t>(dev[i]), bytes[i], h->width[i], h->height[i]};
    return p;
}

uint64_t wire_bytes(const AvdSampleFormat& f, uint64_t pixels) {
    return pixels * (f.kind == AVD_SAMPLE_U8 ? 1u : (f.kind == AVD_SAMPLE_U16 ? 2u : 4u));
}

// Stages one frame and uploads it into the next input set; the engine's stream then waits for it.
AvdStatus upload(AvdHost* h, const void* const* planes, const uint64_t* bytes, size_t n, size_t* set_out) {
    if (n != h->planes)
        return fail(h, AVD_ERR_PLANE_MISMATCH,
                    "expected " + std::to_string(h->planes) + " planes, got " + std::to_string(n), false);
    for (size_t i = 0; i < n; ++i) {
        if (!planes[i]) return fail(h, AVD_ERR_NULL_ARG, "a plane is null", false);
        if (bytes[i] != h->wire_in[i])
            return fail(h, AVD_ERR_PLANE_MISMATCH,
                        "plane " + std::to_string(i) + " holds " + std::to_string(bytes[i]) + " bytes, expected " +
                            std::to_string(h->wire_in[i]),
                        false);
    }
    const size_t k = h->next_in;
    h->next_in = (k + 1) % kSets;
    InputSet& s = h->in[k];
    cudaError_t e;
    if (s.used && (e = cudaEventSynchronize(s.uploaded)) != cudaSuccess) return cuda_fail(h, "input staging", e);
    size_t off = 0;
    for (size_t i = 0; i < n; ++i) {
        std::memcpy(s.pinned + off, planes[i], h->wire_in[i]);
        std::memset(s.pinned + off + h->wire_in[i], 0, h->dev_in[i] - h->wire_in[i]);
        off += h->dev_in[i];
    }
    if (s.used && (e = cudaStreamWaitEvent(h->copy, s.consumed, 0)) != cudaSuccess) return cuda_fail(h, "input reuse", e);
    off = 0;
    for (size_t i = 0; i < n; ++i) {
        if ((e = cudaMemcpyAsync(s.dev[i], s.pinned + off, h->dev_in[i], cudaMemcpyHostToDevice, h->copy)) != cudaSuccess)
            return cuda_fail(h, "upload", e);
        off += h->dev_in[i];
    }
    if ((e = cudaEventRecord(s.uploaded, h->copy)) != cudaSuccess) return cuda_fail(h, "upload event", e);
    if ((e = cudaStreamWaitEvent(h->compute, s.uploaded, 0)) != cudaSuccess) return cuda_fail(h, "upload wait", e);
    s.used = true;
    *set_out = k;
    return AVD_OK;
}

AvdStatus mark_consumed(AvdHost* h, size_t k) {
    cudaError_t e = cudaEventRecord(h->in[k].consumed, h->compute);
    return e == cudaSuccess ? AVD_OK : cuda_fail(h, "ingest event", e);
}

// Emits the engine's next frame into output set `slot` and queues its readback. The set's last
// readback has landed before it is written again (the host waited on it in `recv` or `flush`; the
// engine's stream also waits on its event).
AvdStatus emit_into_slot(AvdHost* h, size_t slot) {
    OutputSet& o = h->out[slot];
    cudaError_t e;
    if (o.used && (e = cudaStreamWaitEvent(h->compute, o.landed, 0)) != cudaSuccess) return cuda_fail(h, "output reuse", e);
    std::vector<AvdPlane> planes = set_planes(h, o.dev, h->dev_out);
    AvdStatus st = avd_engine_emit_into(h->engine, planes.data(), planes.size());
    if (st != AVD_OK) return engine_fail(h, st);
    if ((e = cudaEventRecord(o.emitted, h->compute)) != cudaSuccess) return cuda_fail(h, "emit event", e);
    if ((e = cudaStreamWaitEvent(h->readback, o.emitted, 0)) != cudaSuccess) return cuda_fail(h, "emit wait", e);
    size_t off = 0;
    for (size_t i = 0; i < h->planes; ++i) {
        if ((e = cudaMemcpyAsync(o.pinned + off, o.dev[i], h->wire_out[i], cudaMemcpyDeviceToHost, h->readback)) !=
            cudaSuccess)
            return cuda_fail(h, "readback", e);
        off += h->wire_out[i];
    }
    if ((e = cudaEventRecord(o.landed, h->readback)) != cudaSuccess) return cuda_fail(h, "readback event", e);
    o.used = true;
    return AVD_OK;
}

AvdStatus wait_for(AvdHost* h, size_t slot) {
    cudaError_t e;
    {
        Clock c(&h->output_wait);
        e = cudaEventSynchronize(h->out[slot].landed);
    }
    if (e != cudaSuccess) return cuda_fail(h, "readback wait", e);
    ++h->frames_emitted;
    return AVD_OK;
}

void hand_to_sink(AvdHost* h, AvdHostSink sink, void* user, const std::vector<const void*>& v) {
    Clock c(&h->sink_time);
    sink(user, v.data(), v.size());
}

std::vector<const void*> slot_views(const AvdHost* h, size_t slot) {
    std::vector<const void*> v(h->planes);
    size_t off = 0;
    for (size_t i = 0; i < h->planes; ++i) {
        v[i] = h->out[slot].pinned + off;
        off += h->wire_out[i];
    }
    return v;
}

}  // namespace

extern "C" {

AvdStatus avd_host_create(const AvdEngineSpec* spec, const AvdTuning* tuning, AvdHost** out) {
    if (!spec || !out) return AVD_ERR_NULL_ARG;
    *out = nullptr;
    auto h = new AvdHost();
    AvdStatus st = avd_engine_create(spec, tuning, &h->engine);
    if (st != AVD_OK) {
        g_host_error = avd_last_error();
        delete h;
        return st;
    }
    h->geometry = spec->geometry;
    cudaGetDevice(&h->device);
    const AvdGeometry& g = spec->geometry;
    h->planes = avd::plane_count(g.chroma);
    cudaError_t e = cudaStreamCreateWithFlags(&h->compute, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->copy, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->readback, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        g_host_error = cudaGetErrorString(e);
        delete h;
        return AVD_ERR_GPU;
    }
    avd_engine_set_stream(h->engine, h->compute);
    for (size_t i = 0; i < h->planes; ++i) {
        uint32_t w, ht;
        avd::plane_dims(g, i, &w, &ht);
        h->width.push_back(w);
        h->height.push_back(ht);
        const uint64_t px = static_cast<uint64_t>(w) * ht;
        h->wire_in.push_back(wire_bytes(g.input, px));
        h->wire_out.push_back(wire_bytes(g.output, px));
        h->dev_in.push_back(avd::plane_bytes(g.input, px));
        h->dev_out.push_back(avd::plane_bytes(g.output, px));
        h->pinned_in += h->dev_in.back();
        h->pinned_out += h->wire_out.back();
    }
    for (auto& s : h->in) {
        for (size_t i = 0; i < h->planes && e == cudaSuccess; ++i) {
            void* p = nullptr;
            e = cudaMalloc(&p, h->dev_in[i]);
            s.dev.push_back(p);
        }
        if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&s.pinned), h->pinned_in);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.uploaded, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.consumed, cudaEventDisableTiming);
    }
    for (auto& s : h->out) {
        for (size_t i = 0; i < h->planes && e == cudaSuccess; ++i) {
            void* p = nullptr;
            e = cudaMalloc(&p, h->dev_out[i]);
            s.dev.push_back(p);
        }
        if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&s.pinned), h->pinned_out);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.emitted, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.landed, cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        g_host_error = std::string("host denoiser buffers: ") + cudaGetErrorString(e);
        delete h;
        return AVD_ERR_GPU;
    }
    *out = h;
    return AVD_OK;
}

void avd_host_destroy(AvdHost* h) {
    if (!h) return;
    DeviceScope ds(h->device);
    delete h;
}

uint64_t avd_host_plane_bytes(const AvdHost* h, size_t index) {
    return h && index < h->planes ? h->wire_out[index] : 0;
}

AvdStatus avd_host_push(AvdHost* h, const void* const* planes, const uint64_t* bytes, size_t n) {
    if (!h || !planes || !bytes) return AVD_ERR_NULL_ARG;
    DeviceScope ds(h->device);
    Clock clock(&h->call_time);
    if (h->poisoned) return fail(h, AVD_ERR_POISONED, avd_status_message(AVD_ERR_POISONED), false);
    if (h->pending.size() >= kMaxPending) return fail(h, AVD_ERR_QUEUE_FULL, avd_status_message(AVD_ERR_QUEUE_FULL), false);
    size_t k = 0;
    if (AvdStatus st = upload(h, planes, bytes, n, &k)) return st;
    std::vector<AvdPlane> dev = set_planes(h, h->in[k].dev, h->dev_in);
    size_t ready = 0;
    AvdStatus st = avd_engine_push(h->engine, dev.data(), dev.size(), &ready);
    if (st != AVD_OK) return engine_fail(h, st);
    if (AvdStatus m = mark_consumed(h, k)) return m;
    // mod.rs:273-282: emitting past the free output sets would overwrite a readback in flight.
    if (h->pending.size() + ready > kSets)
        return fail(h, AVD_ERR_GPU,
                    "push readied " + std::to_string(ready) + " frames with " + std::to_string(h->pending.size()) +
                        " in flight, past the 2 output sets",
                    true);
    for (size_t i = 0; i < ready; ++i) {
        const size_t slot = h->next_out;
        h->next_out = (slot + 1) % kSets;
        if (AvdStatus e = emit_into_slot(h, slot)) return e;
        h->pending.push_back(slot);
    }
    return AVD_OK;
}

AvdStatus avd_host_push_priming(AvdHost* h, const void* const* planes, const uint64_t* bytes, size_t n) {
    if (!h || !planes || !bytes) return AVD_ERR_NULL_ARG;
    DeviceScope ds(h->device);
    Clock clock(&h->call_time);
    if (h->poisoned) return fail(h, AVD_ERR_POISONED, avd_status_message(AVD_ERR_POISONED), false);
    size_t k = 0;
    if (AvdStatus st = upload(h, planes, bytes, n, &k)) return st;
    std::vector<AvdPlane> dev = set_planes(h, h->in[k].dev, h->dev_in);
    AvdStatus st = avd_engine_push_context(h->engine, dev.data(), dev.size());
    if (st != AVD_OK) return engine_fail(h, st);
    return mark_consumed(h, k);
}

AvdStatus avd_host_recv(AvdHost* h, void* const* out, size_t n, int* got) {
    if (!h || !out || !got) return AVD_ERR_NULL_ARG;
    DeviceScope ds(h->device);
    Clock clock(&h->call_time);
    *got = 0;
    if (h->poisoned) return fail(h, AVD_ERR_POISONED, avd_status_message(AVD_ERR_POISONED), false);
    if (n != h->planes) return fail(h, AVD_ERR_PLANE_MISMATCH, "recv needs one buffer per plane", false);
    if (h->pending.empty()) return AVD_OK;
    const size_t slot = h->pending.front();
    h->pending.pop_front();
    if (AvdStatus st = wait_for(h, slot)) return st;
    std::vector<const void*> v = slot_views(h, slot);
    for (size_t i = 0; i < n; ++i) std::memcpy(out[i], v[i], h->wire_out[i]);
    *got = 1;
    return AVD_OK;
}

AvdStatus avd_host_flush(AvdHost* h, AvdHostSink sink, void* user) {
    if (!h || !sink) return AVD_ERR_NULL_ARG;
    DeviceScope ds(h->device);
    Clock clock(&h->call_time);
    if (h->poisoned) return fail(h, AVD_ERR_POISONED, avd_status_message(AVD_ERR_POISONED), false);
    while (!h->pending.empty()) {
        const size_t slot = h->pending.front();
        h->pending.pop_front();
        if (AvdStatus st = wait_for(h, slot)) return st;
        hand_to_sink(h, sink, user, slot_views(h, slot));
    }
    size_t tail = 0;
    AvdStatus st = avd_engine_finish(h->engine, &tail);
    if (st != AVD_OK) return engine_fail(h, st);
    for (size_t i = 0; i < tail; ++i) {
        if (AvdStatus e = emit_into_slot(h, 0)) return e;
        if (AvdStatus e = wait_for(h, 0)) return e;
        hand_to_sink(h, sink, user, slot_views(h, 0));
    }
    h->next_out = 0;
    return AVD_OK;
}

void avd_host_reset(AvdHost* h) {
    if (!h) return;
    DeviceScope ds(h->device);
    cudaStreamSynchronize(h->compute);
    cudaStreamSynchronize(h->copy);
    cudaStreamSynchronize(h->readback);
    h->pending.clear();
    avd_engine_reset(h->engine);
    h->next_out = 0;
    h->poisoned = false;
}

AvdStatus avd_host_timing(AvdHost* h, AvdHostTiming* out) {
    if (!h || !out) return AVD_ERR_NULL_ARG;
    DeviceScope ds(h->device);
    AvdPassTimings p{};
    AvdStatus st = avd_engine_timing(h->engine, &p);
    if (st != AVD_OK) return engine_fail(h, st);
    auto busy = [&](const AvdEngineTiming& t) {
        return t.frames ? t.device_time / static_cast<double>(t.frames) * static_cast<double>(h->frames_emitted) : -1.0;
    };
    const double calls = h->call_time - h->sink_time;
    out->blocked = h->output_wait;
    out->submit = calls > h->output_wait ? calls - h->output_wait : 0.0;
    out->frames = h->frames_emitted;
    out->has_luma = p.has_luma;
    out->has_chroma = p.has_chroma;
    out->luma_device_busy = p.has_luma ? busy(p.luma) : -1.0;
    out->chroma_device_busy = p.has_chroma ? busy(p.chroma) : -1.0;
    return AVD_OK;
}

void avd_host_sample_device_time(AvdHost* h, uint32_t every) {
    if (!h) return;
    DeviceScope ds(h->device);
    avd_engine_sample_device_time(h->engine, every);
}

void avd_host_poison_for_test(AvdHost* h) {
    if (h) fail(h, AVD_ERR_POISONED, "poisoned for a test", true);
}

const char* avd_host_last_error(const AvdHost* h) { return h ? h->error.c_str() : g_host_error.c_str(); }

}  // extern "C"
