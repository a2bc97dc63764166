// The launch tuner (tune.h): remembered and stored per-shape choices, and the timing pass.

#include "tune.h"

#include <cuda_runtime.h>

#include "avd_internal.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <vector>

namespace avd {

namespace {

constexpr int kFormat = 1;
const char* kFileName = "av-denoise-b200-tune.jsonl";

struct Remembered {
    std::mutex lock;
    std::map<std::string, int> choices;       // full key -> variant
    std::map<std::string, bool> loaded_dirs;  // store directories already read
};

Remembered& remembered() {
    static Remembered r;
    return r;
}

std::string file_of(const std::string& dir) { return dir + "/" + kFileName; }

std::string escape(const std::string& s) {
    std::string out;
    for (char c : s) {
        if (c == '"' || c == '\\') out.push_back('\\');
        out.push_back(c);
    }
    return out;
}

// One stored line: {"format": 1, "key": "...", "variant": v, "ms": [...]}. Lines of another format
// or that do not parse are skipped.
bool parse_line(const std::string& line, std::string* key, int* variant) {
    int format = 0;
    if (std::sscanf(line.c_str(), "{\"format\": %d,", &format) != 1 || format != kFormat) return false;
    const std::string tag = "\"key\": \"";
    size_t at = line.find(tag);
    if (at == std::string::npos) return false;
    at += tag.size();
    std::string k;
    for (; at < line.size() && line[at] != '"'; ++at) {
        if (line[at] == '\\' && at + 1 < line.size()) ++at;
        k.push_back(line[at]);
    }
    const size_t v = line.find("\"variant\": ", at);
    if (v == std::string::npos) return false;
    *variant = std::atoi(line.c_str() + v + 11);
    *key = k;
    return true;
}

void load_dir(Remembered& r, const std::string& dir) {
    if (dir.empty() || r.loaded_dirs[dir]) return;
    r.loaded_dirs[dir] = true;
    std::ifstream in(file_of(dir));
    std::string line, key;
    int variant = 0;
    while (std::getline(in, line))
        if (parse_line(line, &key, &variant)) r.choices[dir + "|" + key] = variant;
}

void append(const std::string& dir, const std::string& key, int variant, const std::vector<float>& ms) {
    if (dir.empty()) return;
    std::ofstream out(file_of(dir), std::ios::app);
    if (!out) return;  // a store that cannot be written keeps the result for this process only
    std::ostringstream line;
    line << "{\"format\": " << kFormat << ", \"key\": \"" << escape(key) << "\", \"variant\": " << variant
         << ", \"ms\": [";
    for (size_t i = 0; i < ms.size(); ++i) line << (i ? ", " : "") << ms[i];
    line << "]}";
    out << line.str() << "\n";
}

}  // namespace

std::string tune_device_identity() {
    int dev = 0;
    cudaDeviceProp p{};
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&p, dev) != cudaSuccess) return "unknown";
    std::ostringstream id;
    id << p.name << " sm_" << p.major << p.minor << " x" << p.multiProcessorCount;
    return id.str();
}

int tuned_variant(const TuneOptions& options, const std::string& key, int variants,
                  const std::function<float(int)>& time_variant) {
    if (options.mode == TuneMode::Off || variants <= 1) return 0;
    const std::string full = tune_device_identity() + " " + key;
    Remembered& r = remembered();
    {
        std::lock_guard<std::mutex> g(r.lock);
        load_dir(r, options.store);
        auto it = r.choices.find(options.store + "|" + full);
        if (it != r.choices.end()) return it->second < variants ? it->second : 0;
    }
    if (options.mode == TuneMode::Cached) return 0;
    // driver/pass.rs: every variant timed on the site's own launch; the baseline keeps ties.
    std::vector<float> ms(variants, -1.0f);
    int best = 0;
    for (int v = 0; v < variants; ++v) {
        ms[v] = time_variant(v);
        if (ms[v] >= 0.0f && (ms[best] < 0.0f || ms[v] < ms[best])) best = v;
    }
    if (ms[best] < 0.0f) best = 0;
    std::lock_guard<std::mutex> g(r.lock);
    r.choices[options.store + "|" + full] = best;
    append(options.store, full, best, ms);
    return best;
}

void tune_forget() {
    Remembered& r = remembered();
    std::lock_guard<std::mutex> g(r.lock);
    r.choices.clear();
    r.loaded_dirs.clear();
}

}  // namespace avd

// ---- C entry point for the store's tests (include/avd.h) ----------------------------------------

extern "C" int avd_tune_variant_for_test(uint32_t mode, const char* store, const char* key, uint32_t variants,
                                         const float* times_ms) {
    avd::TuneOptions o;
    o.mode = static_cast<avd::TuneMode>(mode > 2 ? 2 : mode);
    if (store) o.store = store;
    return avd::tuned_variant(o, key ? key : "", static_cast<int>(variants),
                              [&](int v) { return times_ms ? times_ms[v] : 0.0f; });
}

extern "C" void avd_tune_forget(void) { avd::tune_forget(); }
