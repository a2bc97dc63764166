// The project's launch tuner (the role of av-denoise-core/src/tune: driver/mod.rs:113 `tune`,
// store.rs `TuneStore`, config.rs:8-75 `TuningMode`/`TuningConfig`). A launch site with several
// variants of one kernel (same results, different launch shapes) asks for the variant of a shape
// key; the tuner answers from the results this process remembers or the store file holds, and in
// Auto mode times every variant once on the site's own launch and keeps the fastest. Results are
// kept per device identity and shape, in memory and, with a store directory, in one JSON-lines file
// there (`av-denoise-b200-tune.jsonl`, one object per key: the key, the variant and each variant's
// milliseconds), which later processes read.
#pragma once

#include <functional>
#include <string>

namespace avd {

enum class TuneMode { Auto = 0, Cached = 1, Off = 2 };

struct TuneOptions {
    TuneMode mode = TuneMode::Auto;
    std::string store;  // directory of the results file; empty: this process only
};

// The device this process runs on, as stored results are keyed: name, compute capability, SM count.
std::string tune_device_identity();

// The variant of `key` among `variants` (0 is the baseline). `time_variant(v)` launches variant v on
// the site's own work and returns its device milliseconds (negative on failure: that variant is
// skipped). Off mode and a site with one variant answer 0 without timing; Cached mode answers the
// remembered or stored variant, else 0.
int tuned_variant(const TuneOptions& options, const std::string& key, int variants,
                  const std::function<float(int)>& time_variant);

// Drops the results this process remembers (the store file stays): for tests of the store.
void tune_forget();

}  // namespace avd
