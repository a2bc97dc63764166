// CPU ORACLE - test infrastructure only (see nlm_oracle.cpp for the rules it follows).
//
// A C++17 restatement of av-denoise's Immerkær spatial noise estimate:
//   partials: av-denoise-core/src/noise/kernels/stats.rs:24-94 (|4c - 2(l+r+u+d) + diagonals| over
//             each 32x8 block's interior pixels, summed in thread order, two lanes per block);
//   totals:   kernels/stats.rs:96-137 (256 strided sums, then summed in order);
//   quartile: noise/spatial.rs:146-200 (`sigma_block_p25_from_partials`: each block's sigma over its
//             interior area, blocks without interior skipped) with noise/stats.rs:24-37
//             (`lower_quartile`, interpolating at 0.25 (n - 1)), which the GPU reading computes from
//             the ranks (n - 1) / 4 and (n + 2) / 4 (kernels/sample.rs:108-114).
// The reference's own tests pin the quartile (noise/tests/spatial.rs:52-105): tests/test_oracle_noise.py
// replays them on this restatement.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace {
constexpr int BX = 32, BY = 8, LANES = 2;
}

extern "C" {

int64_t orc_immerkaer_partials_len(int w, int h) {
    return static_cast<int64_t>((w + BX - 1) / BX) * ((h + BY - 1) / BY) * LANES;
}

void orc_immerkaer_partials(const float* frame, int channels, int w, int h, float* partials) {
    const int cx_n = (w + BX - 1) / BX, cy_n = (h + BY - 1) / BY;
    for (int cy = 0; cy < cy_n; ++cy)
        for (int cx = 0; cx < cx_n; ++cx)
            for (int c = 0; c < LANES; ++c) {
                float sum = 0.0f;
                for (int ty = 0; ty < BY; ++ty)
                    for (int tx = 0; tx < BX; ++tx) {
                        const int x = cx * BX + tx, y = cy * BY + ty;
                        float r = 0.0f;
                        if (c < channels && x >= 1 && x < w - 1 && y >= 1 && y < h - 1) {
                            auto at = [&](int dx, int dy) {
                                return frame[(static_cast<int64_t>(y + dy) * w + x + dx) * channels + c];
                            };
                            const float cross = at(-1, 0) + at(1, 0) + at(0, -1) + at(0, 1);
                            const float diag = at(-1, -1) + at(1, -1) + at(-1, 1) + at(1, 1);
                            r = at(0, 0) * 4.0f - cross * 2.0f + diag;
                        }
                        sum += std::fabs(r);
                    }
                partials[(cy * cx_n + cx) * LANES + c] = sum;
            }
}

void orc_immerkaer_totals(const float* partials, int blocks, float* results) {
    for (int c = 0; c < LANES; ++c) {
        float thread_sums[256];
        for (int t = 0; t < 256; ++t) {
            float s = 0.0f;
            for (int i = t; i < blocks; i += 256) s += partials[i * LANES + c];
            thread_sums[t] = s;
        }
        float total = 0.0f;
        for (int t = 0; t < 256; ++t) total += thread_sums[t];
        results[c] = total;
    }
}

float orc_lower_quartile(const float* sorted, int n) {
    if (n == 1) return sorted[0];
    const int lo = (n - 1) / 4, hi = (n + 2) / 4;
    const float fraction = static_cast<float>((n - 1) % 4) * 0.25f;
    return sorted[lo] + fraction * (sorted[hi] - sorted[lo]);
}

void orc_immerkaer_sigma_low(const float* partials, int channels, int w, int h, float scale, float* sigma_low) {
    const int cx_n = (w + BX - 1) / BX, cy_n = (h + BY - 1) / BY;
    for (int c = 0; c < LANES; ++c) {
        sigma_low[c] = 0.0f;
        if (c >= channels) continue;
        std::vector<float> sig;
        for (int cy = 0; cy < cy_n; ++cy)
            for (int cx = 0; cx < cx_n; ++cx) {
                const int x0 = std::max(cx * BX, 1), y0 = std::max(cy * BY, 1);
                const int x1 = std::min(std::min((cx + 1) * BX, w), w - 1);
                const int y1 = std::min(std::min((cy + 1) * BY, h), h - 1);
                if (x1 <= x0 || y1 <= y0) continue;
                const float area = static_cast<float>((x1 - x0) * (y1 - y0));
                sig.push_back(scale * partials[(cy * cx_n + cx) * LANES + c] / (6.0f * area));
            }
        if (sig.empty()) continue;
        std::sort(sig.begin(), sig.end());
        sigma_low[c] = orc_lower_quartile(sig.data(), static_cast<int>(sig.size()));
    }
}

}  // extern "C"
