// CPU ORACLE - test infrastructure only (see nlm_oracle.cpp for the rules it follows).
//
// The FP64 adjoint of one windowed NLMeans frame, written straight from the forward's formulas
// (av-denoise-core/src/nlmeans/kernels/fused.rs:138-530, helpers.rs:34-73, accumulate.rs:152-202;
// the forward is nlm_oracle.cpp's `nlm_pixel`):
//   D_o = scale * sum_delta sum_c (I(clamp(p+delta)) - F_o(clamp(p+q_o+delta)))^2,
//   w_o = exp(-max(D_o - off_o, 0) h2),  out = (I wref M + sum w_o F_o(p+q_o)) / (wref M + sum w_o),
// M = max w_o with its gradient on the first offset that reaches it. The reference has no adjoint;
// tests/test_oracle_nlm_backward.py checks this one against central finite differences of the FP64
// forward.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace {
inline int clampc(int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }
}  // namespace

extern "C" {

void orc_nlm_backward_f64(const float* const* frames, int w, int h, int C, int d, int a, int s, double strength,
                          double wref, double pair_off, double spatial_off, const double* grad_out,
                          double* grad_frames, double* grad_strength) {
    const int F = 2 * d + 1;
    const size_t fe = static_cast<size_t>(w) * h * C;
    std::fill(grad_frames, grad_frames + F * fe, 0.0);
    const double area = (2.0 * s + 1) * (2.0 * s + 1);
    const double h2 = 65025.0 / (3.0 * strength * strength * area);
    const double scale = C == 1 ? 3.0 : 1.5;
    auto px_at = [&](int f, int x, int y, int c) {
        return static_cast<double>(frames[f][(static_cast<size_t>(clampc(y, h)) * w + clampc(x, w)) * C + c]);
    };
    auto g_at = [&](int f, int x, int y, int c) -> double& {
        return grad_frames[f * fe + (static_cast<size_t>(clampc(y, h)) * w + clampc(x, w)) * C + c];
    };
    struct Off {
        int f, qx, qy;
        double off;
    };
    std::vector<Off> offs;
    for (int k = 0; k < d; ++k)
        for (int qy = -a; qy <= a; ++qy)
            for (int qx = -a; qx <= a; ++qx) {
                offs.push_back({k, qx, qy, pair_off});
                offs.push_back({2 * d - k, -qx, -qy, pair_off});
            }
    for (int qy = -a; qy <= a; ++qy)
        for (int qx = -a; qx <= a; ++qx)
            if (qx || qy) offs.push_back({d, qx, qy, spatial_off});
    double gh2 = 0.0;
    std::vector<double> D(offs.size()), W8(offs.size());
    for (int py = 0; py < h; ++py)
        for (int px = 0; px < w; ++px) {
            double A[2] = {0, 0}, W = 0, M = 0;
            int argmax = -1;
            for (size_t i = 0; i < offs.size(); ++i) {
                const Off& o = offs[i];
                double sum = 0;
                for (int oy = -s; oy <= s; ++oy)
                    for (int ox = -s; ox <= s; ++ox)
                        for (int c = 0; c < C; ++c) {
                            const double diff = px_at(d, px + ox, py + oy, c) - px_at(o.f, px + ox + o.qx, py + oy + o.qy, c);
                            sum += diff * diff * scale;
                        }
                D[i] = sum;
                W8[i] = std::exp(-std::max(sum - o.off, 0.0) * h2);
                for (int c = 0; c < C; ++c) A[c] += W8[i] * px_at(o.f, px + o.qx, py + o.qy, c);
                W += W8[i];
                if (W8[i] > M) {
                    M = W8[i];
                    argmax = static_cast<int>(i);
                }
            }
            const double* g = grad_out + (static_cast<size_t>(py) * w + px) * C;
            const double den = wref * M + W;
            if (!(den > 1e-30)) {
                for (int c = 0; c < C; ++c) g_at(d, px, py, c) += g[c];
                continue;
            }
            const double inv = 1.0 / den;
            double out[2] = {0, 0}, gm = 0;
            for (int c = 0; c < C; ++c) {
                const double I = px_at(d, px, py, c);
                out[c] = (I * wref * M + A[c]) * inv;
                g_at(d, px, py, c) += g[c] * wref * M * inv;
                gm += g[c] * wref * (I - out[c]) * inv;
            }
            for (size_t i = 0; i < offs.size(); ++i) {
                const Off& o = offs[i];
                double gw = static_cast<int>(i) == argmax ? gm : 0.0;
                for (int c = 0; c < C; ++c) {
                    gw += g[c] * (px_at(o.f, px + o.qx, py + o.qy, c) - out[c]) * inv;
                    g_at(o.f, px + o.qx, py + o.qy, c) += g[c] * W8[i] * inv;
                }
                const double excess = D[i] - o.off;
                if (excess > 0) {
                    gh2 += gw * (-excess * W8[i]);
                    const double gd = gw * (-h2 * W8[i]) * 2.0 * scale;
                    for (int oy = -s; oy <= s; ++oy)
                        for (int ox = -s; ox <= s; ++ox)
                            for (int c = 0; c < C; ++c) {
                                const double diff = px_at(d, px + ox, py + oy, c) -
                                                    px_at(o.f, px + ox + o.qx, py + oy + o.qy, c);
                                g_at(d, px + ox, py + oy, c) += gd * diff;
                                g_at(o.f, px + ox + o.qx, py + oy + o.qy, c) -= gd * diff;
                            }
                }
            }
        }
    *grad_strength = gh2 * (-2.0 * h2 / strength);
}

}  // extern "C"
