// CPU ORACLE - test infrastructure only (see nlm_oracle.cpp for the rules it follows).
//
// The NL4D collaborative filter as a smooth function of its frames and noise levels, in f64, and
// its adjoint. The reference has neither an adjoint nor a Wiener stage (its filter,
// av-denoise-core/src/collab/kernels/fused/mod.rs:559-850, stops at the hard or pooled
// threshold), so this file is their oracle; the tests check it by central finite differences of
// its own forward, and check its forward against the f32 restatement (collab_oracle.cpp).
//
// With the groups (member positions) and every keep decision of one pass held fixed - the records
// the f32 restatement writes (member_record, mask_record) - one reference patch's group does:
//   Z = T X                 a 2D DCT per member, then the member-axis transform (the Haar ladder
//                           over the k_use members, or the time/volume grid); T is orthonormal
//   Y = M g Z               keep mask M; gain g = Z^2 / (Z^2 + v) with the Wiener stage, else 1
//   R = sum M g^2 v         over channel 0's coefficients, v = sigma_c^2 prof[lane] prof[slot]
//   w = ws / max(R, 1e-12)  the group weight; the weight-scale word ws is read as proportional to
//                           sigma_0^2, as the engine derives it (aggregate.rs:79-99: sigma_0^2 g_max^2)
//   est = T^T Y
//   A[p, c] += clamp(w K est, -5, 5),  W[p] += clamp(w K, 0, 1)   at every member's pixels
// with K the Kaiser taper. A and W are in real units: the kernels hold A x accum_scale and
// W x accum_scale x 5 in fixed point, and the normalised frame is A / W.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

namespace {

constexpr int P = 8;
constexpr int MAX_K = 8;
constexpr int STEP = 4;
constexpr double RECIPROCAL_FLOOR = 1e-12;  // the f32 filter's floor, 1e-12f widened

struct Collab64Args {
    const double* ring;               // slots x H x W x C
    const uint32_t* members;          // 9 words per reference patch
    const uint64_t* masks;            // refs x C x 8 lanes, bit j * 8 + i
    const uint32_t* neighbour_slots;  // ring slot of neighbour index t - 1
    const double* sigma;              // per channel
    const float* dct_profile;         // 8
    const float* kaiser;              // 8
    double weight_scale;        // the word at sigma_0 = weight_scale_sigma
    double weight_scale_sigma;
    int width, height, channels, centre_slot, grid_frames, wiener;
    double* accum;  // slots x H x W x C, added into (null: not computed)
    double* wsum;   // slots x H x W, added into
    const double* grad_accum;  // the adjoint's inputs, dL/dA and dL/dW (null: no adjoint)
    const double* grad_wsum;
    double* grad_ring;   // slots x H x W x C, added into
    double* grad_sigma;  // per channel, added into
};

// The orthonormal DCT-II rows, c_u cos(pi (2x + 1) u / 16).
struct Dct {
    double d[P][P];
    Dct() {
        for (int u = 0; u < P; ++u)
            for (int x = 0; x < P; ++x)
                d[u][x] = (u == 0 ? 1.0 / std::sqrt(8.0) : 0.5) * std::cos(M_PI * (2.0 * x + 1.0) * u / 16.0);
    }
};
const Dct kDct;

// One Haar level of `len` values read `stride` apart from `start`: pair sums then differences.
void level(double* v, int start, int stride, int len) {
    const double r = std::sqrt(0.5);
    double snap[MAX_K];
    for (int k = 0; k < len; ++k) snap[k] = v[start + k * stride];
    for (int p = 0; p < len / 2; ++p) {
        v[start + p * stride] = (snap[2 * p] + snap[2 * p + 1]) * r;
        v[start + (len / 2 + p) * stride] = (snap[2 * p] - snap[2 * p + 1]) * r;
    }
}

void strided_fwd(double* v, int start, int stride, int len) {
    if (len >= 4) level(v, start, stride, 4);
    if (len >= 2) level(v, start, stride, 2);
}

// The member-axis transform as a matrix: column m is the transform of unit vector m
// (transforms.rs:124-170 for the ladder, grid.rs for the volumes).
void axis_matrix(int k_use, bool grid, int gf, double (&h)[MAX_K][MAX_K]) {
    for (int m = 0; m < MAX_K; ++m) {
        double v[MAX_K] = {};
        v[m] = 1.0;
        if (grid) {
            const int volumes = MAX_K / gf;
            for (int vol = 0; vol < volumes; ++vol) strided_fwd(v, vol * gf, 1, gf);
            for (int f = 0; f < gf; ++f) strided_fwd(v, f, gf, volumes);
        } else {
            if (k_use >= 8) level(v, 0, 1, 8);
            if (k_use >= 4) level(v, 0, 1, 4);
            if (k_use >= 2) level(v, 0, 1, 2);
        }
        for (int j = 0; j < MAX_K; ++j) h[j][m] = v[j];
    }
}

// Stacks are [member or coefficient][lane][slot]. In the pixel domain lane is the column and slot
// the row; in the coefficient domain lane is the row frequency and slot the column frequency.
using Stack = double[MAX_K][P][P];

void forward(const double (&h)[MAX_K][MAX_K], int k, const Stack& x, Stack& z) {
    Stack t;
    for (int m = 0; m < k; ++m)
        for (int u = 0; u < P; ++u)
            for (int v = 0; v < P; ++v) {
                double acc = 0.0;
                for (int col = 0; col < P; ++col)
                    for (int r = 0; r < P; ++r) acc += kDct.d[u][r] * kDct.d[v][col] * x[m][col][r];
                t[m][u][v] = acc;
            }
    for (int j = 0; j < k; ++j)
        for (int u = 0; u < P; ++u)
            for (int v = 0; v < P; ++v) {
                double acc = 0.0;
                for (int m = 0; m < k; ++m) acc += h[j][m] * t[m][u][v];
                z[j][u][v] = acc;
            }
}

void inverse(const double (&h)[MAX_K][MAX_K], int k, const Stack& z, Stack& x) {
    Stack t;
    for (int m = 0; m < k; ++m)
        for (int u = 0; u < P; ++u)
            for (int v = 0; v < P; ++v) {
                double acc = 0.0;
                for (int j = 0; j < k; ++j) acc += h[j][m] * z[j][u][v];
                t[m][u][v] = acc;
            }
    for (int m = 0; m < k; ++m)
        for (int col = 0; col < P; ++col)
            for (int r = 0; r < P; ++r) {
                double acc = 0.0;
                for (int u = 0; u < P; ++u)
                    for (int v = 0; v < P; ++v) acc += kDct.d[u][r] * kDct.d[v][col] * t[m][u][v];
                x[m][col][r] = acc;
            }
}

struct Group {
    int k = 1;
    bool grid = false;
    size_t base[MAX_K];  // pixel index of each member's top-left sample
};

Group group_of(const Collab64Args& a, size_t ref) {
    Group g;
    const uint32_t* words = a.members + ref * (MAX_K + 1);
    g.k = static_cast<int>(words[MAX_K] & 0xFFu);
    g.grid = (words[MAX_K] & 0x100u) != 0;
    const size_t plane = static_cast<size_t>(a.width) * a.height;
    for (int m = 0; m < MAX_K; ++m) {
        const uint32_t p = words[m];
        const uint32_t t = p >> 26;
        const size_t slot = t > 0 ? a.neighbour_slots[t - 1] : static_cast<size_t>(a.centre_slot);
        g.base[m] = slot * plane + static_cast<size_t>((p >> 13) & 0x1FFFu) * a.width + (p & 0x1FFFu);
    }
    return g;
}

// The gain and its partial derivatives at coefficient z of noise variance v.
struct Gain {
    double g = 1.0, dy_dz = 1.0, dy_dv = 0.0, dr_dz = 0.0, dr_dv = 1.0;  // R's term is g^2 v
};

Gain gain_at(double z, double v, bool wiener) {
    Gain q;
    if (!wiener) return q;
    const double den = z * z + v;
    if (!(den > 0.0)) {
        q.dr_dv = 1.0;
        return q;
    }
    q.g = z * z / den;
    q.dy_dz = q.g * (z * z + 3.0 * v) / den;
    q.dy_dv = -q.g * z / den;
    q.dr_dz = 4.0 * q.g * z * v * v / (den * den);
    q.dr_dv = q.g * q.g * (z * z - v) / den;
    return q;
}

void process(const Collab64Args& a, size_t ref) {
    const int C = a.channels;
    const Group grp = group_of(a, ref);
    double h[MAX_K][MAX_K];
    axis_matrix(grp.k, grp.grid, a.grid_frames, h);
    const bool wiener = a.wiener != 0;
    const bool adjoint = a.grad_ring != nullptr;
    const double sigma_ratio = a.sigma[0] / a.weight_scale_sigma;
    const double ws = a.weight_scale * sigma_ratio * sigma_ratio;
    static thread_local Stack x[2], z[2], y[2], est[2];
    double retained = 0.0, weight = 0.0;
    for (int c = 0; c < C; ++c) {
        for (int m = 0; m < grp.k; ++m)
            for (int col = 0; col < P; ++col)
                for (int r = 0; r < P; ++r) x[c][m][col][r] = a.ring[(grp.base[m] + r * a.width + col) * C + c];
        forward(h, grp.k, x[c], z[c]);
        const double s2 = a.sigma[c] * a.sigma[c];
        double rv = 0.0;
        for (int u = 0; u < P; ++u) {
            const uint64_t bits = a.masks[(ref * C + c) * P + u];
            for (int j = 0; j < grp.k; ++j)
                for (int v = 0; v < P; ++v) {
                    const bool keep = (bits >> (j * 8 + v)) & 1u;
                    const double var = s2 * a.dct_profile[u] * a.dct_profile[v];
                    const Gain q = gain_at(z[c][j][u][v], var, wiener);
                    y[c][j][u][v] = keep ? q.g * z[c][j][u][v] : 0.0;
                    if (keep) rv += q.g * q.g * var;
                }
        }
        if (c == 0) {
            retained = rv;
            weight = ws / std::max(rv, RECIPROCAL_FLOOR);
        }
        inverse(h, grp.k, y[c], est[c]);
    }
    const size_t plane = static_cast<size_t>(a.width) * a.height;
    (void)plane;
    if (a.accum) {
        for (int c = 0; c < C; ++c)
            for (int m = 0; m < grp.k; ++m)
                for (int col = 0; col < P; ++col)
                    for (int r = 0; r < P; ++r) {
                        const double wk = weight * a.kaiser[r] * a.kaiser[col];
                        const size_t pixel = grp.base[m] + r * a.width + col;
                        a.accum[pixel * C + c] += std::min(std::max(est[c][m][col][r] * wk, -5.0), 5.0);
                        if (c == 0) a.wsum[pixel] += std::min(std::max(wk, 0.0), 1.0);
                    }
    }
    if (!adjoint) return;
    // Back through the scatter: d est and d w.
    static thread_local Stack dest[2], dy[2];
    double dweight = 0.0;
    for (int c = 0; c < C; ++c) {
        std::memset(dest[c], 0, sizeof(Stack));
        for (int m = 0; m < grp.k; ++m)
            for (int col = 0; col < P; ++col)
                for (int r = 0; r < P; ++r) {
                    const double kk = a.kaiser[r] * a.kaiser[col];
                    const double wk = weight * kk;
                    const size_t pixel = grp.base[m] + r * a.width + col;
                    const double e = est[c][m][col][r];
                    double dwk = 0.0;
                    if (std::fabs(e * wk) < 5.0) {
                        const double g = a.grad_accum[pixel * C + c];
                        dest[c][m][col][r] = g * wk;
                        dwk += g * e;
                    }
                    if (c == 0 && wk > 0.0 && wk < 1.0) dwk += a.grad_wsum[pixel];
                    dweight += dwk * kk;
                }
        forward(h, grp.k, dest[c], dy[c]);
    }
    const double dretained = retained > RECIPROCAL_FLOOR ? -dweight * ws / (retained * retained) : 0.0;
    a.grad_sigma[0] += dweight * 2.0 * weight / a.sigma[0];  // through ws
    static thread_local Stack dz;
    for (int c = 0; c < C; ++c) {
        const double s2 = a.sigma[c] * a.sigma[c];
        double dvar_sigma = 0.0;
        std::memset(dz, 0, sizeof(Stack));
        for (int u = 0; u < P; ++u) {
            const uint64_t bits = a.masks[(ref * C + c) * P + u];
            for (int j = 0; j < grp.k; ++j)
                for (int v = 0; v < P; ++v) {
                    if (!((bits >> (j * 8 + v)) & 1u)) continue;
                    const double pp = static_cast<double>(a.dct_profile[u]) * a.dct_profile[v];
                    const Gain q = gain_at(z[c][j][u][v], s2 * pp, wiener);
                    double dzz = dy[c][j][u][v] * q.dy_dz;
                    double dv = dy[c][j][u][v] * q.dy_dv;
                    if (c == 0) {
                        dzz += dretained * q.dr_dz;
                        dv += dretained * q.dr_dv;
                    }
                    dz[j][u][v] = dzz;
                    dvar_sigma += dv * 2.0 * a.sigma[c] * pp;
                }
        }
        a.grad_sigma[c] += dvar_sigma;
        Stack dx;
        inverse(h, grp.k, dz, dx);
        for (int m = 0; m < grp.k; ++m)
            for (int col = 0; col < P; ++col)
                for (int r = 0; r < P; ++r) a.grad_ring[(grp.base[m] + r * a.width + col) * C + c] += dx[m][col][r];
    }
}

uint32_t refs_along(uint32_t dim) { return (dim - P + STEP - 1) / STEP + 1; }

}  // namespace

extern "C" {

// Every reference patch in raster order (sequential: the sums land in a fixed order). Computes the
// accumulators when `accum` is set and the adjoint when `grad_ring` is set.
void orc64_collab_pass(const Collab64Args* args) {
    const Collab64Args& a = *args;
    const size_t refs = static_cast<size_t>(refs_along(a.width)) * refs_along(a.height);
    for (size_t ref = 0; ref < refs; ++ref) process(a, ref);
}

}  // extern "C"
