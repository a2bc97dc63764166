// CPU ORACLE - test infrastructure only (see nlm_oracle.cpp for the rules it follows).
//
// A C++17 restatement of av-denoise's NL4D collaborative filter, `collab_fused`
// (av-denoise-core/src/collab/kernels/fused/mod.rs:170-891), with the helpers it calls:
// centre search (fused/centre.rs:32-353), trajectory search (fused/trajectory.rs, clipped walk),
// volume grid (fused/grid.rs), pooled threshold (fused/pooled.rs), transforms (transforms.rs),
// reductions and top-8 insert (plane_ops.rs), aggregation (aggregate.rs). One 8-lane group of the
// reference is modelled explicitly: lane `sub` owns column `sub` of every patch, and every
// cross-lane sum follows the reference's xor-1/2/4 butterfly order.
//
// Parity pin: the reference records seven digests of this filter's aggregated output
// (collab/tests/fused/recorded.rs); tests/test_oracle_collab.py rebuilds their inputs and checks
// this oracle against every one.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "colour_table.h"
#include "mirror_math.h"

namespace {

constexpr int P = 8;      // PATCH_SIZE
constexpr int STEP = 4;   // reference grid step
constexpr int MAX_K = 8;  // group size ceiling
constexpr float UNFILLED = 3.0e38f;
constexpr float SELF_PIN = -1.0e38f;
constexpr float RECIPROCAL_FLOOR = 1e-12f;
constexpr float ACCUM_CLAMP = 5.0f;
constexpr float WEIGHT_CLAMP = 1.0f;
constexpr float WEIGHT_GAIN = ACCUM_CLAMP / WEIGHT_CLAMP;
constexpr float VARIANCE_FLOOR = 1.0e-20f;
constexpr float CURVE_SCALE_MIN = 0.33f;
constexpr float CURVE_SCALE_MAX = 3.0f;
constexpr float COLOUR_CURVE_SCALE_MAX = 6.0f;  // fused/mod.rs:57-58: curve and colour gain together
constexpr int CURVE_BINS = 16;
constexpr float FRAC_1_SQRT_2 = 0.70710678118654752440f;

// transforms.rs:41-45 (`dct8_basis`) evaluated in f64 and rounded to f32, as the kernel's
// compile-time taps are.
struct DctTaps {
    float t[8][8];
    DctTaps() {
        for (int row = 0; row < 8; ++row)
            for (int col = 0; col < 8; ++col) {
                double scale = row == 0 ? 1.0 / std::sqrt(8.0) : 0.5;
                double angle = M_PI * (2.0 * col + 1.0) * row / 16.0;
                t[row][col] = static_cast<float>(scale * std::cos(angle));
            }
    }
};
const DctTaps kTaps;

// transforms.rs:53-84 (`dct8_reg_fwd`): pair sums and differences, then the even and odd rows.
void dct8_fwd(float* line) {
    float s[4], d[4];
    for (int k = 0; k < 4; ++k) {
        s[k] = line[k] + line[7 - k];
        d[k] = line[k] - line[7 - k];
    }
    for (int m = 0; m < 4; ++m) {
        float even = 0.0f, odd = 0.0f;
        for (int k = 0; k < 4; ++k) {
            even = even + s[k] * kTaps.t[2 * m][k];
            odd = odd + d[k] * kTaps.t[2 * m + 1][k];
        }
        line[2 * m] = even;
        line[2 * m + 1] = odd;
    }
}

// transforms.rs:90-113 (`dct8_reg_inv`).
void dct8_inv(float* line) {
    float snap[8];
    std::memcpy(snap, line, sizeof(snap));
    for (int k = 0; k < 4; ++k) {
        float even = 0.0f, odd = 0.0f;
        for (int m = 0; m < 4; ++m) {
            even = even + snap[2 * m] * kTaps.t[2 * m][k];
            odd = odd + snap[2 * m + 1] * kTaps.t[2 * m + 1][k];
        }
        line[k] = even + odd;
        line[7 - k] = even - odd;
    }
}

// A group's working set: stack[m][lane][i] is lane `lane`'s slot i of member m.
struct Stack {
    float v[MAX_K][P][P];
};

// transforms.rs:124-170 (`haar_reg_fwd_level`, `haar_reg_inv_level`), on every lane and position.
void haar_fwd_level(Stack& s, int len) {
    int half = len / 2;
    for (int lane = 0; lane < P; ++lane)
        for (int pos = 0; pos < P; ++pos) {
            float snap[MAX_K];
            for (int k = 0; k < len; ++k) snap[k] = s.v[k][lane][pos];
            for (int p = 0; p < half; ++p) {
                float a = snap[2 * p], b = snap[2 * p + 1];
                s.v[p][lane][pos] = (a + b) * FRAC_1_SQRT_2;
                s.v[half + p][lane][pos] = (a - b) * FRAC_1_SQRT_2;
            }
        }
}

void haar_inv_level(Stack& s, int len) {
    int half = len / 2;
    for (int lane = 0; lane < P; ++lane)
        for (int pos = 0; pos < P; ++pos) {
            float snap[MAX_K];
            for (int k = 0; k < len; ++k) snap[k] = s.v[k][lane][pos];
            for (int p = 0; p < half; ++p) {
                float lo = snap[p], hi = snap[half + p];
                s.v[2 * p][lane][pos] = (lo + hi) * FRAC_1_SQRT_2;
                s.v[2 * p + 1][lane][pos] = (lo - hi) * FRAC_1_SQRT_2;
            }
        }
}

// transforms.rs:176-191 (`variance_reg_level`).
void variance_level(float* v, int len) {
    int half = len / 2;
    float snap[MAX_K];
    for (int k = 0; k < len; ++k) snap[k] = v[k];
    for (int p = 0; p < half; ++p) {
        float mean = (snap[2 * p] + snap[2 * p + 1]) * 0.5f;
        v[p] = mean;
        v[half + p] = mean;
    }
}

// grid.rs: strided Haar levels over one position's 8 members.
void strided_level(float* vals, int start, int stride, int len, bool inverse, bool variance) {
    int half = len / 2;
    float snap[MAX_K];
    for (int k = 0; k < len; ++k) snap[k] = vals[start + k * stride];
    for (int p = 0; p < half; ++p) {
        if (variance) {
            float mean = (snap[2 * p] + snap[2 * p + 1]) * 0.5f;
            vals[start + p * stride] = mean;
            vals[start + (half + p) * stride] = mean;
        } else if (!inverse) {
            float a = snap[2 * p], b = snap[2 * p + 1];
            vals[start + p * stride] = (a + b) * FRAC_1_SQRT_2;
            vals[start + (half + p) * stride] = (a - b) * FRAC_1_SQRT_2;
        } else {
            float lo = snap[p], hi = snap[half + p];
            vals[start + 2 * p * stride] = (lo + hi) * FRAC_1_SQRT_2;
            vals[start + (2 * p + 1) * stride] = (lo - hi) * FRAC_1_SQRT_2;
        }
    }
}

void strided_fwd(float* vals, int start, int stride, int len, bool variance) {
    if (len >= 4) strided_level(vals, start, stride, 4, false, variance);
    if (len >= 2) strided_level(vals, start, stride, 2, false, variance);
}

void strided_inv(float* vals, int start, int stride, int len) {
    if (len >= 2) strided_level(vals, start, stride, 2, true, false);
    if (len >= 4) strided_level(vals, start, stride, 4, true, false);
}

// grid.rs (`grid_fwd`, `grid_inv`, `grid_variance`): Haar along time inside each volume, then
// across volumes.
void grid_fwd(Stack& s, int gf) {
    int volumes = MAX_K / gf;
    for (int lane = 0; lane < P; ++lane)
        for (int pos = 0; pos < P; ++pos) {
            float vals[MAX_K];
            for (int m = 0; m < MAX_K; ++m) vals[m] = s.v[m][lane][pos];
            for (int vol = 0; vol < volumes; ++vol) strided_fwd(vals, vol * gf, 1, gf, false);
            for (int f = 0; f < gf; ++f) strided_fwd(vals, f, gf, volumes, false);
            for (int m = 0; m < MAX_K; ++m) s.v[m][lane][pos] = vals[m];
        }
}

void grid_inv(Stack& s, int gf) {
    int volumes = MAX_K / gf;
    for (int lane = 0; lane < P; ++lane)
        for (int pos = 0; pos < P; ++pos) {
            float vals[MAX_K];
            for (int m = 0; m < MAX_K; ++m) vals[m] = s.v[m][lane][pos];
            for (int f = 0; f < gf; ++f) strided_inv(vals, f, gf, volumes);
            for (int vol = 0; vol < volumes; ++vol) strided_inv(vals, vol * gf, 1, gf);
            for (int m = 0; m < MAX_K; ++m) s.v[m][lane][pos] = vals[m];
        }
}

void grid_variance(float* v, int gf) {
    int volumes = MAX_K / gf;
    for (int vol = 0; vol < volumes; ++vol) strided_fwd(v, vol * gf, 1, gf, true);
    for (int f = 0; f < gf; ++f) strided_fwd(v, f, gf, volumes, true);
}

// plane_ops.rs:17-23 (`plane_ssd_reduce8`): the xor-1/2/4 butterfly; every lane ends with the
// same bits, those of ((p0+p1)+(p2+p3)) + ((p4+p5)+(p6+p7)).
float reduce8(const float* p) {
    float a0 = p[0] + p[1], a2 = p[2] + p[3], a4 = p[4] + p[5], a6 = p[6] + p[7];
    float b0 = a0 + a2, b4 = a4 + a6;
    return b0 + b4;
}

// transforms.rs:27-33 (`safe_reciprocal`).
float safe_reciprocal(float denom, float floor) {
    if (std::isnan(denom) || std::isinf(denom)) return 0.0f;
    return 1.0f / std::max(denom, floor);
}

// aggregate.rs:147-160 (`to_fixed`, `to_fixed_weight`): clamp, scale, round half away from zero.
int32_t to_fixed(float value, float scale) {
    float c = std::min(std::max(value, -ACCUM_CLAMP), ACCUM_CLAMP);
    return static_cast<int32_t>(std::round(c * scale));
}

int32_t to_fixed_weight(float weight, float scale) {
    float c = std::min(std::max(weight, 0.0f), WEIGHT_CLAMP);
    float t = c * scale;
    t = t * WEIGHT_GAIN;
    return static_cast<int32_t>(std::round(t));
}

inline uint32_t pack_pos_t(uint32_t x, uint32_t y, uint32_t t) { return (t << 26) | (y << 13) | x; }
inline uint32_t unpack_x(uint32_t p) { return p & 0x1FFFu; }
inline uint32_t unpack_y(uint32_t p) { return (p >> 13) & 0x1FFFu; }
inline uint32_t unpack_t(uint32_t p) { return p >> 26; }

// group.rs (`clamp_top_left`).
inline uint32_t clamp_top_left(int v, uint32_t max_pos) {
    if (v < 0) return 0;
    if (v > static_cast<int>(max_pos)) return max_pos;
    return static_cast<uint32_t>(v);
}

}  // namespace

namespace {

struct CollabArgs {
    const float* ring;             // slots x H x W x C, f32
    const int32_t* mv_field;       // per neighbour: blocks x (dx, dy)
    const float* confidence;       // per neighbour: blocks
    const uint32_t* neighbour_slots;
    const float* sigma;            // per channel
    const float* noise_curve;      // CURVE_BINS ratios
    const float* dct_profile;      // 8
    const float* kaiser;           // 8
    int32_t* accum;                // slots x H x W x C
    int32_t* wsum;                 // slots x H x W
    float* group_weight;           // refs
    int width, height, channels, centre_slot;
    int radius, grid_frames, refine, spatial_radius, k_max;
    int mv_stride, conf_stride, blk_step, blksize, blocks_x, blocks_y;
    float c_min, lambda_ht, accum_scale, pool_ratio, weight_scale;
    int pooled, curve_valid;
    // The colour grain gains (collab/kernels/fused/colour.rs): one log gain table per channel, the
    // centre frame's block means on this plane's 16x16 grid, the factor from a sample to the 8-bit
    // scale; read only with colour_on.
    const float* colour_gains;
    const float* colour_means;
    float colour_scale;
    int colour_on, colour_blocks_x;
    // The empirical Wiener stage, an extension the reference does not have (its filter stops at the
    // threshold): each kept coefficient z of noise variance v is scaled by g = z^2 / (z^2 + v), the
    // group's thresholded spectrum serving as its own pilot, and the retained variance counts
    // g^2 v. Zero keeps the reference's filter.
    int wiener;
    // Records of the pass, written when not null: the 9 member words per reference patch (8 packed
    // positions, then k_use | use_grid << 8), and per reference patch, channel and lane the 64 keep
    // decisions (bit j * 8 + i for member-axis coefficient j, slot i).
    uint32_t* member_record;
    uint64_t* mask_record;
};

struct Group {
    const CollabArgs& a;
    int sub_count = P;
    float cur[P][P][2];  // [lane][row][channel] reference columns

    explicit Group(const CollabArgs& args) : a(args) {}

    float px(int slot, int x, int y, int c) const {
        return a.ring[((static_cast<size_t>(slot) * a.height + y) * a.width + x) * a.channels + c];
    }

    // distance.rs:153-177 then :184-208: per-lane column sums, the butterfly, then the scale.
    float distance(const float (&ref)[P][P][2], uint32_t x, uint32_t y, int slot, float scale) const {
        float partial[P];
        for (int sub = 0; sub < P; ++sub) {
            float s = 0.0f;
            for (int r = 0; r < P; ++r)
                for (int c = 0; c < a.channels; ++c) {
                    float d = ref[sub][r][c] - px(slot, x + sub, y + r, c);
                    s = s + d * d;
                }
            partial[sub] = s;
        }
        return reduce8(partial) * scale;
    }
};

// plane_ops.rs:38-53 (`shift_insert8`): a sorted top-8 where a tie never displaces an incumbent.
void shift_insert8(float* best_d, uint32_t* best_pos, float d, uint32_t packed) {
    float nd[MAX_K];
    uint32_t np[MAX_K];
    for (int lane = 0; lane < MAX_K; ++lane) {
        nd[lane] = best_d[lane];
        np[lane] = best_pos[lane];
        if (d < best_d[lane]) {
            bool lands = lane == 0 || d >= best_d[lane - 1];
            if (lands) {
                nd[lane] = d;
                np[lane] = packed;
            } else {
                nd[lane] = best_d[lane - 1];
                np[lane] = best_pos[lane - 1];
            }
        }
    }
    std::memcpy(best_d, nd, sizeof(nd));
    std::memcpy(best_pos, np, sizeof(np));
}

// trajectory.rs (`covering_lo`).
uint32_t covering_lo(uint32_t patch_start, uint32_t blksize, uint32_t step) {
    uint32_t overhang = std::max(patch_start + P, blksize) - blksize;
    return (overhang + step - 1) / step;
}

struct Rect {
    uint32_t left = 1, right = 0, top = 1, bottom = 0;  // empty
};

// fused/trajectory.rs (`trajectory_search`, the clipped walk): for each neighbour frame, the best
// candidate over one refine rectangle per covering motion block, skipping blocks under c_min,
// rectangles already searched and positions the group already holds; then an insertion into the
// volume's sorted tail.
void trajectory_search(const Group& g, const float (&anchor)[P][P][2], uint32_t ax, uint32_t ay, float scale,
                       float* member_d, uint32_t* member_pos, int first, int tail) {
    const CollabArgs& a = g.a;
    const uint32_t max_x = a.width - P, max_y = a.height - P;
    const int n_neighbours = 2 * a.radius;
    const uint32_t covers = (a.blksize + a.blk_step - 1) / a.blk_step;
    const uint32_t bx_hi = std::min<uint32_t>(ax / a.blk_step, a.blocks_x - 1);
    const uint32_t by_hi = std::min<uint32_t>(ay / a.blk_step, a.blocks_y - 1);
    const uint32_t bx_lo = std::min(covering_lo(ax, a.blksize, a.blk_step), bx_hi);
    const uint32_t by_lo = std::min(covering_lo(ay, a.blksize, a.blk_step), by_hi);

    for (int t = 0; t < n_neighbours; ++t) {
        const int slot = static_cast<int>(a.neighbour_slots[t]);
        const uint32_t packed_t = t + 1;
        float frame_d = UNFILLED;
        uint32_t frame_pos = 0;
        std::vector<Rect> seen(covers * covers);
        for (uint32_t iy = 0; iy < covers; ++iy)
            for (uint32_t ix = 0; ix < covers; ++ix) {
                const uint32_t bx = bx_lo + ix, by = by_lo + iy;
                if (bx > bx_hi || by > by_hi) continue;
                const uint32_t block = by * a.blocks_x + bx;
                if (!(a.confidence[t * a.conf_stride + block] >= a.c_min)) continue;
                const int* mv = a.mv_field + t * a.mv_stride + block * 2;
                const int px_ = static_cast<int>(ax) + mv[0];
                const int py_ = static_cast<int>(ay) + mv[1];
                Rect r;
                r.left = clamp_top_left(px_ - a.refine, max_x);
                r.right = clamp_top_left(px_ + a.refine, max_x);
                r.top = clamp_top_left(py_ - a.refine, max_y);
                r.bottom = clamp_top_left(py_ + a.refine, max_y);
                bool contained = false;
                for (const Rect& s : seen)
                    if (r.left >= s.left && r.right <= s.right && r.top >= s.top && r.bottom <= s.bottom)
                        contained = true;
                if (!contained) {
                    for (uint32_t cy = r.top; cy <= r.bottom; ++cy)
                        for (uint32_t cx = r.left; cx <= r.right; ++cx) {
                            bool in_span = false;
                            for (const Rect& s : seen)
                                if (cy >= s.top && cy <= s.bottom && cx >= s.left && cx <= s.right) in_span = true;
                            const uint32_t packed = pack_pos_t(cx, cy, packed_t);
                            bool held = false;
                            for (int k = 0; k < first; ++k)
                                if (member_pos[k] == packed) held = true;
                            if (in_span || held) continue;
                            float d = g.distance(anchor, cx, cy, slot, scale);
                            if (d < frame_d) {
                                frame_d = d;
                                frame_pos = packed;
                            }
                        }
                }
                seen[iy * covers + ix] = r;
            }
        float carry_d = frame_d;
        uint32_t carry_pos = frame_pos;
        for (int j = 0; j < tail; ++j) {
            const int s = first + j;
            const bool smaller = carry_d < member_d[s];
            const float held_d = member_d[s];
            const uint32_t held_pos = member_pos[s];
            if (smaller) {
                member_d[s] = carry_d;
                member_pos[s] = carry_pos;
                carry_d = held_d;
                carry_pos = held_pos;
            }
        }
    }
}

}  // namespace

namespace {

// fused/pooled.rs: keep a coefficient on the mean energy of itself and its four frequency
// neighbours (shuffled across lanes for the vertical ones). Returns each lane's retained variance.
void pooled_threshold(Stack& s, const float* v, const float* prof, int k_use, float threshold, float dc_lambda,
                      bool wiener, float* retained, uint64_t* bits) {
    float bar = threshold * threshold;
    for (int sub = 0; sub < P; ++sub) retained[sub] = 0.0f;
    for (int j = 0; j < MAX_K; ++j) {
        // Energies from the unmodified coefficients; the DC lane's first energy reads as zero.
        float e[P][P];
        float lane_var[P];
        for (int sub = 0; sub < P; ++sub) {
            lane_var[sub] = v[j] * prof[sub];
            float lane_inv = 1.0f / std::max(lane_var[sub], VARIANCE_FLOOR);
            for (int i = 0; i < P; ++i) {
                float pinv = 1.0f / std::max(prof[i], VARIANCE_FLOOR);
                float c = s.v[j][sub][i];
                e[sub][i] = ((c * c) * lane_inv) * pinv;
            }
            if (sub == 0) e[sub][0] = 0.0f;
        }
        float out[P][P];
        for (int sub = 0; sub < P; ++sub) {
            const bool dc_lane = sub == 0, has_up = sub > 0, has_down = sub < 7;
            const float vertical = 1.0f + (has_up ? 1.0f : 0.0f) + (has_down ? 1.0f : 0.0f);
            const float first_col = bar * (vertical + (sub == 1 ? 0.0f : 1.0f));
            const float second_col = bar * (vertical + (dc_lane ? 1.0f : 2.0f));
            const float middle_col = bar * (vertical + 2.0f);
            const float last_col = bar * (vertical + 1.0f);
            float kept_profile = 0.0f;
            for (int i = 0; i < P; ++i) {
                const float coeff = s.v[j][sub][i];
                float up = has_up ? e[sub - 1][i] : 0.0f;
                float down = has_down ? e[sub + 1][i] : 0.0f;
                float sum = e[sub][i] + down + up;
                if (i > 0) sum = sum + e[sub][i - 1];
                if (i < 7) sum = sum + e[sub][i + 1];
                float col_bar = i == 0 ? first_col : (i == 1 ? second_col : (i == 7 ? last_col : middle_col));
                bool keep = sum >= col_bar;
                if (i == 0) {
                    float dc_var = lane_var[sub] * prof[i];
                    bool own = std::fabs(coeff) >= dc_lambda * std::sqrt(dc_var);
                    keep = dc_lane ? own : keep;
                    if (j == 0) keep = keep || dc_lane;
                }
                const bool live = j < k_use;
                if (wiener && live && keep) {
                    const float cv = lane_var[sub] * prof[i];
                    const float zz = coeff * coeff;
                    const float den = zz + cv;
                    const float gain = den > 0.0f ? zz / den : 1.0f;
                    kept_profile = kept_profile + (gain * gain) * prof[i];
                    out[sub][i] = gain * coeff;
                } else {
                    kept_profile = kept_profile + (keep ? prof[i] : 0.0f);
                    out[sub][i] = (live && !keep) ? 0.0f : coeff;
                }
                if (keep && live) bits[sub] |= uint64_t{1} << (j * 8 + i);
            }
            if (j < k_use) retained[sub] = retained[sub] + kept_profile * lane_var[sub];
        }
        for (int sub = 0; sub < P; ++sub)
            for (int i = 0; i < P; ++i) s.v[j][sub][i] = out[sub][i];
    }
}

void process_reference(const CollabArgs& a, uint32_t ref_x_index, uint32_t ref_y_index, uint32_t refs_x) {
    const uint32_t max_x = a.width - P, max_y = a.height - P;
    const uint32_t rx = std::min<uint32_t>(ref_x_index * STEP, max_x);
    const uint32_t ry = std::min<uint32_t>(ref_y_index * STEP, max_y);
    const int C = a.channels;
    const float scale = C == 1 ? 3.0f : 1.5f;
    Group g(a);
    for (int sub = 0; sub < P; ++sub)
        for (int r = 0; r < P; ++r)
            for (int c = 0; c < C; ++c) g.cur[sub][r][c] = g.px(a.centre_slot, rx + sub, ry + r, c);

    // Centre search over the clipped spatial rectangle, row by row (centre.rs:213-258).
    float best_d[MAX_K];
    uint32_t best_pos[MAX_K];
    for (int k = 0; k < MAX_K; ++k) {
        best_d[k] = UNFILLED;
        best_pos[k] = 0;
    }
    const uint32_t left = clamp_top_left(static_cast<int>(rx) - a.spatial_radius, max_x);
    const uint32_t right = clamp_top_left(static_cast<int>(rx) + a.spatial_radius, max_x);
    const uint32_t top = clamp_top_left(static_cast<int>(ry) - a.spatial_radius, max_y);
    const uint32_t bottom = clamp_top_left(static_cast<int>(ry) + a.spatial_radius, max_y);
    for (uint32_t cy = top; cy <= bottom; ++cy)
        for (uint32_t cx = left; cx <= right; ++cx) {
            float d = g.distance(g.cur, cx, cy, a.centre_slot, scale);
            if (cx == rx && cy == ry) d = SELF_PIN;
            if (d < best_d[MAX_K - 1]) shift_insert8(best_d, best_pos, d, pack_pos_t(cx, cy, 0));
        }
    const uint32_t n_live = (right - left + 1) * (bottom - top + 1);
    uint32_t k_use = 1;
    while (k_use * 2 <= n_live && k_use * 2 <= static_cast<uint32_t>(a.k_max)) k_use *= 2;
    uint32_t member_pos[MAX_K];
    for (int m = 0; m < MAX_K; ++m) member_pos[m] = best_pos[m];

    // Volumes across the neighbour frames (mod.rs:453-531).
    bool use_grid = false;
    if (a.grid_frames > 1 && a.k_max == MAX_K) {
        const int gf = a.grid_frames, volumes = MAX_K / gf, tail = gf - 1;
        uint32_t grid_pos[MAX_K];
        float grid_d[MAX_K];
        for (int vol = 0; vol < volumes; ++vol) {
            const int first = vol * gf;
            const uint32_t anchor_packed = member_pos[vol];
            const uint32_t ax = unpack_x(anchor_packed), ay = unpack_y(anchor_packed);
            grid_pos[first] = anchor_packed;
            grid_d[first] = 0.0f;
            for (int j = 0; j < tail; ++j) {
                grid_pos[first + 1 + j] = 0;
                grid_d[first + 1 + j] = UNFILLED;
            }
            float anchor[P][P][2];
            for (int sub = 0; sub < P; ++sub)
                for (int r = 0; r < P; ++r)
                    for (int c = 0; c < C; ++c) anchor[sub][r][c] = g.px(a.centre_slot, ax + sub, ay + r, c);
            trajectory_search(g, anchor, ax, ay, scale, grid_d, grid_pos, first + 1, tail);
        }
        use_grid = k_use == MAX_K;
        for (int vol = 0; vol < volumes; ++vol) use_grid = use_grid && grid_d[vol * gf + tail] < UNFILLED;
        if (use_grid) {
            for (int m = 0; m < MAX_K; ++m) member_pos[m] = grid_pos[m];
            k_use = MAX_K;
        }
    }

    if (a.member_record) {
        uint32_t* words = a.member_record + static_cast<size_t>(ref_y_index * refs_x + ref_x_index) * (MAX_K + 1);
        for (int m = 0; m < MAX_K; ++m) words[m] = member_pos[m];
        words[MAX_K] = k_use | (use_grid ? 0x100u : 0u);
    }

    // filter_group (mod.rs:559-850).
    int member_slot[MAX_K];
    for (int m = 0; m < MAX_K; ++m) {
        uint32_t t = unpack_t(member_pos[m]);
        member_slot[m] = t > 0 ? static_cast<int>(a.neighbour_slots[t - 1]) : a.centre_slot;
    }
    float col_first[P], col_second[P];
    for (int sub = 0; sub < P; ++sub) {
        float s0 = 0.0f, s1 = 0.0f;
        for (int r = 0; r < P; ++r) {
            s0 = s0 + g.cur[sub][r][0];
            if (C > 1) s1 = s1 + g.cur[sub][r][1];
        }
        col_first[sub] = s0;
        col_second[sub] = s1;
    }
    const float patch_luma = reduce8(col_first) / 64.0f;
    const float patch_second = C > 1 ? reduce8(col_second) / 64.0f : 0.0f;
    const float bins = static_cast<float>(CURVE_BINS);
    const float curve_pos = std::min(std::max(patch_luma * bins - 0.5f, 0.0f), bins - 1.0f);
    const uint32_t lower = std::min<uint32_t>(static_cast<uint32_t>(curve_pos), CURVE_BINS - 2);
    const float fraction = curve_pos - static_cast<float>(lower);
    float ratio = 0.0f;
    if (a.noise_curve) {
        const float lo = a.noise_curve[lower], hi = a.noise_curve[lower + 1];
        ratio = lo + (hi - lo) * fraction;
    }
    // fused/colour.rs:48-83 (`threshold_gains`): a luma patch reads its own mean luma and its block's
    // Cb and Cr, a chroma patch its own Cb and Cr and its block's luma.
    float first_gain = 1.0f, second_gain = 1.0f;
    if (a.colour_on) {
        const uint32_t bx = (rx + P / 2) / 16, by = (ry + P / 2) / 16;
        const float* m = a.colour_means + (by * static_cast<uint32_t>(a.colour_blocks_x) + bx) * 3;
        if (C == 1) {
            first_gain = mirror::exp_mirror(colour_table::table_value(a.colour_gains, patch_luma * a.colour_scale,
                                                                      m[1], m[2]));
        } else {
            const float cb = patch_luma * a.colour_scale - 128.0f, cr = patch_second * a.colour_scale - 128.0f;
            first_gain = mirror::exp_mirror(colour_table::table_value(a.colour_gains, m[0], cb, cr));
            second_gain = mirror::exp_mirror(colour_table::table_value(a.colour_gains + colour_table::CELLS, m[0],
                                                                       cb, cr));
        }
    }
    // A luma gain joins the curve's scale, and a chroma gain scales its channel's threshold.
    float curve_gain = 1.0f, first_channel_gain = first_gain, scale_max = CURVE_SCALE_MAX;
    if (C == 1) {
        curve_gain = first_gain;
        first_channel_gain = 1.0f;
        scale_max = a.colour_on ? COLOUR_CURVE_SCALE_MAX : CURVE_SCALE_MAX;
    }
    const float curve_scale = std::min(std::max(ratio * curve_gain, CURVE_SCALE_MIN), scale_max);
    const float flat_scale = std::min(std::max(curve_gain, CURVE_SCALE_MIN), scale_max);
    const float luma_scale = a.curve_valid ? curve_scale : flat_scale;
    const float first_lambda = (a.lambda_ht * luma_scale) * first_channel_gain;
    const float second_lambda = a.lambda_ht * second_gain;
    const uint32_t ref_idx = ref_y_index * refs_x + ref_x_index;
    float scaled_weight = 0.0f;
    const int plane = a.width * a.height;

    for (int c = 0; c < C; ++c) {
        const float sig = a.sigma[c];
        const float base_sig2 = sig * sig;
        Stack s;
        float mv[MAX_K];
        for (int m = 0; m < MAX_K; ++m) {
            const uint32_t mx = unpack_x(member_pos[m]), my = unpack_y(member_pos[m]);
            mv[m] = base_sig2;
            for (int sub = 0; sub < P; ++sub)
                for (int r = 0; r < P; ++r) s.v[m][sub][r] = g.px(member_slot[m], mx + sub, my + r, c);
        }
        if (a.grid_frames > 1 && use_grid) {
            grid_variance(mv, a.grid_frames);
        } else {
            if (k_use >= 8) variance_level(mv, 8);
            if (k_use >= 4) variance_level(mv, 4);
            if (k_use >= 2) variance_level(mv, 2);
        }
        // Column DCT, transpose, row DCT: lane v ends holding coefficient (u = i, v) at slot i.
        for (int m = 0; m < MAX_K; ++m) {
            for (int sub = 0; sub < P; ++sub) dct8_fwd(s.v[m][sub]);
            float t[P][P];
            for (int sub = 0; sub < P; ++sub)
                for (int i = 0; i < P; ++i) t[sub][i] = s.v[m][i][sub];
            std::memcpy(s.v[m], t, sizeof(t));
            for (int sub = 0; sub < P; ++sub) dct8_fwd(s.v[m][sub]);
        }
        if (a.grid_frames > 1 && use_grid) {
            grid_fwd(s, a.grid_frames);
        } else {
            if (k_use >= 8) haar_fwd_level(s, 8);
            if (k_use >= 4) haar_fwd_level(s, 4);
            if (k_use >= 2) haar_fwd_level(s, 2);
        }
        const float channel_lambda = c == 0 ? first_lambda : second_lambda;
        float retained[P];
        uint64_t bits[P] = {};
        if (a.pooled) {
            pooled_threshold(s, mv, a.dct_profile, static_cast<int>(k_use), channel_lambda * a.pool_ratio,
                             channel_lambda, a.wiener != 0, retained, bits);
        } else {
            for (int sub = 0; sub < P; ++sub) {
                const float prof_sub = a.dct_profile[sub];
                float rv = 0.0f;
                for (int i = 0; i < P; ++i) {
                    const float factor = a.dct_profile[i] * prof_sub;
                    for (int j = 0; j < MAX_K; ++j) {
                        if (j >= static_cast<int>(k_use)) continue;
                        const float cv = mv[j] * factor;
                        float& coeff = s.v[j][sub][i];
                        bool keep = std::fabs(coeff) >= channel_lambda * std::sqrt(cv);
                        if (j == 0 && i == 0 && sub == 0) keep = true;
                        if (keep && a.wiener) {
                            const float zz = coeff * coeff;
                            const float den = zz + cv;
                            const float gain = den > 0.0f ? zz / den : 1.0f;
                            coeff = gain * coeff;
                            rv = rv + (gain * gain) * cv;
                        } else if (keep) {
                            rv = rv + cv;
                        } else {
                            coeff = 0.0f;
                        }
                        if (keep) bits[sub] |= uint64_t{1} << (j * 8 + i);
                    }
                }
                retained[sub] = rv;
            }
        }
        if (a.mask_record)
            for (int sub = 0; sub < P; ++sub) a.mask_record[(static_cast<size_t>(ref_idx) * C + c) * P + sub] = bits[sub];
        const float sum = reduce8(retained);
        const float weight = safe_reciprocal(sum, RECIPROCAL_FLOOR);
        if (c == 0) {
            a.group_weight[ref_idx] = weight;
            scaled_weight = weight * a.weight_scale;
        }
        if (a.grid_frames > 1 && use_grid) {
            grid_inv(s, a.grid_frames);
        } else {
            if (k_use >= 2) haar_inv_level(s, 2);
            if (k_use >= 4) haar_inv_level(s, 4);
            if (k_use >= 8) haar_inv_level(s, 8);
        }
        for (int m = 0; m < MAX_K; ++m) {
            for (int sub = 0; sub < P; ++sub) dct8_inv(s.v[m][sub]);
            float t[P][P];
            for (int sub = 0; sub < P; ++sub)
                for (int i = 0; i < P; ++i) t[sub][i] = s.v[m][i][sub];
            std::memcpy(s.v[m], t, sizeof(t));
            for (int sub = 0; sub < P; ++sub) dct8_inv(s.v[m][sub]);
        }
        // aggregate.rs:176-211 (`scatter_patch`): Kaiser taper, fixed point, integer adds.
        for (int m = 0; m < static_cast<int>(k_use); ++m) {
            const uint32_t mx = unpack_x(member_pos[m]), my = unpack_y(member_pos[m]);
            for (int r = 0; r < P; ++r)
                for (int sub = 0; sub < P; ++sub) {
                    const float window = a.kaiser[r] * a.kaiser[sub];
                    const float w = scaled_weight * window;
                    const size_t pixel = static_cast<size_t>(member_slot[m]) * plane + (my + r) * a.width + mx + sub;
                    a.accum[pixel * C + c] += to_fixed(s.v[m][sub][r] * w, a.accum_scale);
                    if (c == 0) a.wsum[pixel] += to_fixed_weight(w, a.accum_scale);
                }
        }
    }
}

uint32_t refs_along(uint32_t dim) { return (dim - P + STEP - 1) / STEP + 1; }

}  // namespace

extern "C" {

// The whole `collab_fused` launch: every reference patch of the centre slot, scattered into the
// accumulators (which the caller zeroes). Sequential, so the integer adds land in a fixed order.
void orc_collab_fused(const CollabArgs* args) {
    const CollabArgs& a = *args;
    const uint32_t refs_x = refs_along(a.width), refs_y = refs_along(a.height);
    for (uint32_t iy = 0; iy < refs_y; ++iy)
        for (uint32_t ix = 0; ix < refs_x; ++ix) process_reference(a, ix, iy, refs_x);
}

// transforms.rs:196-221 (`dct_noise_profile`), in f64, rounded to f32.
void orc_dct_noise_profile(float rho, float* out) {
    if (rho <= 0.0f) {
        for (int i = 0; i < 8; ++i) out[i] = 1.0f;
        return;
    }
    double r = rho;
    for (int u = 0; u < 8; ++u) {
        double sum = 0.0;
        for (int i = 0; i < 8; ++i)
            for (int j = 0; j < 8; ++j) {
                double bi = (u == 0 ? 1.0 / std::sqrt(8.0) : 0.5) * std::cos(M_PI * (2.0 * i + 1.0) * u / 16.0);
                double bj = (u == 0 ? 1.0 / std::sqrt(8.0) : 0.5) * std::cos(M_PI * (2.0 * j + 1.0) * u / 16.0);
                sum += bi * bj * std::pow(r, std::abs(i - j));
            }
        out[u] = static_cast<float>(sum);
    }
}

// aggregate.rs:101-132 (`kaiser_window`).
void orc_kaiser_window(float beta, float* out) {
    auto i0 = [](double x) {
        double half = x / 2.0, term = 1.0, sum = 1.0;
        for (int k = 1; k < 32; ++k) {
            term *= half / k;
            sum += term * term;
        }
        return sum;
    };
    double denom = i0(beta);
    for (int i = 0; i < 8; ++i) {
        double pos = 2.0 * i / 7.0 - 1.0;
        double radius = std::sqrt(1.0 - pos * pos);
        out[i] = static_cast<float>(i0(beta * radius) / denom);
    }
}

// aggregate.rs:33-54 (`cross_frame_accum_scale`).
float orc_cross_frame_accum_scale(uint32_t spatial_radius, uint32_t temporal_radius) {
    uint32_t refs_per_axis = ((P - 1) + 2 * spatial_radius) / STEP + 1;
    double contribs = static_cast<double>(refs_per_axis) * refs_per_axis * MAX_K;
    double passes = 4.0 * temporal_radius + 1.0;
    double max_raw = contribs * passes * ACCUM_CLAMP;
    double budget = 2147483647.0 / 2.0;
    double exponent = std::floor(std::log2(budget / max_raw));
    return static_cast<float>(std::pow(2.0, exponent));
}

}  // extern "C"
