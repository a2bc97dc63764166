// Host side of the NL4D kernel-level entry points: the collab pass launcher and the reference's
// public helper tables (DCT noise profile, Kaiser taps, fixed-point scale).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "avd_internal.h"
#include "kernels.h"

void avd_set_last_error(const std::string& m);

namespace {
constexpr double kPi = 3.14159265358979323846;
double dct_basis(int row, int col) {
    const double scale = row == 0 ? 1.0 / std::sqrt(8.0) : 0.5;
    return scale * std::cos(kPi * (2.0 * col + 1.0) * row / 16.0);
}
}  // namespace

extern "C" {

void avd_dct_noise_profile(float rho, float* out8) {
    if (!out8) return;
    if (rho <= 0.0f) {
        for (int i = 0; i < 8; ++i) out8[i] = 1.0f;
        return;
    }
    const double r = rho;
    for (int u = 0; u < 8; ++u) {
        double sum = 0.0;
        for (int i = 0; i < 8; ++i)
            for (int j = 0; j < 8; ++j) sum += dct_basis(u, i) * dct_basis(u, j) * std::pow(r, std::abs(i - j));
        out8[u] = static_cast<float>(sum);
    }
}

void avd_kaiser_window(float beta, float* out8) {
    if (!out8) return;
    auto i0 = [](double x) {
        double half = x / 2.0, term = 1.0, sum = 1.0;
        for (int k = 1; k < 32; ++k) {
            term *= half / k;
            sum += term * term;
        }
        return sum;
    };
    const double denom = i0(beta);
    for (int i = 0; i < 8; ++i) {
        const double pos = 2.0 * i / 7.0 - 1.0;
        out8[i] = static_cast<float>(i0(beta * std::sqrt(1.0 - pos * pos)) / denom);
    }
}

uint64_t avd_collab_member_bytes(uint32_t width, uint32_t height) {
    return avd::collab_member_words(static_cast<int>(width), static_cast<int>(height)) * sizeof(uint32_t);
}

float avd_cross_frame_accum_scale(uint32_t spatial_radius, uint32_t temporal_radius) {
    const uint32_t refs_per_axis = (7 + 2 * spatial_radius) / 4 + 1;
    const double contribs = static_cast<double>(refs_per_axis) * refs_per_axis * 8.0;
    const double max_raw = contribs * (4.0 * temporal_radius + 1.0) * 5.0;
    const double exponent = std::floor(std::log2((2147483647.0 / 2.0) / max_raw));
    return static_cast<float>(std::pow(2.0, exponent));
}

}  // extern "C"

namespace {

// The checked launch arguments of one pass, or the status that refuses it.
AvdStatus pass_launch(const AvdCollabPass* p, avd::CollabLaunch& a) {
    if (!p || !p->ring || !p->accum || !p->wsum || !p->group_weight || !p->noise || !p->dct_profile || !p->kaiser ||
        !p->members)
        return AVD_ERR_NULL_ARG;
    if (p->width < 8 || p->height < 8 || (p->channels != 1 && p->channels != 2) || p->k_max < 1 || p->k_max > 8 ||
        p->radius > 8 || p->spatial_radius > 16 || p->refine > 4 || p->blk_step == 0 ||
        (p->blksize + p->blk_step - 1) / p->blk_step > 4) {
        avd_set_last_error("collab pass arguments out of range");
        return AVD_ERR_INVALID_OPTIONS;
    }
    if (p->radius > 0 && (!p->mv_field || !p->confidence || !p->neighbour_slots)) return AVD_ERR_NULL_ARG;
    a = avd::CollabLaunch{};
    a.ring = reinterpret_cast<const float*>(p->ring);
    a.width = static_cast<int>(p->width);
    a.height = static_cast<int>(p->height);
    a.channels = static_cast<int>(p->channels);
    a.centre_slot = static_cast<int>(p->centre_slot);
    a.frame_elems = static_cast<int64_t>(p->width) * p->height * p->channels;
    a.mv_field = reinterpret_cast<const int32_t*>(p->mv_field);
    a.confidence = reinterpret_cast<const float*>(p->confidence);
    a.neighbour_slots = reinterpret_cast<const uint32_t*>(p->neighbour_slots);
    a.noise = reinterpret_cast<const float*>(p->noise);
    a.sigma_word = static_cast<int>(p->sigma_word);
    a.weight_scale_word = static_cast<int>(p->weight_scale_word);
    a.curve_valid_word = static_cast<int>(p->curve_valid_word);
    a.noise_curve = reinterpret_cast<const float*>(p->noise_curve);
    a.dct_profile = reinterpret_cast<const float*>(p->dct_profile);
    a.kaiser = reinterpret_cast<const float*>(p->kaiser);
    a.accum = reinterpret_cast<int32_t*>(p->accum);
    a.wsum = reinterpret_cast<int32_t*>(p->wsum);
    a.group_weight = reinterpret_cast<float*>(p->group_weight);
    a.members = reinterpret_cast<uint32_t*>(p->members);
    a.c_min = p->c_min;
    a.lambda_ht = p->lambda_ht;
    a.accum_scale = p->accum_scale;
    a.pool_ratio = p->pool_ratio;
    a.pooled = static_cast<int>(p->pooled);
    a.radius = static_cast<int>(p->radius);
    a.refine = static_cast<int>(p->refine);
    a.spatial_radius = static_cast<int>(p->spatial_radius);
    a.k_max = static_cast<int>(p->k_max);
    a.mv_stride = static_cast<int>(p->mv_stride);
    a.conf_stride = static_cast<int>(p->conf_stride);
    a.blk_step = static_cast<int>(p->blk_step);
    a.blksize = static_cast<int>(p->blksize);
    a.blocks_x = static_cast<int>(p->blocks_x);
    a.blocks_y = static_cast<int>(p->blocks_y);
    a.wiener = p->wiener != 0;
    return AVD_OK;
}

}  // namespace

extern "C" {

AvdStatus avd_collab_pass(const AvdCollabPass* p, void* stream) {
    avd::CollabLaunch a;
    const AvdStatus st = pass_launch(p, a);
    if (st != AVD_OK) return st;
    cudaError_t e = avd::launch_collab(a, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        avd_set_last_error(std::string("collab launch: ") + cudaGetErrorString(e));
        return AVD_ERR_GPU;
    }
    return AVD_OK;
}

uint64_t avd_collab_refs(uint32_t width, uint32_t height) {
    if (width < 8 || height < 8) return 0;
    return static_cast<uint64_t>((width - 8 + 3) / 4 + 1) * ((height - 8 + 3) / 4 + 1);
}

AvdStatus avd_collab_adjoint(const AvdCollabPass* p, const AvdCollabAdjoint* adj, void* stream) {
    if (!adj || !adj->grad_accum || !adj->grad_wsum || !adj->grad_ring || !adj->grad_sigma_refs)
        return AVD_ERR_NULL_ARG;
    avd::CollabLaunch a;
    const AvdStatus st = pass_launch(p, a);
    if (st != AVD_OK) return st;
    avd::CollabAdjointLaunch b{};
    b.grad_accum = reinterpret_cast<const float*>(adj->grad_accum);
    b.grad_wsum = reinterpret_cast<const float*>(adj->grad_wsum);
    b.grad_ring = reinterpret_cast<float*>(adj->grad_ring);
    b.grad_sigma_refs = reinterpret_cast<float*>(adj->grad_sigma_refs);
    cudaError_t e = avd::launch_collab_adjoint(a, b, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        avd_set_last_error(std::string("collab adjoint launch: ") + cudaGetErrorString(e));
        return AVD_ERR_GPU;
    }
    return AVD_OK;
}

}  // extern "C"
