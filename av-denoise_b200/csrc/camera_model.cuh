// The camera model's prediction at a block (av-denoise-core/src/motion/kernels/candidates.rs:71-134),
// shared by the block search and the truemotion stage. A prediction is 6 f32 words per neighbour,
// m00 m01 m10 m11 tx ty, mapping a full-resolution point of the centre frame into the neighbour.
#pragma once

#include <cuda_runtime.h>

#include "kernels.h"

namespace avd {

// candidates.rs:123-134 (`predicts_motion`): whether the prediction `p` moves anything.
__device__ __forceinline__ bool predicts_motion(const float* p) {
    return p[0] != 1.0f || p[3] != 1.0f || p[1] != 0.0f || p[2] != 0.0f || p[4] != 0.0f || p[5] != 0.0f;
}

// candidates.rs:71-121 (`model_displacement`): the motion `p` gives the centre of the block at (ox, oy)
// on a level `scale` times smaller, capped to the level's size (lw, lh) and rounded with
// floor(x + 0.5); every product and sum rounds on its own, in the reference's order.
__device__ __forceinline__ void model_point(const float* p, int ox, int oy, int blksize, int scale, int lw, int lh,
                                            int* dx, int* dy) {
    const float s = static_cast<float>(scale);
    const int half = blksize / 2;
    const float cx = __fmul_rn(static_cast<float>(ox + half), s);
    const float cy = __fmul_rn(static_cast<float>(oy + half), s);
    const float mx = __fadd_rn(__fadd_rn(__fmul_rn(p[0], cx), __fmul_rn(p[1], cy)), p[4]);
    const float my = __fadd_rn(__fadd_rn(__fmul_rn(p[2], cx), __fmul_rn(p[3], cy)), p[5]);
    float ldx = __fdiv_rn(__fsub_rn(mx, cx), s), ldy = __fdiv_rn(__fsub_rn(my, cy), s);
    const float limx = static_cast<float>(lw), limy = static_cast<float>(lh);
    ldx = ldx < -limx ? -limx : (ldx > limx ? limx : ldx);
    ldy = ldy < -limy ? -limy : (ldy > limy ? limy : ldy);
    const float rx = floorf(__fadd_rn(ldx, 0.5f)), ry = floorf(__fadd_rn(ldy, 0.5f));
    *dx = isnan(rx) ? 0 : static_cast<int>(rx);
    *dy = isnan(ry) ? 0 : static_cast<int>(ry);
}

}  // namespace avd
