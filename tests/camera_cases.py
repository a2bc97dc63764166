"""Shared inputs of the camera-model tests: a continuous texture with no repeat, rendered through a
similarity camera (x' = a x - b y + tx, y' = b x + a y + ty), as the reference's producer tests render
theirs (av-denoise-core/src/motion/global/tests/producer.rs:183-247, with a hash of this file's own)."""

import numpy as np


def inverse(m):
    a, b, tx, ty = m
    n = a * a + b * b
    ia, ib = a / n, -b / n
    return ia, ib, -(ia * tx - ib * ty), -(ib * tx + ia * ty)


def _lattice(ix, iy, seed):
    """A hashed value in 0.2..0.8 per lattice point (a 32-bit integer mix of the cell and the seed)."""
    h = (ix.astype(np.uint64) * np.uint64(0x8DA6B343) ^ iy.astype(np.uint64) * np.uint64(0xD8163841)) & np.uint64(0xFFFFFFFF)
    h = (h ^ np.uint64(seed * 0x9E3779B9 & 0xFFFFFFFF)) & np.uint64(0xFFFFFFFF)
    for _ in range(3):
        h = ((h ^ (h >> np.uint64(16))) * np.uint64(0x45D9F3B)) & np.uint64(0xFFFFFFFF)
    return 0.2 + 0.6 * (h.astype(np.float64) / 4294967295.0)


def _value_noise(x, y, cell, seed):
    sx, sy = x / cell, y / cell
    cx, cy = np.floor(sx), np.floor(sy)
    bx = (sx - cx) ** 2 * (3 - 2 * (sx - cx))
    by = (sy - cy) ** 2 * (3 - 2 * (sy - cy))
    ix, iy = cx.astype(np.int64), cy.astype(np.int64)
    tl, tr = _lattice(ix, iy, seed), _lattice(ix + 1, iy, seed)
    bl, br = _lattice(ix, iy + 1, seed), _lattice(ix + 1, iy + 1, seed)
    up = tl + (tr - tl) * bx
    lo = bl + (br - bl) * bx
    return up + (lo - up) * by


def render(camera, width, height):
    """A frame of a continuous texture with no repeat, each pixel sampled where `camera` (a, b, tx,
    ty) came from."""
    a, b, tx, ty = inverse(camera)
    ys, xs = np.mgrid[0:height, 0:width].astype(np.float64)
    sx, sy = a * xs - b * ys + tx, b * xs + a * ys + ty
    v = 0.6 * _value_noise(sx, sy, 4.0, 1) + 0.4 * _value_noise(sx, sy, 11.0, 2)
    return v.astype(np.float32)
