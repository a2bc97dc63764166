"""Seeded inputs for the motion search tests: textured frames moved by whole pixels, the frames the
reference's block-match tests build (av-denoise-core/src/motion/tests/block_match.rs:97-330)."""

from __future__ import annotations

import numpy as np


def textured(width: int, height: int, seed: int) -> np.ndarray:
    """A frame of smooth structure plus fine texture in [0, 1], so every offset scores differently."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:height, 0:width].astype(np.float32)
    f = 0.5 + 0.2 * np.sin(x * 0.21 + 0.7 * np.sin(y * 0.05)) * np.cos(y * 0.17)
    f += rng.normal(0.0, 0.08, (height, width)).astype(np.float32)
    return np.clip(f, 0.0, 1.0).astype(np.float32)


def shifted(frame: np.ndarray, dx: int, dy: int) -> np.ndarray:
    """neighbour(x, y) = frame(x - dx, y - dy), edges repeated: the block at p matches at p + (dx, dy)."""
    h, w = frame.shape
    ys = np.clip(np.arange(h) - dy, 0, h - 1)
    xs = np.clip(np.arange(w) - dx, 0, w - 1)
    return frame[ys][:, xs]


def moving_window(width: int, height: int, frames: int, seed: int, channels: int = 1) -> np.ndarray:
    """A window of frames under per-frame global motion plus one sprite moving its own way, with
    fresh noise on every frame; returned as a ring (frames, height, width, channels)."""
    rng = np.random.default_rng(seed)
    base = textured(width + 64, height + 64, seed)
    out = np.empty((frames, height, width, channels), np.float32)
    sprite = textured(24, 24, seed + 1)
    for t in range(frames):
        gx, gy = int(rng.integers(-5, 6)), int(rng.integers(-5, 6))
        f = base[32 + gy:32 + gy + height, 32 + gx:32 + gx + width].copy()
        sx, sy = (7 + 3 * t) % max(width - 24, 1), (5 + 2 * t) % max(height - 24, 1)
        f[sy:sy + 24, sx:sx + 24] = sprite[:min(24, height - sy), :min(24, width - sx)]
        f += rng.normal(0.0, 0.02, f.shape).astype(np.float32)
        for c in range(channels):
            out[t, :, :, c] = f if c == 0 else 1.0 - f
    return out
