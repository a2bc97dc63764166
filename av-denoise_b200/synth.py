"""Seeded synthetic clips with the shapes, value ranges and motion of the benchmark workloads.

The reference's benchmark clips are not available, so these stand in for them. One base image is
six sinusoidal gratings (frequency U(0.01, 0.3) cycles/px, random orientation, amplitude
U(5, 30)) over 40 axis-aligned rectangles of uniform intensity U(16, 235), plus a texture field
(uniform noise blurred with a Gaussian of sigma 1.5 px, scaled to amplitude 12), clipped to
[16, 235] (x4 -> [64, 940] for 10-bit, x16 for 12-bit). Frames move the base image (and any
sprites) by integer offsets and add Gaussian noise (plus optional signal-dependent noise), then
round and clamp to the bit depth. Chroma planes come from their own base images at chroma size,
moved by the luma motion halved on subsampled axes.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

try:
    from scipy.ndimage import gaussian_filter
except ImportError:  # pragma: no cover
    gaussian_filter = None


def _blur(a: np.ndarray, sigma: float) -> np.ndarray:
    if gaussian_filter is not None:
        return gaussian_filter(a, sigma, mode="wrap")
    # Separable fallback with a truncated kernel (4 sigma).
    r = int(4 * sigma + 0.5)
    x = np.arange(-r, r + 1)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    k /= k.sum()
    out = a
    for axis in (0, 1):
        out = sum(np.roll(out, i, axis=axis) * k[i + r] for i in range(-r, r + 1))
    return out


def base_image(rng: np.random.Generator, height: int, width: int) -> np.ndarray:
    """One base image in 8-bit code units (float64), clipped to [16, 235]."""
    img = np.full((height, width), 128.0)
    for _ in range(40):
        rw = int(rng.integers(max(2, width // 40), max(3, width // 4)))
        rh = int(rng.integers(max(2, height // 40), max(3, height // 4)))
        x0 = int(rng.integers(0, max(1, width - rw)))
        y0 = int(rng.integers(0, max(1, height - rh)))
        img[y0:y0 + rh, x0:x0 + rw] = rng.uniform(16, 235)
    yy, xx = np.mgrid[0:height, 0:width].astype(np.float64)
    for _ in range(6):
        f = rng.uniform(0.01, 0.3)
        th = rng.uniform(0, np.pi)
        amp = rng.uniform(5, 30)
        ph = rng.uniform(0, 2 * np.pi)
        img += amp * np.sin(2 * np.pi * f * (xx * np.cos(th) + yy * np.sin(th)) + ph)
    tex = _blur(rng.uniform(-1, 1, (height, width)), 1.5)
    tex *= 12.0 / max(np.abs(tex).max(), 1e-9)
    img += tex
    return np.clip(img, 16, 235)


@dataclass
class Sprite:
    image: np.ndarray
    x: int
    y: int
    vx: int
    vy: int


def _paste(canvas: np.ndarray, sprite: np.ndarray, x: int, y: int) -> None:
    h, w = canvas.shape
    sh, sw = sprite.shape
    x0, y0 = max(x, 0), max(y, 0)
    x1, y1 = min(x + sw, w), min(y + sh, h)
    if x0 < x1 and y0 < y1:
        canvas[y0:y1, x0:x1] = sprite[y0 - y:y1 - y, x0 - x:x1 - x]


def make_clip(width: int, height: int, frames: int, *, depth: int = 8, chroma: str = "420",
              sigma_luma: float = 10.0, sigma_chroma: float = 5.0, offsets: list[tuple[int, int]] | None = None,
              global_motion: int = 0, sprites: int = 0, sprite_size: int = 200, sprite_speed: int = 0,
              signal_dependent: float = 0.0, seed: int = 0) -> list[list[np.ndarray]]:
    """Returns `frames` frames, each a list of planes of integer codes (uint8 for depth 8, uint16
    otherwise): [Y] for chroma "gray", [Y, U, V] otherwise.

    Motion: `offsets` gives each frame's integer (x, y) shift of the base image; otherwise
    `global_motion=g` draws an integer pan in
    [-g, g] per frame, accumulated. `sprites` textured squares of `sprite_size` move at integer
    velocities in [-sprite_speed, sprite_speed] (or with the pan when the speed is 0, each with its
    own random pan). Noise sigmas are in codes of the 8-bit scale (multiplied by 2^(depth-8))."""
    rng = np.random.default_rng(seed)
    scale = float(1 << (depth - 8))
    maxc = (1 << depth) - 1
    subs = {"gray": None, "420": (2, 2), "422": (2, 1), "444": (1, 1)}[chroma]

    # Motion offsets per frame.
    if offsets is not None:
        offs = list(offsets)
    else:
        offs = [(0, 0)]
        for _ in range(1, frames):
            dx, dy = rng.integers(-global_motion, global_motion + 1, size=2) if global_motion else (0, 0)
            offs.append((offs[-1][0] + int(dx), offs[-1][1] + int(dy)))
    mx = max(abs(o[0]) for o in offs) + 2
    my = max(abs(o[1]) for o in offs) + 2

    def plane_series(pw: int, ph: int, sx: int, sy: int, sigma: float) -> list[np.ndarray]:
        base = base_image(rng, ph + 2 * (my // sy + 1), pw + 2 * (mx // sx + 1))
        spr = []
        for _ in range(sprites):
            size = max(4, sprite_size // max(sx, sy))
            img = base_image(rng, size, size)
            v = (int(rng.integers(-sprite_speed, sprite_speed + 1)), int(rng.integers(-sprite_speed, sprite_speed + 1))) \
                if sprite_speed else (int(rng.integers(-4, 5)), int(rng.integers(-4, 5)))
            spr.append(Sprite(img, int(rng.integers(0, max(1, pw - size))), int(rng.integers(0, max(1, ph - size))),
                              v[0], v[1]))
        out = []
        oy0, ox0 = my // sy + 1, mx // sx + 1
        for k in range(frames):
            ox, oy = offs[k][0] // sx, offs[k][1] // sy
            fr = base[oy0 + oy:oy0 + oy + ph, ox0 + ox:ox0 + ox + pw].copy()
            for s_ in spr:
                _paste(fr, s_.image, s_.x + k * s_.vx // sx, s_.y + k * s_.vy // sy)
            fr = fr * scale
            noise = rng.normal(0.0, sigma * scale, fr.shape)
            if signal_dependent > 0.0:
                noise += rng.normal(0.0, 1.0, fr.shape) * np.sqrt(signal_dependent * fr)
            codes = np.clip(np.rint(fr + noise), 0, maxc)
            out.append(codes.astype(np.uint8 if depth == 8 else np.uint16))
        return out

    luma = plane_series(width, height, 1, 1, sigma_luma)
    if subs is None:
        return [[y] for y in luma]
    cw, ch = (width + subs[0] - 1) // subs[0], (height + subs[1] - 1) // subs[1]
    u = plane_series(cw, ch, subs[0], subs[1], sigma_chroma)
    v = plane_series(cw, ch, subs[0], subs[1], sigma_chroma)
    return [[luma[k], u[k], v[k]] for k in range(frames)]


def spatial_clip(seed: int = 0, frames: int = 8, width: int = 640, height: int = 360) -> list[list[np.ndarray]]:
    """8 luma frames of 640x360 u8, frame k shifted by (k, k/2) px, sigma 10."""
    return make_clip(width, height, frames, depth=8, chroma="gray", sigma_luma=10.0,
                     offsets=[(k, k // 2) for k in range(frames)], seed=seed)


def temporal_1080p_clip(seed: int = 1000, frames: int = 32, width: int = 1920, height: int = 1080):
    """1080p 4:2:0 u8, integer global pan in [-4, 4] per frame plus 3 moving 200x200 sprites,
    sigma 8 on luma and 5 on chroma."""
    return make_clip(width, height, frames, depth=8, chroma="420", sigma_luma=8.0, sigma_chroma=5.0,
                     global_motion=4, sprites=3, sprite_size=200, seed=seed)
