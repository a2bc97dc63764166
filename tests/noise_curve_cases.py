"""Synthetic temporal records for the noise-curve tests, and a float32 host model of the curve.

The record builder restates the reference's test helpers (av-denoise-core/src/noise/tests/records.rs:
`hashed_unit`, `channel_sums`, `frame_records`, `static_block`, `BlockSpec::uniform`) and the curve
frame of noise/tests/curve.rs:40-111 (`CurveFrame`, `binned_quarter`): a luma frame of static blocks
whose quarters stay textured until a case places flat, unclipped quarters in chosen luma bins. The
arithmetic is float32, in the helpers' order, so the records are the ones the reference's tests
build.

`host_curve` restates the reference's host model of the curve (noise/curve.rs:71-235,
`build_noise_curve`) with numpy sorting, for the cases whose blocks all pass the reading's outlier
ceiling (every block here is static with a sigma of 2 to 4 codes, or moving and rejected by the
static gate).
"""

from __future__ import annotations

from dataclasses import dataclass, field, replace

import numpy as np

F = np.float32
NB = 16
BINS = 16
QUARTER = 8
STATIC_GATE = F(1.5) / F(255.0)
RHO_SIGMA_GATE = F(0.3) / F(255.0)
QUARTER_STATIC_GATE = F(2.0) * STATIC_GATE
CLIP_LOW = F(4.0) / F(255.0)
CLIP_HIGH = F(251.0) / F(255.0)
FLAT_FACTOR = F(0.5)
FLAT_FLOOR = (F(1.0) / F(255.0)) * (F(1.0) / F(255.0))
UNMEASURED_FLATNESS = F(3.0e38)
TEXTURED = F(1.0)
SQRT_2 = F(1.41421356237309504880)
MIN_QUARTERS_PER_BIN = 32
MIN_POPULATED_BINS = 3


def hashed_unit(seed: int, index: int) -> np.float32:
    m = 0xFFFFFFFF
    h = ((index * 0x9E3779B9) & m) ^ ((seed * 0x85EBCA6B) & m)
    h ^= h >> 15
    h = (h * 0x2C1B3C6D) & m
    h ^= h >> 12
    h = (h * 0x297A2D39) & m
    h ^= h >> 15
    return F(h >> 8) / F(1 << 24)


@dataclass
class QuarterSpec:
    mean: np.float32 = F(0)
    sigma: np.float32 = F(0)
    luma: np.float32 = F(0)
    flatness: np.float32 = F(0)
    luma_min: np.float32 = F(0)
    luma_max: np.float32 = F(0)


@dataclass
class BlockSpec:
    mean: np.float32 = F(0)
    sigma: np.float32 = F(0)
    rho: np.float32 = F(0)
    texture: np.float32 = F(0)
    moved: bool = False
    quarters: list = field(default_factory=lambda: [QuarterSpec() for _ in range(4)])


def uniform_block(mean, sigma, rho) -> BlockSpec:
    return BlockSpec(mean=F(mean), sigma=F(sigma), rho=F(rho))


def static_block(seed: int, index: int) -> BlockSpec:
    mean = (hashed_unit(seed, 4 * index) - F(0.5)) * STATIC_GATE
    rho = F(0.1) + F(0.4) * hashed_unit(seed, 4 * index + 1)
    sigma = (F(2.0) + F(2.0) * hashed_unit(seed, 4 * index + 2)) / F(255.0)
    return BlockSpec(mean=mean, sigma=sigma, rho=rho)


def binned_quarter(b: int, unit) -> QuarterSpec:
    luma = (F(b) + F(0.5)) / F(BINS)
    sigma = (F(3.0) + F(0.5) * F(b) + F(2.0) * F(unit)) / F(255.0)
    return QuarterSpec(mean=F(0), sigma=sigma, luma=luma, flatness=F(0), luma_min=luma - F(0.01),
                       luma_max=luma + F(0.01))


def channel_sums(mean, sigma, pixels):
    variance = F(2.0) * sigma * sigma
    return F(mean) * F(pixels), (variance + F(mean) * F(mean)) * F(pixels)


def blocks_of(w: int, h: int) -> tuple[int, int]:
    return -(-w // NB), -(-h // NB)


def block_dims(w: int, h: int, index: int) -> tuple[int, int]:
    bx, _ = blocks_of(w, h)
    return min(NB, w - (index % bx) * NB), min(NB, h - (index // bx) * NB)


def quarter_pixels(w: int, h: int, index: int, q: int) -> int:
    bw, bh = block_dims(w, h, index)
    qw = min(max(bw - (q % 2) * QUARTER, 0), QUARTER)
    qh = min(max(bh - (q // 2) * QUARTER, 0), QUARTER)
    return qw * qh


def frame_records(w: int, h: int, blocks: list[BlockSpec]) -> np.ndarray:
    """One luma frame's records (29 lanes per block), as noise/tests/records.rs:91-149 builds them."""
    bx, by = blocks_of(w, h)
    assert len(blocks) == bx * by
    rl = 29
    out = np.zeros(len(blocks) * rl, np.float32)
    for i, spec in enumerate(blocks):
        bw, bh = block_dims(w, h, i)
        pixels, pairs = F(bw * bh), F(bh * max(bw - 1, 0))
        r = out[i * rl:(i + 1) * rl]
        r[0], r[1] = channel_sums(spec.mean, spec.sigma, pixels)
        variance = F(2.0) * spec.sigma * spec.sigma
        r[2] = (spec.rho * variance + spec.mean * spec.mean) * pairs
        r[3] = spec.texture
        r[4] = 1.0 if spec.moved else 0.0
        for q, qs in enumerate(spec.quarters):
            qp = F(quarter_pixels(w, h, i, q))
            f = r[5 + 6 * q:11 + 6 * q]
            f[0], f[1] = channel_sums(qs.mean, qs.sigma, qp)
            f[2] = F(qs.luma) * qp
            f[3], f[4], f[5] = qs.flatness, qs.luma_min, qs.luma_max
    return out


class CurveFrame:
    """noise/tests/curve.rs:40-97: static blocks whose quarters are textured until placed."""

    def __init__(self, w: int, h: int, seed: int):
        self.w, self.h = w, h
        bx, by = blocks_of(w, h)
        textured = replace(binned_quarter(8, F(0.5)), flatness=TEXTURED)
        self.blocks = []
        for i in range(bx * by):
            b = static_block(seed, i)
            b.quarters = [replace(textured) for _ in range(4)]
            self.blocks.append(b)
        self.next = 0

    def place(self, count: int, quarter):
        for p in range(count):
            slot = self.next + p
            self.blocks[slot // 4].quarters[slot % 4] = quarter(p)
        self.next += count

    def place_bin(self, b: int, count: int):
        self.place(count, lambda p: binned_quarter(b, hashed_unit(b + 100, p)))

    def records(self) -> np.ndarray:
        return frame_records(self.w, self.h, self.blocks)


def _median(v: list) -> np.float32:
    s = np.sort(np.asarray(v, np.float32))
    n = len(s)
    return (s[(n - 1) // 2] + s[n // 2]) * F(0.5)


def host_curve(frame: CurveFrame, records: np.ndarray):
    """noise/curve.rs:71-235 on the frame's accepted blocks: the quarter median and the 16 ratios,
    or None without a curve."""
    rl = 29
    accepted, kept = [], []
    for i in range(len(frame.blocks)):
        bw, bh = block_dims(frame.w, frame.h, i)
        r = records[i * rl:(i + 1) * rl]
        pixels = F(bw * bh)
        mean = r[0] / pixels
        sigma = np.sqrt(max(r[1] / pixels - mean * mean, F(0))) / SQRT_2
        if abs(mean) < STATIC_GATE and sigma > RHO_SIGMA_GATE:
            accepted.append(i)
            kept.append(sigma)
    if not kept:
        return None
    sigma_block_median = _median(kept)
    quarters = []
    for i in accepted:
        for q in range(4):
            pixels = F(quarter_pixels(frame.w, frame.h, i, q))
            if pixels == 0:
                continue
            f = records[i * rl + 5 + 6 * q:i * rl + 11 + 6 * q]
            mean = f[0] / pixels
            if abs(mean) >= QUARTER_STATIC_GATE:
                continue
            sigma = np.sqrt(max(f[1] / pixels - mean * mean, F(0))) / SQRT_2
            if sigma <= RHO_SIGMA_GATE:
                continue
            quarters.append((sigma, f[2] / pixels, f[3], f[4], f[5]))
    if not quarters:
        return None
    quarter_median = _median([q[0] for q in quarters])
    if quarter_median <= 0:
        return None
    flat_limit = max(FLAT_FACTOR * sigma_block_median * sigma_block_median, FLAT_FLOOR)
    bins = [[] for _ in range(BINS)]
    for sigma, luma, flat, lo, hi in quarters:
        if flat > flat_limit or lo < CLIP_LOW or hi > CLIP_HIGH:
            continue
        bins[min(int(max(luma * F(BINS), F(0))), BINS - 1)].append(sigma)
    populated = [(b, _median(v)) for b, v in enumerate(bins) if len(v) >= MIN_QUARTERS_PER_BIN]
    if len(populated) < MIN_POPULATED_BINS:
        return None
    ratios = []
    for b in range(BINS):
        if b <= populated[0][0]:
            s = populated[0][1]
        elif b >= populated[-1][0]:
            s = populated[-1][1]
        else:
            up = next(k for k, (pb, _) in enumerate(populated) if pb >= b)
            (hi_b, hi_s), (lo_b, lo_s) = populated[up], populated[up - 1]
            s = lo_s + (hi_s - lo_s) * (F(b - lo_b) / F(hi_b - lo_b))
        ratios.append(s / quarter_median)
    return quarter_median, np.asarray(ratios, np.float32)


def ulp_gap(a, b) -> int:
    a, b = np.float32(a), np.float32(b)
    if np.isnan(a) or np.isnan(b):
        return 1 << 32
    ia = int(np.array(a).view(np.int32))
    ib = int(np.array(b).view(np.int32))
    ia = ia if ia >= 0 else -(ia & 0x7FFFFFFF)
    ib = ib if ib >= 0 else -(ib & 0x7FFFFFFF)
    return abs(ia - ib)


# The cases of noise/tests/curve.rs as (name, frame builder, expected populated bins, expected
# curve flag); every builder returns a CurveFrame.
def case_bins(seed):
    f = CurveFrame(256, 192, seed)
    for b in [1, 3, 7, 9, 13]:
        f.place_bin(b, 120)
    return f


def case_bin_count(count):
    f = CurveFrame(256, 192, 11)
    for b in [2, 6, 10]:
        f.place_bin(b, 40)
    f.place(count, lambda p: replace(binned_quarter(4, hashed_unit(4, p)),
                                     sigma=F(3.0) * binned_quarter(4, hashed_unit(4, p)).sigma))
    return f


def case_two_bins(third):
    f = CurveFrame(256, 192, 13)
    f.place_bin(3, 60)
    f.place_bin(11, 60)
    if third:
        f.place_bin(7, 60)
    return f


def flat_gate_frame():
    """noise/tests/curve.rs:262-307: quarters of bins 4 and 13 at 1.25 and 0.8 times the flat gate
    built from the blocks' sigma median; only bin 13's pass."""
    f = CurveFrame(256, 192, 17)
    blank = f.records()
    rl = 29
    sig = []
    for i in range(len(f.blocks)):
        bw, bh = block_dims(f.w, f.h, i)
        pixels = F(bw * bh)
        mean = blank[i * rl] / pixels
        sig.append(np.sqrt(max(blank[i * rl + 1] / pixels - mean * mean, F(0))) / SQRT_2)
    med = _median(sig)
    flat_limit = FLAT_FACTOR * med * med
    for b in [2, 6, 10]:
        f.place_bin(b, 40)
    for b, scale in [(4, 1.25), (13, 0.8)]:
        f.place(40, lambda p, b=b, scale=scale: replace(
            binned_quarter(b, hashed_unit(b, p)), sigma=F(3.0) * binned_quarter(b, hashed_unit(b, p)).sigma,
            flatness=F(scale) * flat_limit))
    return f


def clipped_frame():
    """noise/tests/curve.rs:309-366: quarters clipped high (bin 14) and low (bin 1) never bin; ones
    exactly at the clip limits (bin 13) do."""
    f = CurveFrame(256, 192, 19)
    for b in [2, 6, 10]:
        f.place_bin(b, 40)
    f.place(40, lambda p: replace(binned_quarter(14, hashed_unit(14, p)), luma_max=F(0.99)))
    f.place(40, lambda p: replace(binned_quarter(1, hashed_unit(1, p)), luma_min=F(0.01)))
    f.place(40, lambda p: replace(binned_quarter(13, hashed_unit(13, p)), luma_min=CLIP_LOW, luma_max=CLIP_HIGH))
    return f


def ragged_frame():
    """noise/tests/curve.rs:383-430: a 70x54 frame whose ragged quarters read the unmeasured
    flatness; only the 48 full quarters reach bin 8."""
    f = CurveFrame(70, 54, 23)
    slots = len(f.blocks) * 4

    def quarter(slot):
        px = quarter_pixels(f.w, f.h, slot // 4, slot % 4)
        ragged = 0 < px < QUARTER * QUARTER
        return replace(binned_quarter(8, hashed_unit(8, slot)), flatness=UNMEASURED_FLATNESS if ragged else F(0))

    f.place(slots, quarter)
    return f


def no_sample_frame(accepted):
    """noise/tests/curve.rs:432-457: only the first `accepted` blocks are static; the rest move and
    carry quarters that would fill bin 12."""
    f = CurveFrame(640, 360, 29)
    moving = binned_quarter(12, F(0.5))
    for i in range(accepted, len(f.blocks)):
        b = uniform_block(F(4.0) * STATIC_GATE, F(3.0) / F(255.0), 0.2)
        b.quarters = [replace(moving) for _ in range(4)]
        f.blocks[i] = b
    for b in [2, 6, 10]:
        f.place_bin(b, 50)
    return f


CASES = [
    ("bins_seed3", lambda: case_bins(3), 5, True),
    ("bins_seed5", lambda: case_bins(5), 5, True),
    ("bin_31_quarters", lambda: case_bin_count(31), 3, True),
    ("bin_32_quarters", lambda: case_bin_count(32), 4, True),
    ("two_bins", lambda: case_two_bins(False), 2, False),
    ("three_bins", lambda: case_two_bins(True), 3, True),
    ("flat_gate", flat_gate_frame, 4, True),
    ("clipped", clipped_frame, 4, True),
    ("ragged", ragged_frame, 1, False),
    ("no_sample_40", lambda: no_sample_frame(40), 3, False),
    ("no_sample_46", lambda: no_sample_frame(46), 3, True),
]
