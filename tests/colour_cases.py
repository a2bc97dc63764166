"""Scenes for the colour grain gain tests, and a float64 host model of the fit.

The scene builders restate the reference's test scenes (av-denoise-core/src/noise/tests/colour.rs
`ColourBlock`, `CellRun`; noise/tests/colour_fit.rs `FitBlock`, `SceneRng`, `random_scene`,
`cell_scene`, `FitRun`): blocks with a mean colour on the 8-bit scale and a grain in codes, turned
into temporal records (a static residual of that sigma) and block means, pooled frame by frame into
a window of cell sums.

`host_fit` is a float64 model of the fit written from the reference's description of it
(noise/kernels/colour_fit.rs: the brightness base by penalised least squares solved exactly, the
Gaussian-kernel lift, the pulled and filled table, the ceilings, the normaliser median by bisection,
the ramps), against which the float32 oracle must agree to 1e-4, as the reference's own test
(`gpu_fit_matches_the_host_reference`) holds its kernels.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

CELLS = 976
PER_BRIGHTNESS = 61
HUES = 12
WORDS = 69
SAT_CENTRES = [3.0, 9.0, 16.0, 25.0, 37.0, 51.0]
SAT_EDGES = [6.0, 12.0, 20.0, 30.0, 44.0]
LOG_MIN, LOG_STEP, HIST_BINS = -3.5, 0.125, 64
KNOTS = 17
FRAME_WIDTH = 1024
FRAME_BLOCKS = 64 * 64
F = np.float32


def record_len(channels: int) -> int:
    return 3 * channels + 26


def texture_lane(channels: int, c: int) -> int:
    return 2 * channels + 1 if c == 0 else 2 * channels + 3 + 24 + c - 1


def block_records(grains, means_codes, channels: int, w: int, h: int) -> np.ndarray:
    """Temporal records of static blocks: channel c of block i holds a residual of mean
    means_codes[i][c] and sigma grains[i][c], both in codes (noise/tests/records.rs:82-149)."""
    bx, by = -(-w // 16), -(-h // 16)
    assert len(grains) == bx * by
    rl = record_len(channels)
    out = np.zeros(bx * by * rl, np.float32)
    for i, (g, m) in enumerate(zip(grains, means_codes)):
        bw, bh = min(16, w - (i % bx) * 16), min(16, h - (i // bx) * 16)
        pixels = F(bw * bh)
        r = out[i * rl:(i + 1) * rl]
        for c in range(channels):
            sigma = F(g[c]) / F(255.0)
            mean = F(m[c]) / F(255.0)
            r[c] = mean * pixels
            r[channels + c] = (F(2.0) * sigma * sigma + mean * mean) * pixels
    return out


@dataclass
class ColourBlock:
    luma: float
    cb: float
    cr: float
    grain: float
    mean: float = 0.0
    second_mean: float | None = None

    @staticmethod
    def coloured(luma, saturation, sector, grain):
        angle = F(-math.pi) + (F(sector) + F(0.5)) * (F(2 * math.pi) / F(HUES))
        return ColourBlock(luma, float(F(saturation) * F(math.cos(angle))), float(F(saturation) * F(math.sin(angle))),
                           grain)


class CellRun:
    """noise/tests/colour.rs:131-212: frames of blocks pooled as stream frames 0 onwards."""

    def __init__(self, oracle, w, h, channels, luma):
        self.o, self.w, self.h, self.channels, self.luma = oracle, w, h, channels, luma
        self.capacity = 18
        self.words = oracle.colour_records(channels, luma) * WORDS
        self.ring = np.zeros((self.capacity, self.words), np.int32)
        self.pooled = 0
        self.frames = []  # (records, means) per pooled frame

    def inputs(self, blocks):
        grains = [[b.grain] * 2 for b in blocks]
        means = [[b.mean, b.second_mean if b.second_mean is not None else b.mean] for b in blocks]
        records = block_records(grains, means, self.channels, self.w, self.h)
        colour = np.array([[b.luma, b.cb, b.cr] for b in blocks], np.float32)
        return records, colour

    def pool(self, blocks):
        records, colour = self.inputs(blocks)
        self.frames.append((records, colour))
        self.ring[self.pooled % self.capacity] = self.o.colour_accumulate(records, colour, self.w, self.h,
                                                                          self.channels, self.luma, 255.0)
        self.pooled += 1

    def scene(self):
        return self.o.colour_window(self.ring, self.capacity, 0, self.pooled - 1)


def record(scene, index):
    return scene[index * WORDS:(index + 1) * WORDS]


def total_count(scene, indices):
    return sum(float(record(scene, i)[0]) for i in indices)


def reference_cell(luma, cb, cr):
    """The cell of a colour by exact geometry (noise/tests/colour.rs:84-102)."""
    brightness = min(max(math.floor(luma / 16.0), 0), 15)
    saturation = math.hypot(cb, cr)
    level = sum(1 for e in SAT_EDGES if saturation >= e)
    if level == 0:
        return brightness * PER_BRIGHTNESS
    turn = (math.atan2(cr, cb) + math.pi) / (2 * math.pi)
    sector = max(math.floor(turn * HUES), 0) % HUES
    return brightness * PER_BRIGHTNESS + 1 + (level - 1) * HUES + sector


# ---- the fit scenes (noise/tests/colour_fit.rs:60-900) ------------------------------------------

class SceneRng:
    """A seeded stream of values in [0, 1) from SplitMix64."""

    def __init__(self, seed):
        self.state = seed & 0xFFFFFFFFFFFFFFFF

    def unit(self):
        m = 0xFFFFFFFFFFFFFFFF
        self.state = (self.state + 0x9E3779B97F4A7C15) & m
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
        z ^= z >> 31
        return float(F(z >> 40) / F(1 << 24))

    def log_noise(self):
        return ((self.unit() + self.unit() + self.unit()) - 1.5) * 0.4

    def jitter(self):
        return 2.0 * self.unit() - 1.0


@dataclass
class FitBlock:
    luma: float
    cb: float
    cr: float
    grain: tuple

    @staticmethod
    def in_cell(brightness, level, sector, jitter, grain):
        luma = (brightness + 0.5) * 16.0 + 4.0 * jitter
        saturation = 2.0 + jitter if level == 0 else SAT_CENTRES[level] + jitter
        angle = -math.pi + (sector + 0.5 + 0.2 * jitter) * (2 * math.pi / HUES)
        return FitBlock(luma, saturation * math.cos(angle), saturation * math.sin(angle), tuple(grain))


def random_scene(count, seed, grain_of):
    rng = SceneRng(seed)
    out = []
    for _ in range(count):
        luma = 22.0 + 216.0 * rng.unit()
        su = rng.unit()
        saturation = 60.0 * su * su
        angle = 2 * math.pi * rng.unit()
        cb, cr = saturation * math.cos(angle), saturation * math.sin(angle)
        g = grain_of(luma, cb, cr)
        residual = 6.0 if rng.unit() < 0.03 else 1.0
        spread = math.exp(rng.log_noise()) * residual
        second = math.exp(rng.log_noise()) * residual
        out.append(FitBlock(luma, cb, cr, (g[0] * spread, g[1] * second)))
    return out


def planted(cb, cr):
    saturation = math.hypot(cb, cr)
    turn = (math.atan2(cr, cb) + math.pi) / (2 * math.pi)
    return saturation >= SAT_EDGES[2] and int(math.floor(turn * 4.0)) % 4 == 0


def cell_scene(per_cell, seed, bins, factor_of):
    rng = SceneRng(seed)
    blocks = []
    for brightness in bins:
        for ring in range(1 + HUES):
            level, sector = (0, 0) if ring == 0 else (3, ring - 1)
            for _ in range(per_cell):
                probe = FitBlock.in_cell(brightness, level, sector, rng.jitter(), (1.0, 1.0))
                factor = factor_of(brightness, probe.cb, probe.cr)
                spread, second = math.exp(rng.log_noise()), math.exp(rng.log_noise())
                blocks.append(FitBlock(probe.luma, probe.cb, probe.cr, (2.0 * factor * spread, 1.2 * factor * second)))
        for _ in range(per_cell // 20):
            blocks.append(FitBlock.in_cell(brightness, 0, 0, rng.jitter(), (16.0, 9.6)))
    return blocks


def planted_factor(_brightness, cb, cr):
    return 3.0 if planted(cb, cr) else 1.0


FLAT_CURVE = [1.0] * 16
RISING_CURVE = [0.7 + 0.7 * b / 15 for b in range(16)]


def fit_frames(blocks, planes):
    """Each pooled frame's (records, means) for a 1024x1024 frame of 64x64 blocks, padded."""
    h = (FRAME_BLOCKS // 64) * 16
    frames = []
    for start in range(0, len(blocks), FRAME_BLOCKS):
        chunk = blocks[start:start + FRAME_BLOCKS]
        chunk = chunk + [FitBlock(0.0, 0.0, 0.0, (0.0, 0.0))] * (FRAME_BLOCKS - len(chunk))
        records = block_records([b.grain for b in chunk], [(0.0, 0.0)] * len(chunk), planes, FRAME_WIDTH, h)
        means = np.array([[b.luma, b.cb, b.cr] for b in chunk], np.float32)
        frames.append((records, means))
    assert len(frames) <= 17
    return frames, FRAME_WIDTH, h


def fit_window(oracle, blocks, planes, luma):
    frames, w, h = fit_frames(blocks, planes)
    cap = 18
    words = oracle.colour_records(planes, luma) * WORDS
    ring = np.zeros((cap, words), np.int32)
    for f, (records, means) in enumerate(frames):
        ring[f % cap] = oracle.colour_accumulate(records, means, w, h, planes, luma, 255.0)
    return oracle.colour_window(ring, cap, 0, len(frames) - 1), frames, ring


def populated_cells(window, plane):
    return [c for c in range(CELLS) if window[(plane * CELLS + c) * WORDS] >= 40.0]


# ---- the float64 host model -------------------------------------------------------------------

def host_centre(cell):
    brightness, ring = divmod(cell, PER_BRIGHTNESS)
    luma = (brightness + 0.5) * 16.0
    if ring == 0:
        return luma, 0.0, 0.0
    level, sector = (ring - 1) // HUES + 1, (ring - 1) % HUES
    angle = -math.pi + (sector + 0.5) * 2 * math.pi / HUES
    return luma, SAT_CENTRES[level] * math.cos(angle), SAT_CENTRES[level] * math.sin(angle)


def host_index(brightness, level, sector):
    return brightness * PER_BRIGHTNESS + (0 if level == 0 else 1 + (level - 1) * HUES + sector)


def host_lookup(table, luma, cb, cr):
    bpos = min(max(luma / 16.0 - 0.5, 0.0), 15.0)
    blow = min(int(math.floor(bpos)), 14)
    bfr = bpos - blow
    s = math.hypot(cb, cr)
    if s <= SAT_CENTRES[0]:
        lpos = 0.0
    elif s >= SAT_CENTRES[-1]:
        lpos = 5.0
    else:
        seg = next(i for i in range(5) if s < SAT_CENTRES[i + 1])
        lpos = seg + (s - SAT_CENTRES[seg]) / (SAT_CENTRES[seg + 1] - SAT_CENTRES[seg])
    llow = min(int(math.floor(lpos)), 4)
    lfr = lpos - llow
    hpos = (math.atan2(cr, cb) + math.pi) / (2 * math.pi) * HUES - 0.5
    hfloor = math.floor(hpos)
    hfr = hpos - hfloor
    slow = int(hfloor) % HUES
    value = 0.0
    for corner in range(8):
        bs, ls, ss = corner // 4, (corner // 2) % 2, corner % 2
        w = (bfr if bs else 1 - bfr) * (lfr if ls else 1 - lfr) * (hfr if ss else 1 - hfr)
        value += w * table[host_index(blow + bs, llow + ls, (slow + ss) % HUES)]
    return value


def host_levels(window, ceilings, cells, mean_level):
    out = []
    for cell in range(cells):
        r = window[cell * WORDS:(cell + 1) * WORDS].astype(np.float64)
        hist = r[5:5 + HIST_BINS]
        ceiling = ceilings[cell]
        dropped = dropped_log = 0.0
        shares = []
        for b in range(HIST_BINS):
            low = LOG_MIN + b * LOG_STEP
            high = low + LOG_STEP
            above = min(max((high - ceiling) / LOG_STEP, 0.0), 1.0)
            dropped += hist[b] * above
            dropped_log += hist[b] * above * (max(low, ceiling) + high) * 0.5
            shares.append((low, hist[b] * (1 - above), 1 - above))
        kept = max(r[0] - dropped, 0.0)
        if kept <= 0:
            level = 0.0
        elif mean_level:
            level = (r[1] - dropped_log) / max(kept, 1.0)
        else:
            target, below, level = kept * 0.5, 0.0, 0.0
            for low, kc, share in shares:
                if kc > 0 and below + kc >= target:
                    level = low + (target - below) / kc * share * LOG_STEP
                    break
                below += kc
        out.append((kept, level))
    return out


def _tents(luma):
    pos = min(max(luma * 16 / 255.0, 0.0), 16.0)
    low = min(int(math.floor(pos)), 15)
    return low, pos - low


def host_model(window, levels, plane, luma):
    means, weights, lv, blocks = [], [], [], 0.0
    for cell in range(CELLS):
        r = window[(plane * CELLS + cell) * WORDS:].astype(np.float64)
        n = max(r[0], 1.0)
        means.append((r[2] / n, r[3] / n, r[4] / n))
        kept, level = levels[plane * CELLS + cell]
        weights.append(kept if kept >= 8.0 else 0.0)
        lv.append(level)
        blocks += kept
    pop = [c for c in range(CELLS) if weights[c] > 0]
    if not pop:
        return np.zeros(CELLS), False, blocks
    lo, hi = min(means[c][0] for c in pop), max(means[c][0] for c in pop)

    def curve(knots, l):
        low, fr = _tents(min(max(l, lo), hi))
        return knots[low] * (1 - fr) + knots[low + 1] * fr

    a = np.zeros((KNOTS, KNOTS))
    rhs = np.zeros(KNOTS)
    for c in pop:
        low, fr = _tents(means[c][0])
        for row, rw in ((low, 1 - fr), (low + 1, fr)):
            rhs[row] += weights[c] * lv[c] * rw
            for col, cw in ((low, 1 - fr), (low + 1, fr)):
                a[row, col] += weights[c] * rw * cw
    mean_root = sum(math.sqrt(weights[c]) for c in pop) / len(pop)
    pen = 4.0 * mean_root
    for row in range(KNOTS - 2):
        co = ((row, 1.0), (row + 1, -2.0), (row + 2, 1.0))
        for i, wi in co:
            for j, wj in co:
                a[i, j] += pen * wi * wj
    a[np.diag_indices(KNOTS)] *= 1.0 + 1.0e-5
    knots = np.linalg.solve(a, rhs)
    resid = [lv[c] - curve(knots, means[c][0]) for c in range(CELLS)]
    prior = 0.002 * blocks

    def base(q):
        num = den = 0.0
        for c in pop:
            d = ((q[0] - means[c][0]) / 32) ** 2 + ((q[1] - means[c][1]) / 12) ** 2 + ((q[2] - means[c][2]) / 12) ** 2
            k = math.exp(-0.5 * d)
            num += k * weights[c] * resid[c]
            den += k * weights[c]
        lift = num / (den + prior) if den + prior > 0 else 0.0
        return curve(knots, q[0]) + lift

    dz = 0.1 if luma else 0.0
    moves = [0.0] * CELLS
    for c in pop:
        gap = lv[c] - base(means[c])
        moves[c] = weights[c] / (weights[c] + 15.0) * math.copysign(max(abs(gap) - dz, 0.0), gap)
    has = lambda c: weights[c] > 0  # noqa: E731
    table = np.zeros(CELLS)
    for c in range(CELLS):
        if has(c):
            filled = moves[c]
        else:
            b, ring = divmod(c, PER_BRIGHTNESS)
            nb = []
            if b > 0 and has(c - PER_BRIGHTNESS):
                nb.append(moves[c - PER_BRIGHTNESS])
            if b + 1 < 16 and has(c + PER_BRIGHTNESS):
                nb.append(moves[c + PER_BRIGHTNESS])
            row = b * PER_BRIGHTNESS
            if ring == 0:
                rm = [moves[row + 1 + s] for s in range(HUES) if has(row + 1 + s)]
                if rm:
                    nb.append(sum(rm) / len(rm))
            else:
                level, sector = (ring - 1) // HUES, (ring - 1) % HUES
                cand = [row if level == 0 else c - HUES]
                if level + 2 < 6:
                    cand.append(c + HUES)
                start = row + 1 + level * HUES
                cand += [start + (sector + 1) % HUES, start + (sector + HUES - 1) % HUES]
                nb += [moves[n] for n in cand if has(n)]
            filled = sum(nb) / len(nb) if nb else 0.0
        table[c] = base(host_centre(c)) + filled
    return table, True, blocks


def host_median(histograms):
    total = sum(h.sum() for h, _ in histograms)
    if total <= 0:
        return None

    def share(p):
        s = 0.0
        for h, shift in histograms:
            lows = LOG_MIN + np.arange(HIST_BINS) * LOG_STEP + shift
            s += float((h * np.clip((p - lows) / LOG_STEP, 0, 1)).sum())
        return s

    lo, hi = -100.0, 100.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if share(mid) < total * 0.5:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def host_fit(window, planes, luma, ratios, curve_valid):
    """The float64 (tables, gains) of every plane."""
    cells = planes * CELLS
    first = host_levels(window, [float(np.finfo(np.float32).max)] * cells, cells, luma)
    ceilings = []
    for p in range(planes):
        table, _, _ = host_model(window, first, p, luma)
        for c in range(CELLS):
            r = window[(p * CELLS + c) * WORDS:].astype(np.float64)
            n = max(r[0], 1.0)
            ceilings.append(host_lookup(table, r[2] / n, r[3] / n, r[4] / n) + math.log(2) if r[0] > 0
                            else float(np.finfo(np.float32).max))
    second = host_levels(window, ceilings, cells, luma)
    tables, gains = [], []
    for p in range(planes):
        table, populated, blocks = host_model(window, second, p, luma)
        shifts = [-math.log(r) if (luma and curve_valid and r > 0) else 0.0 for r in ratios]
        if luma:
            hists = [(window[(planes * CELLS + b) * WORDS + 5:(planes * CELLS + b) * WORDS + 5 + HIST_BINS]
                      .astype(np.float64), shifts[b]) for b in range(16)]
        else:
            merged = np.zeros(HIST_BINS)
            for c in range(CELLS):
                merged += window[(p * CELLS + c) * WORDS + 5:(p * CELLS + c) * WORDS + 5 + HIST_BINS]
            hists = [(merged, 0.0)]
        norm = host_median(hists)
        ramp = blocks / (blocks + 256.0)
        if luma:
            neutral = sum(h.sum() for h, _ in hists)
            ramp *= neutral / (neutral + 256.0)
        for c in range(CELLS):
            if populated and norm is not None:
                lg = table[c] - norm
                lg = lg + shifts[c // PER_BRIGHTNESS] if luma else min(max(lg, math.log(0.4)), math.log(3.0))
            else:
                lg = 0.0
            gains.append(ramp * lg)
        tables.extend(table)
    return np.array(tables), np.array(gains)
