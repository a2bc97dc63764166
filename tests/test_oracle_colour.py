"""The oracle's colour grain gains on the CPU.

Replays the reference's own tests of the cell sums (av-denoise-core/src/noise/tests/colour.rs) and
of the fit (noise/tests/colour_fit.rs) on the restatement: which cell and record every block lands
in, the gates and level edges, the colour-relative outlier rule, the block means at every bit depth,
and the fit's gains on planted, neutral, thin and one-bin scenes. The fit is also held within 1e-4
of a float64 host model, as the reference holds its kernels.
"""

import math

import numpy as np
import pytest

import colour_cases as cc

CELLS, WORDS = cc.CELLS, cc.WORDS


@pytest.fixture(scope="module")
def o():
    import oracle

    return oracle


def test_mirror_functions_stay_within_two_ulp(o):
    rng = np.random.default_rng(3)
    xs = np.exp(rng.uniform(-8, 8, 4000)).astype(np.float32)
    for x in xs:
        want = np.float32(math.log(float(x)))
        assert abs(int(np.float32(o.log_mirror(float(x))).view(np.int32)) - int(want.view(np.int32))) <= 2
    for y, x in rng.normal(0, 60, (4000, 2)).astype(np.float32):
        want = np.float32(math.atan2(float(y), float(x)))
        assert abs(int(np.float32(o.atan2_mirror(float(y), float(x))).view(np.int32)) - int(want.view(np.int32))) <= 2


def test_blocks_bin_into_the_expected_cells(o):
    B = cc.ColourBlock
    blocks = [B(100.0, 0.0, 0.0, 2.0), B.coloured(100.0, 9.0, 0, 2.0), B.coloured(100.0, 9.0, 11, 1.5),
              B.coloured(130.0, 16.0, 3, 3.0), B.coloured(130.0, 25.0, 6, 2.5), B.coloured(60.0, 37.0, 8, 1.2),
              B.coloured(60.0, 80.0, 5, 4.0), B(200.0, 3.0, -4.0, 0.8), B.coloured(200.0, 13.0, 9, 1.0),
              B.coloured(25.0, 50.0, 2, 2.0), B.coloured(235.0, 7.0, 7, 2.2), B.coloured(150.0, 44.5, 10, 0.6)]
    run = cc.CellRun(o, 64, 48, 2, False)
    run.pool(blocks)
    scene = run.scene()
    assert cc.reference_cell(100.0, 0.0, 0.0) == 6 * 61
    assert cc.reference_cell(blocks[1].luma, blocks[1].cb, blocks[1].cr) == 6 * 61 + 1
    assert cc.reference_cell(blocks[2].luma, blocks[2].cb, blocks[2].cr) == 6 * 61 + 12
    for channel in range(2):
        base = channel * CELLS
        assert cc.total_count(scene, range(base, base + CELLS)) == len(blocks)
        for b in blocks:
            cell = cc.reference_cell(b.luma, b.cb, b.cr)
            assert o.colour_cell(b.luma, b.cb, b.cr) == cell
            words = cc.record(scene, base + cell)
            log_grain = math.log(b.grain)
            assert words[0] == 1.0
            assert abs(words[1] - log_grain) <= 1e-3
            assert abs(words[2] - b.luma) <= 0.04 and abs(words[3] - b.cb) <= 0.04 and abs(words[4] - b.cr) <= 0.04
            assert words[5 + int(math.floor((log_grain + 3.5) / 0.125))] == 1.0
        # Each channel also pools every block into its plane record.
        assert cc.record(scene, 2 * CELLS + channel)[0] == len(blocks)


def level_count(scene, channel, brightness, level):
    first = channel * CELLS + brightness * 61
    cells = range(first, first + 1) if level == 0 else range(first + 1 + (level - 1) * 12, first + 13 + (level - 1) * 12)
    return cc.total_count(scene, cells)


def test_blocks_at_the_gate_and_level_edges(o):
    B = cc.ColourBlock
    moving = B(100.0, 0.0, 0.0, 2.0, mean=3.0)
    blocks = [B(20.0, 0.0, 0.0, 2.0), B(240.0, 0.0, 0.0, 2.0), B(20.01, 0.0, 0.0, 2.0), B(239.9, 0.0, 0.0, 2.0),
              B(100.0, 6.0, 0.0, 2.0), B(100.0, 5.99, 0.0, 2.0), B(100.0, 0.0, 44.0, 2.0), B(100.0, 0.0, 43.99, 2.0),
              B(100.0, 7.5, 0.0, 2.0), B(100.0, 8.0, 0.0, 2.0), B(100.0, 0.0, 0.0, 0.04), B(100.0, 0.0, 0.0, 0.06),
              moving, moving, moving, moving]
    run = cc.CellRun(o, 64, 64, 1, True)
    run.pool(blocks)
    luma = run.scene()
    assert cc.total_count(luma, range(CELLS)) == 9.0
    assert level_count(luma, 0, 1, 0) == 1.0 and level_count(luma, 0, 14, 0) == 1.0
    assert level_count(luma, 0, 6, 0) == 2.0
    assert level_count(luma, 0, 6, 1) == 3.0
    assert level_count(luma, 0, 6, 4) == 1.0 and level_count(luma, 0, 6, 5) == 1.0
    calibration = lambda b: cc.record(luma, CELLS + b)[0]  # noqa: E731
    assert calibration(6) == 4.0 and calibration(1) == 1.0 and calibration(14) == 1.0
    chroma_run = cc.CellRun(o, 64, 64, 2, False)
    chroma_run.pool(blocks)
    chroma = chroma_run.scene()
    for channel in range(2):
        assert level_count(chroma, channel, 6, 0) == 3.0


def test_each_chroma_channel_gates_on_its_own_residual(o):
    B = cc.ColourBlock
    moving = B(100.0, 0.0, 0.0, 2.0, mean=3.0)
    cb_static = B.coloured(100.0, 25.0, 3, 2.0)
    cb_static.second_mean = 3.0
    cr_static = B.coloured(180.0, 37.0, 9, 1.5)
    cr_static.mean, cr_static.second_mean = 3.0, 0.0
    run = cc.CellRun(o, 64, 48, 2, False)
    run.pool([cb_static, cr_static] + [moving] * 10)
    scene = run.scene()
    assert cc.total_count(scene, range(CELLS)) == 1.0
    assert cc.total_count(scene, range(CELLS, 2 * CELLS)) == 1.0
    assert cc.record(scene, cc.reference_cell(cb_static.luma, cb_static.cb, cb_static.cr))[0] == 1.0
    assert cc.record(scene, CELLS + cc.reference_cell(cr_static.luma, cr_static.cb, cr_static.cr))[0] == 1.0


@pytest.mark.parametrize("mean_level", [True, False])
def test_heavy_colour_grain_is_kept_and_motion_residual_dropped(o, mean_level):
    B = cc.ColourBlock
    neutral, residual = B(120.0, 0.0, 0.0, 1.0), B(120.0, 0.0, 0.0, 5.0)
    moving = B(120.0, 0.0, 0.0, 1.0, mean=3.0)
    red = B.coloured(120.0, 40.0, 7, 4.0)
    run = cc.CellRun(o, 128, 64, 1, mean_level)
    run.pool([neutral] * 16 + [residual] * 4 + [red] * 10 + [moving] * 2)
    scene = run.scene()
    first = o.colour_levels(scene, np.full(CELLS, np.finfo(np.float32).max, np.float32), CELLS, mean_level)
    second = o.colour_levels(scene, (first[:, 1] + np.float32(math.log(2))).astype(np.float32), CELLS, mean_level)
    nc, rc = cc.reference_cell(120.0, 0.0, 0.0), cc.reference_cell(red.luma, red.cb, red.cr)
    assert first[nc, 0] == 20.0
    assert abs(second[nc, 0] - 16.0) <= 1e-3 and abs(second[nc, 1]) <= 0.125
    assert abs(second[rc, 0] - 10.0) <= 1e-3 and abs(second[rc, 1] - math.log(4.0)) <= 0.125


def test_extreme_chroma_values_index_inside_the_table(o):
    blocks = [cc.ColourBlock(luma, cb, cr, 2.0) for luma in (20.5, 239.5) for cb in (-128.0, 127.0, -300.0, 300.0)
              for cr in (-128.0, 127.0)]
    run = cc.CellRun(o, 64, 64, 1, True)
    run.pool(blocks)
    scene = run.scene()
    assert cc.total_count(scene, range(CELLS)) == len(blocks)
    for b in blocks:
        cell = o.colour_cell(b.luma, b.cb, b.cr)
        assert cell < CELLS and cc.record(scene, cell)[0] >= 1.0
    assert cc.total_count(scene, range(CELLS, CELLS + 16)) == 0.0


def test_a_frame_read_again_replaces_its_cells(o):
    """noise/tests/colour.rs:794-820: the window holds each frame's latest sums."""
    run = cc.CellRun(o, 64, 48, 1, True)
    a = [cc.ColourBlock(100.0, 0.0, 0.0, 2.0)] * 12
    b = [cc.ColourBlock(180.0, 0.0, 0.0, 3.0)] * 12
    run.pool(a)
    records, colour = run.inputs(b)
    run.ring[0] = o.colour_accumulate(records, colour, 64, 48, 1, True, 255.0)  # frame 0 read again
    scene = run.scene()
    assert cc.record(scene, cc.reference_cell(180.0, 0.0, 0.0))[0] == 12.0
    assert cc.record(scene, cc.reference_cell(100.0, 0.0, 0.0))[0] == 0.0


def _pack(codes, kind, depth=8):
    """Word-packed plane of integer codes (u8: 4 per word, u16: 2 per word) or f32 samples."""
    codes = np.asarray(codes).reshape(-1)
    if kind == "f32":
        return np.ascontiguousarray(codes.astype(np.float32)).view(np.uint32)
    per = 4 if kind == "u8" else 2
    dt = np.uint8 if kind == "u8" else np.uint16
    pad = (-len(codes)) % per
    return np.concatenate([codes.astype(dt), np.zeros(pad, dt)]).view(np.uint32)


@pytest.mark.parametrize("w,h,sx,sy", [(64, 48, 1, 1), (70, 37, 1, 0), (50, 34, 0, 0)])
def test_block_means_at_every_bit_depth_are_the_same(o, w, h, sx, sy):
    """noise/tests/colour.rs:571-658: the same content at 8, 10 and 16 bits and in float lands on
    the same 8-bit-scale means (to float rounding), and each block averages its own pixels."""
    rng = np.random.default_rng(w)
    cw, ch = -(-w // (1 << sx)), -(-h // (1 << sy))
    y8 = rng.integers(0, 256, (h, w))
    u8 = rng.integers(0, 256, (ch, cw))
    v8 = rng.integers(0, 256, (ch, cw))
    ref_l, ref_c = o.colour_means(_pack(y8, "u8"), _pack(u8, "u8"), _pack(v8, "u8"), w, h, sx, sy, 4, False, 1.0, 0.0)
    for depth in (10, 16):
        up = 1 << (depth - 8)
        lm, cm = o.colour_means(_pack(y8 * up, "u16"), _pack(u8 * up, "u16"), _pack(v8 * up, "u16"), w, h, sx, sy,
                                2, False, 1.0 / up, 0.0)
        assert np.allclose(lm, ref_l, atol=1e-3) and np.allclose(cm, ref_c, atol=1e-3)
    lm, cm = o.colour_means(_pack(y8 / 255.0, "f32"), _pack(u8 / 255.0 - 0.5, "f32"), _pack(v8 / 255.0 - 0.5, "f32"),
                            w, h, sx, sy, 1, True, 255.0, 0.5)
    assert np.allclose(lm, ref_l, atol=2e-3) and np.allclose(cm, ref_c, atol=2e-3)
    # A luma-grid block averages its own luma and the chroma pixels its area covers (rounded out).
    bx = -(-w // 16)
    i = min(bx + 1, len(ref_l) - 1)
    x0, y0 = (i % bx) * 16, (i // bx) * 16
    x1, y1 = min(x0 + 16, w), min(y0 + 16, h)
    assert abs(ref_l[i, 0] - y8[y0:y1, x0:x1].mean()) < 1e-3
    c0x, c0y = x0 >> sx, y0 >> sy
    c1x, c1y = (x1 + (1 << sx) - 1) >> sx, (y1 + (1 << sy) - 1) >> sy
    assert abs(ref_l[i, 1] - (u8[c0y:c1y, c0x:c1x].mean() - 128)) < 1e-3


# ---- the fit ------------------------------------------------------------------------------------

@pytest.fixture(scope="module")
def luma_scene():
    def grain(luma, cb, cr):
        g = (1.2 + luma / 200.0) * (1.0 + max(cr - cb, 0.0) / 40.0)
        return (g, g)

    return cc.random_scene(60_000, 11, grain)


@pytest.fixture(scope="module")
def chroma_scene():
    return cc.random_scene(60_000, 23, lambda luma, cb, cr: (0.8 + 0.6 * (max(cb, 0.0) / 30.0) + luma / 400.0,
                                                              0.6 + 0.9 * (abs(cr) / 40.0)))


@pytest.mark.parametrize("planes,luma,which,ratios,curve_valid", [
    (1, True, "luma", cc.RISING_CURVE, True),
    (1, True, "luma", cc.RISING_CURVE, False),
    (2, False, "chroma", cc.FLAT_CURVE, False),
])
def test_fit_matches_the_host_model(o, luma_scene, chroma_scene, planes, luma, which, ratios, curve_valid):
    scene = luma_scene if which == "luma" else chroma_scene
    window, _, _ = cc.fit_window(o, scene, planes, luma)
    table, gains, _ = o.colour_fit(window, planes, luma, ratios, curve_valid)
    host_table, host_gains = cc.host_fit(window, planes, luma, ratios, curve_valid)
    assert np.abs(table - host_table).max() <= 1e-4
    assert np.abs(gains - host_gains).max() <= 1e-4
    rng = np.random.default_rng(planes)
    queries = np.stack([255 * rng.random(512), 140 * rng.random(512) - 70, 140 * rng.random(512) - 70], 1)
    for p in range(planes):
        _, looked = o.colour_lookup(gains[p * CELLS:(p + 1) * CELLS], queries.astype(np.float32))
        host = np.exp([cc.host_lookup(host_gains[p * CELLS:(p + 1) * CELLS], *q) for q in queries.astype(np.float32)])
        assert np.all(np.abs(looked - host) <= 1e-4 * np.maximum(host, 1.0))


def test_the_fit_recovers_a_planted_colour_field(o):
    scene = cc.cell_scene(220, 5, range(2, 14), cc.planted_factor)
    window, _, _ = cc.fit_window(o, scene, 1, True)
    _, gains, _ = o.colour_fit(window, 1, True, cc.FLAT_CURVE, True)
    cells = cc.populated_cells(window, 0)
    assert len(cells) >= 100
    blocks = sum(float(window[c * WORDS]) for c in range(CELLS))
    neutral = sum(float(window[(CELLS + b) * WORDS]) for b in range(16))
    ramp = blocks / (blocks + 256.0) * neutral / (neutral + 256.0)
    for c in cells:
        centre = cc.host_centre(c)
        planted = 3.0 if cc.planted(centre[1], centre[2]) else 1.0
        assert abs(float(gains[c]) - ramp * math.log(planted)) <= 0.07 + 0.1, c


def test_a_field_without_colour_effect_gives_gains_near_one(o):
    scene = cc.cell_scene(300, 37, range(2, 14), lambda *_: 1.0)
    for planes, luma in ((1, True), (2, False)):
        window, _, _ = cc.fit_window(o, scene, planes, luma)
        _, gains, _ = o.colour_fit(window, planes, luma, cc.FLAT_CURVE, luma)
        for p in range(planes):
            cells = cc.populated_cells(window, p)
            assert len(cells) >= 100
            gaps = [abs(math.exp(float(gains[p * CELLS + c])) - 1.0) for c in cells]
            assert max(gaps) <= 0.1 and sum(gaps) / len(gaps) <= 0.055


def test_a_thin_scene_gives_gains_of_one(o):
    scene = cc.cell_scene(5, 9, range(2, 14), cc.planted_factor)
    for planes, luma in ((1, True), (2, False)):
        window, _, _ = cc.fit_window(o, scene, planes, luma)
        _, gains, _ = o.colour_fit(window, planes, luma, cc.FLAT_CURVE, luma)
        assert not gains.any()


def test_one_or_two_brightness_bins_keep_gains_near_one_elsewhere(o):
    scene = cc.cell_scene(300, 61, range(7, 9), lambda b, *_: 0.9 if b == 7 else 1.1)
    ratios = [0.9 if b < 8 else 1.1 for b in range(16)]
    window, _, _ = cc.fit_window(o, scene, 1, True)
    _, gains, _ = o.colour_fit(window, 1, True, ratios, True)
    for b in list(range(0, 5)) + list(range(11, 16)):
        assert np.all(np.abs(gains[b * 61:(b + 1) * 61]) <= 0.1)


def test_a_single_neutral_block_barely_moves_the_luma_gains(o):
    scene = [b for b in cc.cell_scene(220, 71, range(2, 14), cc.planted_factor) if math.hypot(b.cb, b.cr) >= 8.0]
    scene.append(cc.FitBlock.in_cell(8, 0, 0, 0.0, (2.0, 1.2)))
    window, _, _ = cc.fit_window(o, scene, 1, True)
    _, gains, _ = o.colour_fit(window, 1, True, cc.FLAT_CURVE, True)
    assert np.all(np.abs(gains) <= 0.01) and gains.any()


def test_chroma_gains_preserve_the_plane_average(o):
    scene = cc.random_scene(60_000, 53, lambda luma, cb, cr: (1.0 + 1.5 * (max(cb, 0.0) / 40.0) + luma / 300.0,
                                                              0.7 + 1.2 * (max(-cr, 0.0) / 40.0)))
    window, _, _ = cc.fit_window(o, scene, 2, False)
    _, gains, _ = o.colour_fit(window, 2, False)
    measured = [b for b in scene if 20.0 < b.luma < 240.0]
    queries = np.array([[b.luma, b.cb, b.cr] for b in measured], np.float32)
    for p in range(2):
        _, g = o.colour_lookup(gains[p * CELLS:(p + 1) * CELLS], queries)
        grains = np.array([b.grain[p] for b in measured])
        shift = math.log(np.sort(grains / g)[len(grains) // 2] / np.sort(grains)[len(grains) // 2])
        assert abs(shift) <= 0.05
    blue = (128.0, 40.0, 0.0)
    cb_on_blue = cc.host_lookup(gains[:CELLS].astype(np.float64), *blue)
    cr_on_blue = cc.host_lookup(gains[CELLS:].astype(np.float64), *blue)
    assert cb_on_blue - cr_on_blue >= 0.3
