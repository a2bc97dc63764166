"""The camera-model fit of the oracle against the behaviour the reference pins for it
(av-denoise-core/src/motion/global/tests/fit.rs and compose.rs): known similarities come back within
1e-3 (a, b) and 0.05 px (tx, ty), outlier groups, still bars and stale priors do not move the fit,
and implausible or unsupported fields fall back to identity with `valid` 0. Fields are built the way
those tests build them: every block's vector is the similarity applied to the block's centre
(origin + 8), rounded."""

import math

import numpy as np
import pytest

import oracle
from camera_cases import render

W, H, BLK, OVL = 960, 540, 16, 8
STEP = BLK - OVL
BX, BY = -(-W // STEP), -(-H // STEP)
BLOCKS = BX * BY


def similarity(degrees, zoom, sx, sy):
    """A roll and zoom about the frame centre followed by a shift: (a, b, tx, ty)."""
    r = math.radians(degrees)
    a, b = zoom * math.cos(r), zoom * math.sin(r)
    cx, cy = W / 2, H / 2
    return a, b, cx - (a * cx - b * cy) + sx, cy - (b * cx + a * cy) + sy


def inverse(m):
    a, b, tx, ty = m
    n = a * a + b * b
    ia, ib = a / n, -b / n
    return ia, ib, -(ia * tx - ib * ty), -(ib * tx + ia * ty)


def camera_field(m):
    a, b, tx, ty = m
    col = np.arange(BLOCKS) % BX
    row = np.arange(BLOCKS) // BX
    x = col * STEP + BLK / 2
    y = row * STEP + BLK / 2
    mx = a * x - b * y + tx
    my = b * x + a * y + ty
    # Rust's f64::round rounds halves away from zero.
    rnd = lambda v: np.sign(v) * np.floor(np.abs(v) + 0.5)
    return np.stack([rnd(mx - x), rnd(my - y)], 1).astype(np.int32)


def random_field(seed):
    rng = np.random.default_rng(seed)
    return rng.integers(-12, 13, (BLOCKS, 2)).astype(np.int32)


def fit(field, *, sad=None, has_contrast=False, older_to_newer=True, prior=None):
    ring = np.zeros(2 * oracle.MODEL_WORDS, np.float32)
    if prior is not None:
        ring[:4] = np.asarray(prior, np.float32)
        ring[4] = 1.0
    models, _ = oracle.model_fit(field, W, H, BLK, OVL, sad=sad, has_contrast=has_contrast,
                                 older_to_newer=older_to_newer, models=ring, slot=1,
                                 prior=0 if prior is not None else None)
    return models[5:10]


def assert_matches(words, m):
    assert words[4] == 1.0, f"the fit should be accepted, got {words}"
    a, b, tx, ty = m
    assert abs(words[0] - a) < 1e-3 and abs(words[1] - b) < 1e-3, (words, m)
    assert abs(words[2] - tx) < 0.05 and abs(words[3] - ty) < 0.05, (words, m)


def assert_identity(words):
    assert np.array_equal(words, np.array([1, 0, 0, 0, 0], np.float32)), words


def rows_cols():
    return np.arange(BLOCKS) // BX, np.arange(BLOCKS) % BX


def with_group(camera):
    f = camera_field(camera)
    row, col = rows_cols()
    f[(col < 60) & (row < 41)] = (-12, 7)
    return f


def test_recovers_a_known_roll_zoom_and_shift():
    cam = similarity(2.5, 1.01, 6.0, -4.0)
    assert_matches(fit(camera_field(cam)), cam)


def test_fits_the_newer_to_older_direction_as_the_same_model():
    cam = similarity(-1.5, 0.99, -8.0, 3.0)
    assert_matches(fit(camera_field(inverse(cam)), older_to_newer=False), cam)


def test_rejects_an_independently_moving_block_group():
    cam = similarity(1.5, 1.0, 5.0, 2.0)
    assert_matches(fit(with_group(cam)), cam)


def test_a_uniform_zero_field_fits_identity():
    assert_identity(fit(np.zeros((BLOCKS, 2), np.int32)))


def test_a_nonsense_field_falls_back_to_identity():
    assert_identity(fit(random_field(5)))


def test_a_static_border_band_does_not_anchor_the_fit():
    cam = similarity(0.0, 1.0, 18.0, 3.0)
    f = camera_field(cam)
    row, _ = rows_cols()
    f[(row < 20) | (row >= BY - 20)] = 0
    assert_matches(fit(f), cam)


def test_roll_inside_15_degrees_is_accepted_and_beyond_it_is_not():
    cam = similarity(14.0, 1.0, 0.0, 0.0)
    assert_matches(fit(camera_field(cam)), cam)
    assert_identity(fit(camera_field(similarity(20.0, 1.0, 0.0, 0.0))))


@pytest.mark.parametrize("share", [0.2, 0.3, 0.4])
def test_a_moving_subject_on_a_still_camera_falls_back_to_identity(share):
    side = math.sqrt(share)
    gc, gr = round(BX * side), round(BY * side)
    c0, r0 = (BX - gc) // 2, (BY - gr) // 2
    row, col = rows_cols()
    f = np.zeros((BLOCKS, 2), np.int32)
    f[(col >= c0) & (col < c0 + gc) & (row >= r0) & (row < r0 + gr)] = (6, -2)
    assert fit(f)[4] == 0.0


@pytest.mark.parametrize("share", [0.2, 0.3, 0.4, 0.5])
def test_a_moving_layer_under_a_still_top_falls_back_to_identity(share):
    row, _ = rows_cols()
    f = np.zeros((BLOCKS, 2), np.int32)
    f[row >= BY - round(BY * share)] = (6, 0)
    assert fit(f)[4] == 0.0


def test_a_moving_strip_down_one_side_falls_back_to_identity():
    _, col = rows_cols()
    f = np.zeros((BLOCKS, 2), np.int32)
    f[col >= BX - round(BX * 0.3)] = (6, 0)
    assert_identity(fit(f))


def test_a_pillarboxed_pan_is_recovered():
    cam = similarity(0.0, 1.0, 5.0, 1.0)
    f = camera_field(cam)
    _, col = rows_cols()
    bar = round(BX * 0.12)
    f[(col < bar) | (col >= BX - bar)] = 0
    assert_matches(fit(f), cam)


def stats_sad(per_row):
    """The producer's SAD layout: winning SADs, window means, block means, one block count apart."""
    row, _ = rows_cols()
    values = np.zeros(3 * BLOCKS, np.float32)
    for b in range(BLOCKS):
        best, mean, luma = per_row(row[b])
        values[b], values[BLOCKS + b], values[2 * BLOCKS + b] = best, mean, luma
    return values


def layer_between_bands():
    band = math.floor(BY * 0.33)
    in_layer = lambda r: band <= r < BY - band
    row, _ = rows_cols()
    f = np.zeros((BLOCKS, 2), np.int32)
    f[(row >= band) & (row < BY - band)] = (6, 0)
    return f, in_layer


DETAILED = (1.0, 4.0, 0.4)


def test_still_dark_bands_with_detail_are_not_bars():
    f, in_layer = layer_between_bands()
    dark_detail = (1.0, 4.0, np.float32(18.0) / np.float32(255.0))
    assert fit(f)[4] == 1.0, "premise: without stats the bands pass as bars"
    sad = stats_sad(lambda r: DETAILED if in_layer(r) else dark_detail)
    assert_identity(fit(f, sad=sad, has_contrast=True))


def test_only_dark_flat_bands_are_bars():
    f, in_layer = layer_between_bands()
    grey = (1.0, 1.24, 0.5)
    black = (1.0, 1.24, np.float32(18.0) / np.float32(255.0))
    assert_identity(fit(f, sad=stats_sad(lambda r: DETAILED if in_layer(r) else grey), has_contrast=True))
    assert fit(f, sad=stats_sad(lambda r: DETAILED if in_layer(r) else black), has_contrast=True)[4] == 1.0


def test_zoom_and_corner_plausibility_bounds():
    assert_identity(fit(camera_field(similarity(0.0, 1.2, 0.0, 0.0))))
    assert_identity(fit(camera_field(similarity(0.0, 1.0, 410.0, 0.0))))


def test_weights_survive_high_grain():
    cam = similarity(1.0, 1.0, 9.0, -3.0)
    f = camera_field(cam)
    _, col = rows_cols()
    th = oracle.thsad(BLK, 1.0)
    rng = np.random.default_rng(33)
    grain = (th * (3.0 + 2.0 * rng.random(BLOCKS))).astype(np.float32)
    wrong = col >= 60
    f[wrong] = (10, -8)
    sad = np.where(wrong, 3.0 * grain, grain).astype(np.float32)
    assert_matches(fit(f, sad=sad), cam)


def test_a_stale_prior_does_not_bias_the_fit():
    cam = similarity(-1.0, 1.0, -3.0, 2.0)
    stale = similarity(4.0, 1.0, 30.0, 0.0)
    assert_matches(fit(with_group(cam), prior=stale), cam)


def test_a_valid_prior_holds_the_fit_on_the_camera():
    cam = similarity(1.0, 1.0, 9.0, -3.0)
    previous = similarity(1.1, 1.0, 8.5, -3.0)
    f = camera_field(cam)
    _, col = rows_cols()
    f[col >= 48] = (10, -8)
    without = fit(f)
    assert abs(without[1] - cam[1]) > 0.01, "the majority group should win without a prior"
    assert_matches(fit(f, prior=previous), cam)


def test_the_fit_is_bit_identical_across_runs():
    f = with_group(similarity(1.5, 1.0, 5.0, 2.0))
    assert np.array_equal(fit(f).view(np.uint32), fit(f).view(np.uint32))


# ---- composition (global/tests/compose.rs) --------------------------------------------------------

def model_words(m, valid=1.0):
    return np.array([m[0], m[1], m[2], m[3], valid], np.float32)


def apply(pred, x, y):
    return pred[0] * x + pred[1] * y + pred[4], pred[2] * x + pred[3] * y + pred[5]


def test_future_neighbours_chain_pairs_and_past_ones_invert_them():
    # Window frames 10..14 centred on 12: pairs 11, 12 (past, steps back from the centre), 13, 14.
    pairs = {f: similarity(0.5 * (f - 10), 1.0, 2.0 * (f - 10), -1.0) for f in range(11, 15)}
    frames = [10, 11, 12, 13, 14]
    index = {f: i for i, f in enumerate(frames)}
    ring = np.concatenate([model_words(pairs[f]) if f in pairs else model_words((1, 0, 0, 0), 0.0) for f in frames])
    gaps = oracle.compose_gaps(frames, 2, 4, lambda f: index[f])
    preds = oracle.compose_models(ring, gaps, 4, 4, 2).reshape(4, 6)
    x, y = 300.0, 200.0

    def fwd(m, p):
        return m[0] * p[0] - m[1] * p[1] + m[2], m[1] * p[0] + m[0] * p[1] + m[3]

    # Neighbour 14 (future, two steps): pair 13 then pair 14.
    ex = fwd(pairs[14], fwd(pairs[13], (x, y)))
    assert np.allclose(apply(preds[3], x, y), ex, atol=1e-3)
    # Neighbour 10 (past, two steps): the inverse of pair 11 then pair 12.
    ex = fwd(inverse(pairs[11]), fwd(inverse(pairs[12]), (x, y)))
    assert np.allclose(apply(preds[0], x, y), ex, atol=1e-3)


def test_a_duplicate_or_invalid_pair_composes_as_no_motion():
    frames = [5, 5, 6]  # an edge duplicate, then a real pair
    ring = np.concatenate([model_words(similarity(0, 1, 3, 0)), model_words(similarity(0, 1, 4, 0), 0.0)])
    gaps = oracle.compose_gaps(frames, 1, 2, lambda f: f - 5)
    assert gaps[0] == oracle.NO_PAIR
    preds = oracle.compose_models(ring, gaps, 2, 2, 1).reshape(2, 6)
    assert np.array_equal(preds[0], np.array([1, 0, 0, 1, 0, 0], np.float32))
    assert np.array_equal(preds[1], np.array([1, 0, 0, 1, 0, 0], np.float32))  # valid word 0


# ---- the producer over rendered frames (global/tests/producer.rs) -----------------------------------

PW, PH = 640, 360


def _shift(dx):
    return (1.0, 0.0, dx, 0.0)


@pytest.mark.parametrize("velocity", [30.0, 34.7])
def test_the_producer_recovers_a_fast_pan(velocity):
    # 30 px per frame lies past the mode's own reach (4 * 2 + 4); the deep first search finds it.
    pm = oracle.PairModels(PW, PH)
    tol = 0.1 if velocity == int(velocity) else 0.5
    for frame in range(4):
        pm.push(render(_shift(velocity * frame), PW, PH), frame)
        m = pm.model(frame)
        if frame == 0:
            assert np.array_equal(m, np.array([1, 0, 0, 0, 0], np.float32))
            continue
        assert m[4] == 1.0 and abs(m[0] - 1) < 1e-3 and abs(m[1]) < 1e-3, m
        assert abs(m[2] - velocity) < tol and abs(m[3]) < tol, m


def test_the_producer_starts_over_after_a_gap_and_fits_a_still_shot_as_no_motion():
    pm = oracle.PairModels(PW, PH)
    for frame in range(3):
        pm.push(render(_shift(0.0), PW, PH), frame)
    assert pm.model(2)[4] == 0.0, "a still shot fits no motion"
    pm.push(render(_shift(8.0), PW, PH), 7)  # does not follow frame 2: a new run
    assert np.array_equal(pm.model(7), np.array([1, 0, 0, 0, 0], np.float32))
    pm.push(render(_shift(16.0), PW, PH), 8)
    assert pm.model(8)[4] == 1.0 and abs(pm.model(8)[2] - 8.0) < 0.1
