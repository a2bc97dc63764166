"""The CPU oracle's block-matching motion search on the reference's own block-match cases
(av-denoise-core/src/motion/tests/block_match.rs:97-330) and the confidence formulas
(motion/confidence.rs:75-100); the ABI's host formulas agree with the oracle's."""

import numpy as np
import pytest

from motion_cases import shifted, textured


def pair_ring(centre: np.ndarray, neighbour: np.ndarray) -> np.ndarray:
    return np.stack([centre, neighbour]).astype(np.float32).reshape(-1)


def test_clean_shift_is_found_exactly(oracle):
    # block_match.rs:123-211: a (+2, +1) shift of rich content, 64x64, blksize 16 at step 16,
    # radius 4, one level: the middle block's vector is exactly (2, 1).
    c = textured(64, 64, 123)
    n = shifted(c, 2, 1)
    pyr = oracle.motion_pyramid(pair_ring(c, n), 1, 64, 64, 1)
    mv, _ = oracle.motion_search(pyr, 64, 64, 2, 0, [1], blksize=16, overlap=0, search_radius=4, levels=1)
    assert tuple(mv[0, 1 * 4 + 1]) == (2, 1)


def test_uniform_mismatch_sad_from_confidence(oracle):
    # block_match.rs:96-120: |delta| = 0.1 over a 16x16 block gives a SAD of 25.6, recovered from
    # the confidence within 1%.
    c = np.full((16, 16), 0.25, np.float32)
    n = np.full((16, 16), 0.35, np.float32)
    pyr = oracle.motion_pyramid(pair_ring(c, n), 1, 16, 16, 1)
    expected = 256 * 0.1
    th = 3.0 * expected
    _, conf = oracle.motion_search(pyr, 16, 16, 2, 0, [1], blksize=16, overlap=0, search_radius=0, levels=1,
                                   confidence=True, sad_floor=0.0, thsad=th)
    c0 = float(conf[0, 0])
    sad = th * np.sqrt((1.0 - c0) / (1.0 + c0))
    assert abs(sad - expected) < expected * 0.01


@pytest.mark.parametrize("levels", [1, 2])
def test_flat_region_tie_resolves_to_zero_motion(oracle, levels):
    # block_match.rs:275-330: every candidate ties on a flat block; the window's centre wins.
    flat = np.full((32, 32), 0.5, np.float32)
    pyr = oracle.motion_pyramid(pair_ring(flat, flat), 1, 32, 32, levels)
    mv, conf = oracle.motion_search(pyr, 32, 32, 2, 0, [1], levels=levels, confidence=True, thsad=5.12)
    assert not mv.any()
    assert np.all(conf == 1.0)


def test_global_shift_recovered_through_the_coarse_level(oracle):
    # A shift beyond the fine radius (6 > 4) is reached through the coarse seed (x2 at level 1).
    c = textured(96, 80, 7)
    n = shifted(c, 6, -5)
    pyr = oracle.motion_pyramid(pair_ring(c, n), 1, 96, 80, 2)
    mv, _ = oracle.motion_search(pyr, 96, 80, 2, 0, [1], levels=2)
    inner = mv[0].reshape(10, 12, 2)[2:-2, 2:-2]
    assert np.mean(np.all(inner == (6, -5), axis=-1)) > 0.9


def test_confidence_formulas_match_the_reference_tests(oracle, lib):
    # confidence.rs:75-100.
    sigma = 4.0 / 255.0
    want = 256 * 2.0 * sigma / np.sqrt(np.pi)
    assert abs(oracle.sad_noise_floor(16, sigma) - want) < 1e-6
    assert oracle.sad_noise_floor(16, 0.0) == 0.0
    assert abs(oracle.thsad(16, 2.0) - 2.0 * 256 * 0.02) < 1e-6
    assert oracle.thsad(16, 1.0) > 0.0
    for b, s in [(16, sigma), (8, 0.02), (32, 0.1), (16, 0.0)]:
        assert np.float32(lib.avd_sad_noise_floor(b, s)) == np.float32(oracle.sad_noise_floor(b, s))
    for b, t in [(16, 1.0), (8, 0.5), (32, 2.0)]:
        assert np.float32(lib.avd_thsad(b, t)) == np.float32(oracle.thsad(b, t))


def test_pyramid_layout_and_downscale(oracle, lib):
    # pyramid.rs:10-37: odd sizes repeat the edge; slots are padded to 8 floats.
    w, h = 13, 7
    frame = np.arange(w * h, dtype=np.float32).reshape(h, w) / 100.0
    pyr = oracle.motion_pyramid(frame.reshape(-1), 1, w, h, 2)
    assert pyr.size == lib.avd_motion_pyramid_floats(w, h, 1, 2) == 96 + 24
    l1 = pyr[96:96 + 18].reshape(3, 6)
    f = frame
    assert l1[0, 0] == np.float32((((f[0, 0] + f[0, 1]) + f[1, 0]) + f[1, 1]) * np.float32(0.25))


# ---- the truemotion stage (motion/truemotion), restated from its behavioural suite ------------------

def _ring(frames):
    return np.stack([f[..., None] for f in frames]).astype(np.float32)


def test_truemotion_keeps_a_static_scene_still(oracle):
    f = textured(96, 64, 3)
    ring = _ring([f, f, f])
    pyr = oracle.motion_pyramid(ring, 1, 96, 64, 2)
    mv, conf = oracle.motion_search(pyr, 96, 64, 3, 1, [0, 2], confidence=True, sad_floor=0.0,
                                    thsad=oracle.thsad(16, 1.0), field_lambda=1.0)
    assert not mv.any()
    assert np.all(conf == 1.0)


def test_truemotion_pulls_a_stray_vector_to_the_consensus_on_flat_content(oracle):
    """truemotion/tests/stage.rs (`the_penalty_prefers_the_consensus_on_a_flat_noisy_block`): a pan
    over a flat, grainy frame gives the flat blocks vectors the grain picked; the penalty brings a
    planted stray vector back to its neighbourhood's."""
    w, h = 96, 64
    rng = np.random.default_rng(4)
    flat = np.full((h, w), 0.5, np.float32)
    a = flat + rng.normal(0, 0.01, (h, w)).astype(np.float32)
    b = flat + rng.normal(0, 0.01, (h, w)).astype(np.float32)
    ring = _ring([a, b])
    pyr = oracle.motion_pyramid(ring, 1, w, h, 1)
    step = 8
    bx, by = -(-w // step), -(-h // step)
    field = np.tile(np.array([2, 1], np.int32), (1, bx * by, 1))
    stray = 3 * bx + 4
    field[0, stray] = (-3, 2)
    th = oracle.thsad(16, 1.0)
    out, _ = oracle.truemotion_pass(pyr, w, h, 2, 0, [1], field, None, field_lambda=1.0, thsad=th,
                                    sad_floor=oracle.sad_noise_floor(16, 0.01), reads_floor=True)
    assert tuple(out[0, stray]) == (2, 1)
    assert np.all(out[0] == (2, 1)), "every block keeps or joins the consensus"


def test_truemotion_keeps_true_motion_on_texture(oracle):
    """stage.rs (`the_penalty_keeps_the_true_motion_on_a_textured_block`): a textured frame shifted
    by (3, -2) keeps that vector through the stage, even from a field seeded off by one."""
    w, h = 96, 64
    f = textured(w, h, 8)
    g = shifted(f, 3, -2)
    ring = _ring([f, g])
    pyr = oracle.motion_pyramid(ring, 1, w, h, 2)
    th = oracle.thsad(16, 1.0)
    mv, _ = oracle.motion_search(pyr, w, h, 2, 0, [1], search_radius=4, thsad=th, field_lambda=1.0)
    inner = mv[0].reshape(-(-h // 8), -(-w // 8), 2)[1:-2, 1:-2]
    assert np.all(inner[..., 0] == 3) and np.all(inner[..., 1] == -2)


def test_truemotion_values_follow_the_stage(oracle):
    """truemotion/stage.rs:52-62: lambda_base = lambda * area * 0.02, fade level 2 thsad."""
    base, noise, fade = oracle.truemotion_values(1.0, 16, oracle.thsad(16, 1.0))
    assert base == pytest.approx(256 * 0.02) and noise == 1.0 and fade == pytest.approx(2 * 256 * 0.02)
    assert oracle.truemotion_values(0.0, 16, 5.0)[:2] == (0.0, 0.0)


# ---- luma motion mapped onto chroma (motion/kernels/chroma_map.rs), the reference's own cases -------
# (motion/tests/chroma_map.rs: blksize 16, step 8 on both planes)

def _grid(w, h):
    return (-(-w // 8), -(-h // 8), 8, 16)


def _field(grid, fn):
    bx, by = grid[0], grid[1]
    return np.array([[fn(c, r) for r in range(by) for c in range(bx)]], np.int32)


def test_map_444_is_the_identity(oracle):
    g = _grid(48, 40)
    v = _field(g, lambda c, r: (c * 3 - 7, r * -5 + 2))
    assert np.array_equal(oracle.map_luma_fields(v, g, g, 0, 0), v)


def test_map_420_halves_both_axes_and_422_x_only(oracle):
    lg = _grid(64, 64)
    out = oracle.map_luma_fields(_field(lg, lambda c, r: (12, -20)), lg, _grid(32, 32), 1, 1)
    assert np.all(out[0] == (6, -10))
    cg = _grid(32, 64)
    out = oracle.map_luma_fields(_field(lg, lambda c, r: (12, r * 10 - 30)), lg, cg, 1, 0)
    for r in range(cg[1]):
        for c in range(cg[0]):
            assert tuple(out[0, r * cg[0] + c]) == (6, r * 10 - 30)


def test_map_takes_the_footprint_median_per_component(oracle):
    lg, cg = _grid(64, 64), _grid(32, 32)
    fx = [[2, 4, 6], [8, 10, 12], [14, 16, 18]]
    fy = [[-40, 4, 8], [-8, 100, 0], [12, -4, 6]]
    v = _field(lg, lambda c, r: (fx[r][c], fy[r][c]) if c < 3 and r < 3 else (500, 500))
    assert tuple(oracle.map_luma_fields(v, lg, cg, 1, 1)[0, 0]) == (5, 2)


@pytest.mark.parametrize("vector,expected", [((1, -1), (1, -1)), ((3, -3), (2, -2)), ((5, -7), (3, -4)),
                                             ((0, 2), (0, 1))])
def test_map_rounds_odd_vectors_half_away_from_zero(oracle, vector, expected):
    lg, cg = _grid(64, 64), _grid(32, 32)
    out = oracle.map_luma_fields(_field(lg, lambda c, r: vector), lg, cg, 1, 1)
    assert tuple(out[0, 1 * cg[0] + 1]) == expected


def test_map_ragged_edges_take_in_bounds_vectors(oracle):
    lg, cg = _grid(37, 35), _grid(19, 18)
    assert lg[:2] == (5, 5) and cg[:2] == (3, 3)
    out = oracle.map_luma_fields(_field(lg, lambda c, r: (c * 20, r * 40)), lg, cg, 1, 1)
    assert tuple(out[0, 2 * 3 + 2]) == (40, 80)
    assert tuple(out[0, 1 * 3 + 1]) == (30, 60)
    lg, cg = _grid(29, 16), _grid(15, 8)
    assert lg[:2] == (4, 2) and cg[:2] == (2, 1)
    out = oracle.map_luma_fields(_field(lg, lambda c, r: (c * 20, r * 40)), lg, cg, 1, 1)
    assert tuple(out[0, 1]) == (20, 0)


# ---- search escalation (motion/escalate.rs; restating motion/tests/escalate.rs) ----

def smooth(w, h, seed):
    """Rows of a horizontal sinusoid, each with its own phase: a SAD surface that falls toward the
    true horizontal motion from every side (the reference suite's smooth world)."""
    phase = np.random.default_rng(seed).random(h)[:, None] * 2 * np.pi
    return (0.5 + 0.3 * np.sin(0.1 * np.arange(w)[None, :] + phase)).astype(np.float32)


def _escalate(oracle, dx, dy, first, ceiling, w=96, h=80, seed=31):
    c = smooth(w, h, seed)
    n = shifted(c, dx, dy)
    pyr = oracle.motion_pyramid(pair_ring(c, n), 1, w, h, 1)
    # A pinned floor and a lenient thsad: only the edge and neighbour rules fail blocks.
    kw = dict(blksize=16, overlap=8, search_radius=first, levels=1, confidence=True, thsad=200.0, sad_floor=0.5,
              esc_reads_floor=True)
    plain, _ = oracle.motion_search(pyr, w, h, 2, 0, [1], **{k: v for k, v in kw.items() if k != "esc_reads_floor"})
    esc, conf = oracle.motion_search(pyr, w, h, 2, 0, [1], ceiling=ceiling, **kw)
    bx, by = -(-w // 8), -(-h // 8)
    inner = lambda f: f[0].reshape(by, bx, 2)[2:-3, 2:-3]  # noqa: E731
    return inner(plain), inner(esc), conf


def test_in_window_motion_needs_no_escalation(oracle):
    plain, esc, _ = _escalate(oracle, 1, 1, 2, 6)
    assert np.all(plain == (1, 1)) and np.array_equal(plain, esc)


def test_an_edge_winner_escalates_to_the_true_motion(oracle):
    plain, esc, _ = _escalate(oracle, 3, 0, 2, 4)
    assert np.all(np.abs(plain[..., 0]) <= 2)  # the first window cannot reach it
    assert np.all(esc == (3, 0))


def test_escalation_stops_at_the_ceiling(oracle):
    _, within, _ = _escalate(oracle, 4, 0, 2, 4)
    assert np.all(within == (4, 0))
    _, beyond, _ = _escalate(oracle, 6, 0, 2, 4)
    assert np.all(np.abs(beyond[..., 0]) <= 4)


def test_escalation_widens_the_coarse_level_too(oracle):
    # Two levels: the coarse seed reaches 2 * 2 = 4 pixels; escalation to 8 re-searches the coarse
    # level at 8, whose winner (x2) seeds a second fine window.
    w, h = 128, 96
    c = smooth(w, h, 5)
    n = shifted(c, 12, 0)
    pyr = oracle.motion_pyramid(pair_ring(c, n), 1, w, h, 2)
    kw = dict(blksize=16, overlap=8, search_radius=2, levels=2, confidence=True, thsad=200.0, sad_floor=0.5)
    plain, _ = oracle.motion_search(pyr, w, h, 2, 0, [1], **kw)
    esc, _ = oracle.motion_search(pyr, w, h, 2, 0, [1], ceiling=8, esc_reads_floor=True, **kw)
    inner = lambda f: f[0].reshape(h // 8, w // 8, 2)[3:-4, 3:-4]  # noqa: E731
    assert np.mean(np.all(inner(plain) == (12, 0), axis=-1)) < 0.5
    assert np.all(inner(esc) == (12, 0))


def test_second_truemotion_pass_keeps_quiet_neighbourhoods(oracle):
    """With change flags in, a block whose 3x3 neighbourhood changed nothing copies its own vector;
    with none set the pass is a copy of its input."""
    w, h = 64, 48
    c = textured(w, h, 9)
    n = shifted(c, 2, 0)
    pyr = oracle.motion_pyramid(pair_ring(c, n), 1, w, h, 1)
    bx, by = w // 8, h // 8
    rng = np.random.default_rng(3)
    mv_in = rng.integers(-3, 4, (1, bx * by, 2)).astype(np.int32)
    out, _ = oracle._truemotion_once(pyr, w, h, 2, 0, [1], mv_in, None, blksize=16, overlap=8, field_lambda=1.0,
                                     thsad=5.12, sad_floor=0.0, reads_floor=True, confidence=False,
                                     changes_in=np.zeros(bx * by, np.uint32))
    assert np.array_equal(out, mv_in)
    flags = np.zeros(bx * by, np.uint32)
    changes = np.zeros(bx * by, np.uint32)
    flags[2 * bx + 3] = 1
    out2, _ = oracle._truemotion_once(pyr, w, h, 2, 0, [1], mv_in, None, blksize=16, overlap=8, field_lambda=1.0,
                                      thsad=5.12, sad_floor=0.0, reads_floor=True, confidence=False,
                                      changes_in=flags, changes_out=changes)
    full, _ = oracle._truemotion_once(pyr, w, h, 2, 0, [1], mv_in, None, blksize=16, overlap=8, field_lambda=1.0,
                                      thsad=5.12, sad_floor=0.0, reads_floor=True, confidence=False)
    near = {(r * bx + c) for r in range(1, 4) for c in range(2, 5)}
    for b in range(bx * by):
        want = full[0, b] if b in near else mv_in[0, b]
        assert tuple(out2[0, b]) == tuple(want), b
        assert changes[b] == (0 if tuple(out2[0, b]) == tuple(mv_in[0, b]) else 1)
