"""Pins the oracle's automatic noise estimate (oracle/noise_estimate_oracle.cpp) to the reference's
own tests:

- the reading replays av-denoise-core/src/noise/tests/temporal.rs: the same synthetic block
  records, the same expected sample (or its absence) and the same tolerances;
- the window fold is checked against a separate restatement of the reference's host model
  (noise/tests/fold_reference.rs `fold_window`, noise/derived.rs `derive_host`) within the
  reference's 4-ulp bound, and replays noise/tests/window.rs's spike, Immerkaer-fallback and
  clipped-window cases;
- the temporal stats are checked for the record layout of noise/temporal.rs:98-123 and against
  plain sums.
"""

import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import oracle as o  # noqa: E402

F32 = np.float32
STATIC_GATE = F32(1.5) / F32(255.0)
RHO_SIGMA_GATE = F32(0.3) / F32(255.0)
SIGMA_FLOOR = F32(0.1) / F32(255.0)
R_VALID, R_SIGMA, R_SIGMA_LOW, R_RHO, R_STATIC, R_ACCEPTED = 2, 4, 6, 8, 9, 10


# ---- the reading (noise/tests/temporal.rs) ---------------------------------------------------------

def scalar_record(sum_d, sum_d2, sum_lag, channels=1):
    r = np.zeros(o.noise_record_len(channels), np.float32)
    r[0], r[1], r[2] = sum_d, sum_d2, sum_lag
    return r


def zero_mean_block_record(sigma_255, rho):
    sigma = F32(sigma_255) / F32(255.0)
    variance = F32(2.0) * sigma * sigma
    return scalar_record(0.0, F32(256.0) * variance, F32(240.0) * F32(rho) * variance)


def sample(records, channels, w, h):
    """The reading's sample, or None when no channel has one (`aggregate_temporal_noise_stats`)."""
    r = o.noise_reading(np.concatenate(records) if isinstance(records, list) else records, [0, 0], channels, w, h,
                        True)
    if not (r[R_VALID] or r[R_VALID + 1]):
        return None
    return dict(sigma=r[R_SIGMA:R_SIGMA + 2], sigma_low=r[R_SIGMA_LOW:R_SIGMA_LOW + 2], rho=r[R_RHO],
                static_fraction=r[R_STATIC], valid=r[R_VALID:R_VALID + 2])


def test_record_layout():
    assert o.noise_record_len(1) == 29 and o.noise_record_len(2) == 32
    assert o.stats_blocks(32, 16) == (2, 1) and o.stats_blocks(33, 17) == (3, 2)


def test_only_static_block_contributes_to_sigma_and_rho():
    sigma, rho = F32(4.0) / F32(255.0), F32(0.5)
    var = F32(2.0) * sigma * sigma
    static = scalar_record(0.0, F32(256.0) * var, F32(240.0) * rho * var)
    moving = scalar_record(F32(256.0) * (F32(10.0) / F32(255.0)), 0.0, 0.0)
    s = sample([static, moving], 1, 32, 16)
    assert abs(s["static_fraction"] - 0.5) < 1e-6
    assert abs(s["sigma"][0] - sigma) < 1e-4 and abs(s["rho"] - rho) < 1e-4


def test_excludes_perfectly_static_blocks_from_the_population():
    recs = [zero_mean_block_record(s, 0.5) for s in [0.0, 0.0, 0.0, 2.0, 2.5, 3.0, 3.5, 4.0]]
    s = sample(recs, 1, 128, 16)
    assert abs(s["static_fraction"] - 0.625) < 1e-6
    assert abs(s["sigma"][0] - 3.0 / 255) < 1e-4 and abs(s["sigma_low"][0] - 2.5 / 255) < 1e-4


def test_median_over_multiple_static_blocks():
    recs = [zero_mean_block_record(s, r) for s, r in zip([0.1, 2.0, 3.0, 4.0, 5.0], [0.0, 0.1, 0.3, 0.5, 0.7])]
    s = sample(recs, 1, 80, 16)
    assert abs(s["static_fraction"] - 0.8) < 1e-6
    assert abs(s["sigma"][0] - 3.5 / 255) < 1e-4 and abs(s["sigma_low"][0] - 2.75 / 255) < 1e-4
    assert abs(s["rho"] - 0.4) < 1e-4


def test_below_static_floor_returns_none():
    rl = o.noise_record_len(1)
    records = np.zeros(25 * rl, np.float32)
    for b in range(1, 25):
        records[b * rl] = F32(256.0) * (F32(10.0) / F32(255.0))
    sigma = F32(4.0) / F32(255.0)
    var = F32(2.0) * sigma * sigma
    records[1] = F32(256.0) * var
    records[2] = F32(240.0) * F32(0.5) * var
    assert sample(records, 1, 80, 80) is None


def test_zeroed_slot_returns_none():
    assert sample(np.zeros(4 * o.noise_record_len(1), np.float32), 1, 32, 32) is None


def test_multi_channel_layout_reads_correct_offsets():
    r = np.zeros(o.noise_record_len(2), np.float32)
    luma_var = None
    for c, s255 in enumerate([2.0, 4.0]):
        sigma = F32(s255) / F32(255.0)
        var = F32(2.0) * sigma * sigma
        r[2 + c] = F32(256.0) * var
        if c == 0:
            luma_var = var
    r[4] = F32(240.0) * F32(0.6) * luma_var
    s = sample(r, 2, 16, 16)
    assert abs(s["sigma"][0] - 2 / 255) < 1e-4 and abs(s["sigma"][1] - 4 / 255) < 1e-4
    assert abs(s["rho"] - 0.6) < 1e-4


def test_rejects_majority_zero_mean_texture_outliers():
    recs = [zero_mean_block_record(2.0, 0.1)] * 6 + [zero_mean_block_record(20.0, 0.0)] * 10
    s = sample(recs, 1, 64, 64)
    assert abs(s["sigma"][0] - 2 / 255) < 1e-4
    assert abs(s["static_fraction"] - 6 / 16) < 1e-4 and abs(s["rho"] - 0.1) < 1e-4


def test_keeps_genuinely_static_blocks_despite_spatial_sigma_spread():
    recs = [zero_mean_block_record(2.0, 0.1)] * 8 + [zero_mean_block_record(6.0, 0.1)] * 8
    assert abs(sample(recs, 1, 64, 64)["static_fraction"] - 1.0) < 1e-6


@pytest.mark.parametrize("ratio,fraction", [(4.99, 1.0), (5.01, 8.0 / 9.0)])
def test_outlier_factor_boundary(ratio, fraction):
    recs = [zero_mean_block_record(2.0, 0.1)] * 8 + [zero_mean_block_record(2.0 * ratio, 0.0)]
    assert abs(sample(recs, 1, 48, 48)["static_fraction"] - fraction) < 1e-6


def test_correct_sigma_with_letterbox_zero_population():
    levels = [3.8, 3.9, 4.0, 4.1, 4.2]
    recs = [zero_mean_block_record(0.0, 0.0)] * 26 + [zero_mean_block_record(levels[i % 5], 0.2) for i in range(74)]
    s = sample(recs, 1, 160, 160)
    assert abs(s["sigma"][0] - 4 / 255) < 1e-4 and abs(s["rho"] - 0.2) < 1e-4


def test_none_when_the_only_above_gate_population_is_texture():
    recs = [zero_mean_block_record(0.0, 0.0)] * 26 + [zero_mean_block_record(20.0, 0.0)] * 74
    assert sample(recs, 1, 160, 160) is None


def test_rejects_texture_outliers_with_zero_population_present():
    recs = ([zero_mean_block_record(2.0, 0.1)] * 6 + [zero_mean_block_record(20.0, 0.0)] * 10
            + [zero_mean_block_record(0.0, 0.0)] * 4)
    s = sample(recs, 1, 64, 80)
    assert abs(s["sigma"][0] - 2 / 255) < 1e-4
    assert abs(s["static_fraction"] - 6 / 20) < 1e-4 and abs(s["rho"] - 0.1) < 1e-4


def test_keeps_static_spread_with_zero_population_present():
    recs = ([zero_mean_block_record(2.0, 0.1)] * 8 + [zero_mean_block_record(6.0, 0.1)] * 8
            + [zero_mean_block_record(0.0, 0.0)] * 4)
    assert abs(sample(recs, 1, 64, 80)["static_fraction"] - 0.8) < 1e-6


def test_rho_estimate_stays_within_unit_range():
    row = np.array([F32(0.007) * np.sin(F32(i) * F32(np.pi) / F32(17)) for i in range(1, 17)], np.float32)
    sum_d = F32(row.sum(dtype=np.float32)) * F32(16)
    sum_d2 = F32((row * row).sum(dtype=np.float32)) * F32(16)
    sum_lag = F32((row[:-1] * row[1:]).sum(dtype=np.float32)) * F32(16)
    s = sample(scalar_record(sum_d, sum_d2, sum_lag), 1, 16, 16)
    assert 0.0 <= s["rho"] <= 1.0


LOW_TEXTURE, HIGH_TEXTURE = 10.0, 100.0
BRIEF = [(10, 1.0, 0.1, LOW_TEXTURE, False), (5, 1.0, 0.5, LOW_TEXTURE, True), (5, 3.0, 0.5, HIGH_TEXTURE, True)]
MAJORITY = [(3, 1.0, 0.1, LOW_TEXTURE, False), (7, 1.0, 0.1, LOW_TEXTURE, True),
            (10, 3.0, 0.5, HIGH_TEXTURE, True)]


def motion_frame(runs):
    recs = []
    for count, s255, rho, texture, moved in runs:
        r = zero_mean_block_record(s255, rho)
        r[3] = texture  # 2 * channels + BLOCK_TEXTURE_LANE
        r[4] = 1.0 if moved else 0.0  # 2 * channels + BLOCK_MOVED_LANE
        recs += [r] * count
    return recs, 16 * len(recs)


def motion_sample(runs):
    recs, w = motion_frame(runs)
    return sample(recs, 1, w, 16)


def test_moved_high_texture_blocks_leave_sigma_but_keep_rho_and_static_fraction():
    s = motion_sample(BRIEF)
    assert abs(s["sigma"][0] - 1 / 255) < 1e-6 and abs(s["rho"] - 0.3) < 1e-6 and s["static_fraction"] == 1.0


def test_moved_high_texture_majority_leaves_the_sigma_median():
    s = motion_sample(MAJORITY)
    assert abs(s["sigma"][0] - 1 / 255) < 1e-6 and abs(s["sigma_low"][0] - 1 / 255) < 1e-6
    assert abs(s["rho"] - 0.3) < 1e-6 and s["static_fraction"] == 1.0


def test_unmoved_blocks_ignore_texture():
    for runs, expected in [(BRIEF, 1 / 255), (MAJORITY, 2 / 255)]:
        s = motion_sample([(c, s2, r, t, False) for c, s2, r, t, _ in runs])
        assert abs(s["sigma"][0] - expected) < 1e-6 and s["static_fraction"] == 1.0


def test_a_sample_with_every_sigma_left_out_is_invalid():
    recs, w = motion_frame([(8, 20.0, 0.1, LOW_TEXTURE, True), (12, 1.0, 0.1, HIGH_TEXTURE, True)])
    assert sample(recs, 1, w, 16) is None


def test_min_static_blocks():
    for total in [1, 19, 20, 21, 100, 8160, 32400]:
        m = o.min_static_blocks(total)
        assert np.float32(m) / np.float32(total) >= np.float32(0.05)
        assert m == 0 or np.float32(m - 1) / np.float32(total) < np.float32(0.05)


# ---- the temporal stats ------------------------------------------------------------------------

def test_temporal_stats_sums_and_ragged_edges():
    rng = np.random.default_rng(3)
    w, h = 37, 21
    prev = rng.random((h, w, 2), dtype=np.float32)
    new = (prev + rng.normal(0, 0.02, prev.shape)).astype(np.float32)
    rec = o.temporal_stats(new, prev, 2, w, h).reshape(-1, o.noise_record_len(2))
    d = (new - prev).astype(np.float64)
    bx, by = o.stats_blocks(w, h)
    for b in range(bx * by):
        x0, y0 = (b % bx) * 16, (b // bx) * 16
        blk = d[y0:y0 + 16, x0:x0 + 16]
        for c in range(2):
            assert abs(rec[b, c] - blk[..., c].sum()) < 1e-4
            assert abs(rec[b, 2 + c] - (blk[..., c] ** 2).sum()) < 1e-5
        lag = (blk[:, :-1, 0] * blk[:, 1:, 0]).sum()
        assert abs(rec[b, 4] - lag) < 1e-5
        assert rec[b, 6] == 0.0  # moved lane without motion
    # A frame identical to its predecessor reads zero residuals everywhere.
    same = o.temporal_stats(prev, prev, 2, w, h).reshape(-1, o.noise_record_len(2))
    assert not same[:, :5].any()


def test_stats_reading_recovers_the_noise_level():
    rng = np.random.default_rng(4)
    w, h = 160, 96
    base = rng.random((h, w, 1), dtype=np.float32) * 0.2 + 0.4
    frames = [np.clip(base + rng.normal(0, 6 / 255, base.shape), 0, 1).astype(np.float32) for _ in range(3)]
    readings, _ = o.noise_readings(frames, 1, w, h, True)
    assert readings[0][R_VALID] == 0.0  # the first frame's zero records give no sample
    for r in readings[1:]:
        assert r[R_VALID] == 1.0
        assert abs(r[R_SIGMA] * 255 - 6.0) < 0.5, r[R_SIGMA] * 255
        assert r[R_RHO] < 0.1


# ---- the window fold (noise/tests/window.rs, fold_reference.rs) ---------------------------------

COEFF = dict(h2_per_inverse_variance=3.5e-5, h2_fixed=0.0, pilot_h2_factor=0.64, offset_per_variance=50.0,
             main_offset=True, sad_per_sigma=120.0, confidence_sad_per_sigma=180.0)
G_MAX = 1.3
TABLE_RADIUS = 3


def host_factor(rho):
    """noise/correlation.rs:19-36 (`interpolate_table`)."""
    table = [(0.0, 1.0), (0.3, 1.05), (0.5, 1.25), (0.65, 1.45)]
    x = min(max(F32(rho), F32(0.0)), F32(0.65))
    for (x0, y0), (x1, y1) in zip(table, table[1:]):
        if x <= F32(x1):
            return F32(y0) + (x - F32(x0)) / (F32(x1) - F32(x0)) * (F32(y1) - F32(y0))
    return F32(1.45)


def host_fold(readings, imm, first, last, sigma_scale, channels):
    """fold_reference.rs `fold_window` + derived.rs `derive_host`, in f32."""
    win = range(first, last + 1)

    def med(v):
        v = sorted(v)
        return (F32(v[(len(v) - 1) // 2]) + F32(v[len(v) // 2])) * F32(0.5)

    chains = {k: [F32(0)] * 2 for k in ("median", "low", "unb")}
    for c in range(2):
        raw, low, unb = [], [], []
        for f in win:
            r = readings[f]
            has = r[R_VALID + c] != 0
            factor = host_factor(r[R_RHO])
            i, il = imm[f][c], r[c]
            raw.append((max(i, r[R_SIGMA + c] * factor) if has else i) * F32(sigma_scale))
            low.append((max(il, r[R_SIGMA_LOW + c] * factor) if has else il) * F32(sigma_scale))
            unb.append((max(il, r[R_SIGMA_LOW + c]) if has else il) * F32(sigma_scale))
        chains["median"][c] = max(med(raw), SIGMA_FLOOR)
        chains["low"][c] = max(med(low), SIGMA_FLOOR)
        chains["unb"][c] = max(med(unb), SIGMA_FLOOR)
    temporal = list(chains["unb"])
    any_sampled = False
    for c in range(channels):
        v = [readings[f][R_SIGMA + c] * F32(sigma_scale) for f in win if readings[f][R_VALID + c] != 0]
        if v:
            temporal[c] = max(med(v), SIGMA_FLOOR)
            any_sampled = True
    rhos = [readings[f][R_RHO] for f in win if readings[f][R_VALID] != 0]
    rho = med(rhos) if rhos else F32(0)
    sigma = temporal if any_sampled else chains["unb"]
    msum = sum((chains["median"][c] * chains["median"][c] for c in range(channels)), F32(0))
    lsum = sum((chains["low"][c] * chains["low"][c] for c in range(channels)), F32(0))
    h2 = F32(COEFF["h2_per_inverse_variance"]) * F32(channels) / msum
    offset = F32(COEFF["offset_per_variance"]) * lsum
    norm = sigma[0] * sigma[0] * F32(G_MAX) * F32(G_MAX)
    return dict(sigma0=sigma[0], weight=norm, sad=F32(COEFF["sad_per_sigma"]) * chains["median"][0],
                conf=F32(COEFF["confidence_sad_per_sigma"]) * chains["median"][0], h2=h2,
                pilot=h2 * F32(COEFF["pilot_h2_factor"]), offset=offset, rho=rho)


def hashed_readings(n, channels, seed, with_samples=True):
    rng = np.random.default_rng(seed)
    readings, imm = [], []
    for _ in range(n):
        r = np.zeros(o.READING_WORDS, np.float32)
        r[0:channels] = rng.uniform(1, 8, channels) / 255
        if with_samples and rng.random() < 0.8:
            r[R_VALID:R_VALID + channels] = 1.0
            r[R_SIGMA:R_SIGMA + channels] = rng.uniform(1, 8, channels) / 255
            r[R_SIGMA_LOW:R_SIGMA_LOW + channels] = r[R_SIGMA:R_SIGMA + channels] * F32(0.8)
            r[R_RHO] = rng.uniform(0, 0.7)
            r[R_STATIC] = rng.uniform(0.05, 1)
        readings.append(r)
        imm.append(np.concatenate([rng.uniform(1, 8, channels) / 255, np.zeros(2 - channels)]).astype(np.float32))
    return readings, imm


def run_fold(readings, imm, first, last, sigma_scale, channels, w=200, h=120):
    settings = o.fold_words(w, h, sigma_scale=sigma_scale, curve_applies=True, g_max=G_MAX, **COEFF)
    cap = 17 + 2
    records = np.zeros(cap * o.READING_WORDS, np.float32)
    results = np.zeros(cap * 2, np.float32)
    for f in range(first, last + 1):
        records[(f % cap) * 30:(f % cap) * 30 + 30] = readings[f]
        # The fold reads the Immerkaer sigma as factor * abs_sum: store abs sums that give imm.
        results[(f % cap) * 2:(f % cap) * 2 + 2] = imm[f] / settings[12]
    state, derived, spatial, pilot = o.noise_fold(records, results, cap, first, last, settings, channels,
                                                  TABLE_RADIUS)
    imm_read = [settings[12] * (imm[f] / settings[12]) for f in range(len(readings))]
    return state, derived, spatial, pilot, imm_read


def ulps(a, b):
    a, b = np.float32(a), np.float32(b)
    return abs(int(a.view(np.int32)) - int(b.view(np.int32)))


@pytest.mark.parametrize("channels,sigma_scale", [(1, 1.1), (2, 1.0), (1, 0.9)])
def test_window_fold_matches_the_host_model(channels, sigma_scale):
    readings, imm = hashed_readings(20, channels, 17 + channels)
    for centre in [0, 10, 19]:
        first, last = o.noise_window(centre, 19)
        state, derived, spatial, pilot, imm_read = run_fold(readings, imm, first, last, sigma_scale, channels)
        host = host_fold(readings, imm_read, first, last, sigma_scale, channels)
        got = dict(sigma0=derived[0], weight=derived[2], sad=derived[4], conf=derived[5], h2=derived[6],
                   pilot=derived[7], offset=derived[8], rho=derived[10])
        for k, v in host.items():
            assert ulps(got[k], v) <= 4, (k, got[k], v)
        # The tables: spatial at the folded rho, pilot flat; both zero at the centre.
        side = 2 * TABLE_RADIUS + 1
        for i in range(side * side):
            dx, dy = i % side - TABLE_RADIUS, i // side - TABLE_RADIUS
            if dx == dy == 0:
                assert spatial[i] == 0 and pilot[i] == 0
                continue
            rho = derived[10]
            factor = 1.0 if rho <= 0 else 1.0 - float(rho) ** np.sqrt(dx * dx + dy * dy)
            assert abs(spatial[i] - derived[8] * factor) <= 1e-6 * abs(derived[8]) + 1e-12
            assert pilot[i] == derived[9]


def level_readings(n, sigma):
    readings = []
    for _ in range(n):
        r = np.zeros(o.READING_WORDS, np.float32)
        r[0] = sigma
        r[R_VALID] = 1.0
        r[R_SIGMA] = sigma
        r[R_SIGMA_LOW] = sigma
        r[R_RHO] = 0.2
        readings.append(r)
    return readings, [np.array([sigma, 0], np.float32)] * n


def test_one_spiked_record_does_not_move_the_window():
    calm, imm = level_readings(17, F32(2.0) / F32(255.0))
    spiked, imm_s = level_readings(17, F32(2.0) / F32(255.0))
    spiked[5], imm_s[5] = level_readings(1, F32(6.0) / F32(255.0))[0][0], np.array([6 / 255, 0], np.float32)
    a = run_fold(calm, imm, 0, 16, 1.0, 1)
    b = run_fold(spiked, imm_s, 0, 16, 1.0, 1)
    for x, y in zip(a[:4], b[:4]):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


def test_a_window_without_samples_falls_back_to_immerkaer():
    readings, imm = hashed_readings(9, 1, 3, with_samples=False)
    _, derived, _, _, _ = run_fold(readings, imm, 0, 8, 1.0, 1)
    expected = max(sorted(r[0] for r in readings)[4], SIGMA_FLOOR)
    assert derived[0] == expected
    assert derived[10] == 0.0 and np.isfinite(derived).all()


def test_a_clipped_window_uses_only_frames_inside_it():
    readings, imm = hashed_readings(19, 1, 5)
    outside = [r.copy() for r in readings]
    for r in outside[9:]:
        r[:] = level_readings(1, F32(1000.0) / F32(255.0))[0][0]
    a = run_fold(readings, imm, 0, 8, 1.0, 1)
    b = run_fold(outside, imm, 0, 8, 1.0, 1)
    for x, y in zip(a[:4], b[:4]):
        assert np.array_equal(x, y)


def test_correlation_factor_matches_the_host_table():
    settings = o.fold_words(64, 64)
    for rho in np.linspace(-0.2, 0.9, 45, dtype=np.float32):
        assert abs(o.correlation_factor(float(rho), settings) - host_factor(rho)) <= 2e-7
