"""NLMeans prefilters on the CPU: the host API (nlmeans/prefilter/mod.rs, params.rs:349-420) and the
oracle's bilateral and pilot against the reference's behavioural suite (nlmeans/tests/prefilter.rs),
restated on the oracle."""

import re

import numpy as np
import pytest

from conftest import avd

import oracle


def geo():
    fmt = avd.SampleFormat.u8()
    return avd.Geometry(64, 48, avd.ChromaLayout.GRAY, fmt, fmt)


def nlm(prefilter, s=2):
    tuning = avd.NlmTuning(search_radius=2, patch_radius=s, strength=1.2)
    return avd.NlmeansAlgorithm.fast(avd.NlmeansOptions(prefilter=prefilter, tuning=tuning))


# ---- prefilter/mod.rs:119-218 ----

def test_reference_buffer_and_gpu_internal():
    assert not avd.PrefilterMode.none().needs_reference_buf()
    assert not avd.PrefilterMode.none().is_gpu_internal()
    for mode in (avd.PrefilterMode.bilateral(3.0, 0.02), avd.PrefilterMode.nlm_spatial(1.0)):
        assert mode.needs_reference_buf() and mode.is_gpu_internal()


def test_bilateral_radius_truncates_at_two_sigma():
    assert [avd.bilateral_radius(x) for x in (0.1, 1.0, 3.0, 3.5)] == [1, 2, 6, 7]
    assert [oracle.bilateral_radius(x) for x in (0.1, 1.0, 3.0, 3.5)] == [1, 2, 6, 7]


def test_parse_prefilter():
    assert avd.parse_prefilter("none").kind == 0
    assert avd.parse_prefilter("").kind == 0
    b = avd.parse_prefilter("bilateral:3.0,0.02")
    assert b.kind == 1 and abs(b.sigma_s - 3.0) < 1e-7 and abs(b.sigma_r - 0.02) < 1e-7
    n = avd.parse_prefilter("nlm")
    assert n.kind == 2 and n.strength_scale == avd.DEFAULT_PILOT_STRENGTH_SCALE == 0.4
    assert avd.parse_prefilter("nlm:0.8").strength_scale == 0.8
    with pytest.raises(ValueError, match="nlm"):
        avd.parse_prefilter("nlm:x")
    with pytest.raises(ValueError):
        avd.parse_prefilter("garbage")
    with pytest.raises(ValueError, match="two values"):
        avd.parse_prefilter("bilateral:1.0")


# ---- params.rs:349-420 ----

def test_validate_accepts_prefilters():
    avd.EngineSpec.nlmeans(nlm(avd.PrefilterMode.bilateral(1.0, 0.1)), None, geo()).validate()
    avd.EngineSpec.nlmeans(nlm(avd.PrefilterMode.bilateral(11.0, 0.1)), None, geo()).validate()
    avd.EngineSpec.nlmeans(nlm(avd.PrefilterMode.nlm_spatial(0.4)), None, geo()).validate()
    avd.EngineSpec.nlmeans(nlm(avd.PrefilterMode.nlm_spatial(0.4), s=8), None, geo()).validate()


@pytest.mark.parametrize("prefilter,text", [
    (avd.PrefilterMode.bilateral(0.0, 0.1), "sigma_s must be finite and greater than 0"),
    (avd.PrefilterMode.bilateral(float("nan"), 0.1), "sigma_s must be finite"),
    (avd.PrefilterMode.bilateral(1.0, 0.0), "sigma_r must be finite and greater than 0"),
    (avd.PrefilterMode.bilateral(11.5, 0.1), "tile radius of 23"),
    (avd.PrefilterMode.bilateral(1e-30, 0.1), "sigma_s is too small"),
    (avd.PrefilterMode.bilateral(1.0, 1e-30), "sigma_r is too small"),
    (avd.PrefilterMode.nlm_spatial(0.0), "strength_scale must be finite and greater than 0"),
    (avd.PrefilterMode.nlm_spatial(float("inf")), "strength_scale must be finite"),
])
def test_validate_rejects_bad_prefilters(prefilter, text):
    with pytest.raises(avd.InvalidOptions, match=re.escape(text)):
        avd.EngineSpec.nlmeans(nlm(prefilter), None, geo()).validate()


def test_pilot_patch_radius_limit():
    with pytest.raises(avd.InvalidOptions, match="supports patch_radius up to 8"):
        avd.EngineSpec.nlmeans(nlm(avd.PrefilterMode.nlm_spatial(0.4), s=9), None, geo()).validate()


# ---- the oracle against nlmeans/tests/prefilter.rs ----

def uniform(w, h, c, v):
    return np.full((h, w, c), v, np.float32)


def noisy_region(w, h, c, base, cx, cy, r, peak, seed=1):
    rng = np.random.default_rng(seed)
    f = uniform(w, h, c, base)
    f[cy - r:cy + r + 1, cx - r:cx + r + 1] = peak + rng.normal(0, 0.05, (2 * r + 1, 2 * r + 1, c))
    return np.clip(f, 0.0, 1.0).astype(np.float32)


def gaussian(w, h, c, mean, sigma, seed=2):
    rng = np.random.default_rng(seed)
    return np.clip(mean + rng.normal(0, sigma, (h, w, c)), 0.0, 1.0).astype(np.float32)


def roughness(f):
    return float(np.mean(np.abs(np.diff(f[..., 0], axis=1))) + np.mean(np.abs(np.diff(f[..., 0], axis=0))))


def test_bilateral_uniform_image_passthrough():
    f = uniform(16, 16, 1, 0.5)
    ref = oracle.bilateral(f, 1.0, 0.1)
    assert np.abs(ref - 0.5).max() < 1e-4
    h2 = oracle.h2_inv_norm(1.2, 2)
    out = oracle.nlm_stream_repeat([f], 0, 2, 2, h2, prefilter=("bilateral", 1.0, 0.1))[0]
    assert np.abs(out - 0.5).max() < 1e-4


def test_bilateral_noisy_image_finite():
    f = noisy_region(16, 16, 1, 0.4, 8, 8, 3, 0.8)
    ref = oracle.bilateral(f, 2.0, 0.05)
    assert np.isfinite(ref).all()
    out = oracle.nlm_stream_repeat([f], 0, 2, 2, oracle.h2_inv_norm(1.2, 2), prefilter=("bilateral", 2.0, 0.05))[0]
    assert np.isfinite(out).all() and out.min() >= -0.01 and out.max() <= 1.01


def test_bilateral_keeps_an_edge():
    """A step larger than sigma_r stays a step: the range term keeps the two sides apart."""
    f = uniform(24, 8, 1, 0.2)
    f[:, 12:] = 0.8
    ref = oracle.bilateral(f, 2.0, 0.05)
    assert np.abs(ref[:, :12] - 0.2).max() < 1e-4 and np.abs(ref[:, 12:] - 0.8).max() < 1e-4


def test_bilateral_two_channels_against_a_direct_sum():
    """The FP32 mirror against a float64 restatement of the same sum."""
    f = gaussian(12, 9, 2, 0.5, 0.1)
    ss, sr = 1.3, 0.2
    r = oracle.bilateral_radius(ss)
    inv_s, inv_r = 1.0 / (2 * ss * ss), 1.0 / (2 * sr * sr)
    got = oracle.bilateral(f, ss, sr)
    h, w, _ = f.shape
    want = np.zeros_like(got, np.float64)
    for y in range(h):
        for x in range(w):
            acc, ws = np.zeros(2), 0.0
            for dy in range(-r, r + 1):
                for dx in range(-r, r + 1):
                    n = f[min(max(y + dy, 0), h - 1), min(max(x + dx, 0), w - 1)].astype(np.float64)
                    wt = np.exp(-((dx * dx + dy * dy) * inv_s + np.sum((n - f[y, x]) ** 2) * inv_r))
                    acc += wt * n
                    ws += wt
            want[y, x] = acc / ws
    assert np.abs(got - want).max() < 2e-6


def test_nlm_spatial_pilot_fills_reference():
    f = gaussian(16, 16, 1, 0.5, 6.0 / 255.0)
    h2 = oracle.h2_inv_norm(1.2, 2)
    ref = oracle.prefilter_refs([f], ("nlm", oracle.pilot_h2(h2, 1.0), None), 2, 2)[0]
    assert np.isfinite(ref).all() and ref.min() >= 0.0 and ref.max() <= 1.0
    assert np.abs(ref - f).max() > 1e-6


def test_nlm_spatial_pilot_smooths():
    f = gaussian(32, 32, 1, 0.5, 10.0 / 255.0)
    h2 = oracle.h2_inv_norm(1.2, 2)
    ref = oracle.prefilter_refs([f], ("nlm", oracle.pilot_h2(h2, 1.0), None), 2, 2)[0]
    assert roughness(ref) < roughness(f)


def test_nlm_spatial_pilot_uniform_passthrough():
    f = uniform(16, 16, 1, 0.5)
    h2 = oracle.h2_inv_norm(1.2, 2)
    ref = oracle.prefilter_refs([f], ("nlm", oracle.pilot_h2(h2, 1.0), None), 2, 2)[0]
    assert np.abs(ref - 0.5).max() < 1e-4


def test_reference_frames_only_steer_the_weights():
    """With the reference equal to the input, the `_ref` form is the plain pass bit for bit; with
    another reference the output stays a weighted mean of the input's own values."""
    rng = np.random.default_rng(5)
    win = [rng.random((10, 14, 1), dtype=np.float32) for _ in range(3)]
    h2 = oracle.h2_inv_norm(3.0, 1)
    plain = oracle.nlm_frame(win, 1, 2, 1, h2)
    same = oracle.nlm_frame(win, 1, 2, 1, h2, refs=win)
    assert np.array_equal(plain, same)
    refs = [oracle.bilateral(x, 1.0, 0.2) for x in win]
    other = oracle.nlm_frame(win, 1, 2, 1, h2, refs=refs)
    lo = min(float(x.min()) for x in win)
    hi = max(float(x.max()) for x in win)
    assert other.min() >= lo - 1e-6 and other.max() <= hi + 1e-6
    assert not np.array_equal(other, plain)


def test_pilot_fold_words_zero_the_main_offset():
    """nlmeans/tests/prefilter.rs (`nlm_spatial_zeros_main_offset_but_keeps_input_offset`) on the
    measured path: the fold writes no main-pass offset under the pilot but keeps the input's, and
    the pilot strength is h2 / scale^2."""
    w, h = 64, 48
    rng = np.random.default_rng(9)
    frames = [np.clip(0.5 + rng.normal(0, 8 / 255, (h, w, 1)), 0, 1).astype(np.float32) for _ in range(4)]
    readings, totals = oracle.noise_readings(frames, 1, w, h, True)
    scale = 0.5
    common = dict(h2_per_inverse_variance=2.0, h2_fixed=oracle.h2_inv_norm(1.0, 2), offset_per_variance=30.0)
    main = oracle.fold_words(w, h, **common)
    pilot = oracle.fold_words(w, h, pilot_h2_factor=1.0 / (scale * scale), main_offset=False, **common)
    fm = oracle.fold_stream(readings, totals, main, 1, 2, 1)[1]
    fp = oracle.fold_stream(readings, totals, pilot, 1, 2, 1)[1]
    assert fm[1][8] > 0.0 and fp[1][8] == 0.0
    assert fp[1][9] == fm[1][9] == fm[1][8]
    assert np.float32(fp[1][7]) == np.float32(np.float32(fp[1][6]) * np.float32(1.0 / (scale * scale)))
    assert not fp[2].any() and fp[3].any()
