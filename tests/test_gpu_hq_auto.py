"""NLMeans-HQ with the automatic noise estimate (no sigma_override) on the GPU through the C ABI
against the oracle's stream restatement: the 8-frame look-ahead reads every frame against the one
before it, each output's window of readings is folded around its centre into h2, the noise offsets
(the spatial table at the folded correlation) and the confidence SAD floor, and the frame is
denoised with them (nlmeans/denoiser/lookahead.rs, noise.rs; noise/*).

The estimate itself is bit-exact (tests/test_gpu_noise_estimate.py); the denoised samples meet the
NLMeans bar (at most 1 LSB apart, >= 99.9% identical outside rounding ties)."""

import numpy as np
import pytest

from conftest import avd
from gpu_util import Parity, Runner

pytestmark = pytest.mark.gpu


def clip(w, h, n, depth=8, chroma="gray", seed=0, sigma=8.0, motion=2):
    from av_denoise_b200 import synth

    return synth.make_clip(w, h, n, depth=depth, chroma=chroma, sigma_luma=sigma, sigma_chroma=sigma * 0.6,
                           global_motion=motion, sprites=1 if motion else 0, sprite_size=24, seed=seed)


def hq_auto(d, a, s, strength=None, confidence=True, auto_strength=True, noise_floor=True, sigma_scale=1.0):
    mode = avd.DenoisingMode.temporal(d) if d else avd.DenoisingMode.spacial()
    tuning = avd.NlmTuning(search_radius=a, patch_radius=s, strength=strength)
    params = avd.HqParams(sigma_override=None, temporal_confidence=confidence, auto_strength=auto_strength,
                          noise_floor=noise_floor, sigma_scale=sigma_scale)
    return avd.NlmeansAlgorithm.hq_(avd.NlmeansHqOptions(nlm=avd.NlmeansOptions(tuning=tuning, mode=mode), hq=params))


def check(oracle, got_planes, frames, fmt, d, a, s, strength, chroma=False, **hq):
    bias = 0.0
    f32 = [oracle.ingest(p, fmt.kind, fmt.max_value(), bias) for p in frames]
    outs, folds = oracle.nlm_stream_hq_auto(f32, d, a, s, strength, **hq)
    exact, _ = oracle.nlm_stream_hq_auto(f32, d, a, s, strength, fp64=True, **hq)
    want = [oracle.egress(o, fmt.kind, fmt.max_value(), bias) for o in outs]
    assert len(got_planes) == len(want)
    par = Parity()
    for g, wn, ex in zip(got_planes, want, exact):
        for c in range(len(wn)):
            par.add(g[c], wn[c], ex[..., c], fmt.max_value())
    st = par.check()
    print(st, "sigma*255 of the first fold:", folds[0][1][0] * 255)
    return folds


@pytest.mark.parametrize("w,h,n,d,a,s,conf", [(128, 80, 12, 2, 3, 2, True), (96, 64, 5, 1, 4, 1, True),
                                              (120, 72, 22, 1, 2, 2, False), (80, 48, 6, 0, 5, 2, False),
                                              (67, 45, 10, 3, 2, 1, True)])
def test_hq_auto_luma_matches_oracle(oracle, w, h, n, d, a, s, conf):
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, n, seed=w + n + d, sigma=7.0)
    spec = avd.EngineSpec.nlmeans(hq_auto(d, a, s, confidence=conf), None,
                                  avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    assert spec.max_held_frames() == d + 8
    got = Runner(spec).run(frames)
    strength = avd.hq_default_strength(1, d)
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, a, s, strength, temporal_confidence=conf)


@pytest.mark.parametrize("d", [0, 2])
def test_hq_auto_finds_the_noise_level_of_a_still_clip(oracle, d):
    """On still content the temporal residual is noise alone (its sigma over sqrt 2), and without a
    temporal sample the Immerkaer estimate stands in: both find the 7-code noise. (On a panning clip
    without motion compensation the residual is shifted texture that clears the static gate, so the
    estimate reads high, as the reference's does.)"""
    w, h, n, a, s = 160, 96, 10, 3, 2
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, n, seed=21, sigma=7.0, motion=0)
    spec = avd.EngineSpec.nlmeans(hq_auto(d, a, s), None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    folds = check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, a, s,
                  avd.hq_default_strength(1, d))
    sig = folds[n // 2][1][0] * 255
    assert 5.5 < sig < 8.5, sig


def test_hq_auto_fixed_strength_without_floor(oracle):
    w, h, n, d, a, s = 96, 64, 9, 2, 3, 2
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, n, seed=5, sigma=12.0)
    spec = avd.EngineSpec.nlmeans(hq_auto(d, a, s, strength=9.0, auto_strength=False, noise_floor=False,
                                          sigma_scale=1.3), None,
                                  avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, a, s, 9.0, auto_strength=False,
          noise_floor=False, sigma_scale=1.3)


def test_hq_auto_chroma_10bit(oracle):
    w, h, n, d, a, s = 112, 72, 11, 1, 3, 2
    fmt = avd.SampleFormat.u16(10)
    frames = clip(w, h, n, depth=10, chroma="420", seed=9, sigma=10.0)
    spec = avd.EngineSpec.nlmeans(None, hq_auto(d, a, s, strength=0.9),
                                  avd.Geometry(w, h, avd.ChromaLayout.YUV420, fmt, fmt))
    got = Runner(spec).run(frames)
    check(oracle, [[g[1], g[2]] for g in got], [[f[1], f[2]] for f in frames], fmt, d, a, s, 0.9)


def test_hq_auto_reset_and_reuse(oracle):
    """A reset drops the look-ahead and the recorded history: a second stream gives the same output."""
    w, h, n, d, a, s = 80, 48, 10, 1, 2, 1
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, n, seed=13)
    spec = avd.EngineSpec.nlmeans(hq_auto(d, a, s), None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    r = Runner(spec)
    first = r.run(frames)
    second = r.run(frames)
    for x, y in zip(first, second):
        assert np.array_equal(x[0], y[0])
    bufs, planes = r.planes_for(frames[0], fmt)
    r.engine.push(planes)
    r.engine.reset()
    third = r.run(frames)
    for x, y in zip(first, third):
        assert np.array_equal(x[0], y[0])


def hq_auto_pilot(d, a, s, scale, confidence=True):
    mode = avd.DenoisingMode.temporal(d) if d else avd.DenoisingMode.spacial()
    tuning = avd.NlmTuning(search_radius=a, patch_radius=s)
    params = avd.HqParams(sigma_override=None, temporal_confidence=confidence)
    opts = avd.NlmeansOptions(prefilter=avd.PrefilterMode.nlm_spatial(scale), tuning=tuning, mode=mode)
    return avd.NlmeansAlgorithm.hq_(avd.NlmeansHqOptions(nlm=opts, hq=params))


@pytest.mark.parametrize("w,h,n,d,a,s,scale,conf", [(96, 64, 12, 1, 3, 2, 0.4, True), (80, 48, 5, 2, 2, 1, 1.0, True),
                                                    (72, 40, 11, 0, 4, 2, 0.6, False)])
def test_hq_auto_with_the_pilot(oracle, w, h, n, d, a, s, scale, conf):
    """The pilot reads the derived words of the latest fold as each frame enters the ring, the first
    frame's after a fold around frame 0 (nlmeans/denoiser/noise.rs:147-165); the main pass compares
    pilot outputs with no noise offset. The oracle replays the front event by event."""
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, n, seed=500 + n + d, sigma=7.0)
    spec = avd.EngineSpec.nlmeans(hq_auto_pilot(d, a, s, scale, conf), None,
                                  avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    strength = avd.hq_default_strength(1, d)
    f32 = [oracle.ingest([f[0]], fmt.kind, fmt.max_value(), 0.0) for f in frames]
    outs, used = oracle.nlm_stream_hq_auto_pilot(f32, d, a, s, strength, scale, temporal_confidence=conf)
    exact, _ = oracle.nlm_stream_hq_auto_pilot(f32, d, a, s, strength, scale, temporal_confidence=conf, fp64=True)
    assert [u[0] for u in used] == list(range(n))
    assert all(u[1][8] == 0.0 for u in used)
    want = [oracle.egress(o, fmt.kind, fmt.max_value(), 0.0) for o in outs]
    assert len(got) == len(want)
    par = Parity()
    for g, wn, ex in zip(got, want, exact):
        par.add(g[0], wn[0], ex[..., 0], fmt.max_value())
    print(par.check())


@pytest.mark.parametrize("w,h,n,d,est,ceiling", [(112, 72, 11, 1, "auto", 0), (96, 64, 12, 3, "auto", 0),
                                                 (88, 56, 6, 2, "chained", 0), (96, 64, 9, 2, "auto", 8)])
def test_hq_auto_with_motion_compensation(oracle, w, h, n, d, est, ceiling):
    """The look-ahead reads each frame along its motion to the frame before it (as NL4D's does);
    each window's fold gives h2, the offsets and the window search's SAD floor, per unit sigma
    sad_noise_floor(16, 1) (nlmeans/denoiser/noise.rs:226-229); the search scores confidence against
    it and the temporal passes compare the warped neighbours."""
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, n, seed=700 + n + d, sigma=7.0)
    estimation = avd.MotionEstimation.CHAINED if est == "chained" else avd.MotionEstimation.AUTO
    # With a ceiling the window search and the look-ahead's pair searches escalate.
    ms = avd.MotionSearch(estimation=estimation, max_search_escalation=max(4, ceiling))
    mode = avd.DenoisingMode.temporal(d)
    opts = avd.NlmeansOptions(motion_compensation=avd.MotionCompensationMode(ms),
                              tuning=avd.NlmTuning(search_radius=3, patch_radius=2), mode=mode)
    alg = avd.NlmeansAlgorithm.hq_(avd.NlmeansHqOptions(nlm=opts, hq=avd.HqParams(sigma_override=None)))
    spec = avd.EngineSpec.nlmeans(alg, None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    strength = avd.hq_default_strength(1, d)
    f32 = [oracle.ingest([f[0]], fmt.kind, fmt.max_value(), 0.0) for f in frames]
    readings, totals = oracle.noise_readings_mc(f32, 1, w, h, blksize=16, overlap=8, search_radius=4, levels=2,
                                                thsad=oracle.thsad(16, 1.0), ceiling=ceiling)
    fl = np.float32
    settings = oracle.fold_words(w, h, h2_per_inverse_variance=oracle.h2_inv_norm(float(fl(strength) * fl(255.0)), 2),
                                 h2_fixed=oracle.h2_inv_norm(strength, 2),
                                 offset_per_variance=float(((fl(2.0) * fl(3.0)) * fl(1.0)) * fl(25.0)),
                                 sad_per_sigma=oracle.sad_noise_floor(16, 1.0))
    folds = oracle.fold_stream(readings, totals, settings, 1, 3, d)

    def derived(frame):
        dv = folds[frame][1]
        return float(dv[6]), float(dv[8]), folds[frame][2], float(dv[4])

    chained = est == "chained" or d >= 3
    kw = dict(confidence=True, chained=chained, derived=derived, ceiling=ceiling)
    outs = oracle.nlm_stream_mc(f32, d, 3, 2, 0.0, **kw)
    exact = oracle.nlm_stream_mc(f32, d, 3, 2, 0.0, fp64=True, **kw)
    want = [oracle.egress(o, fmt.kind, fmt.max_value(), 0.0) for o in outs]
    assert len(got) == len(want) == n
    par = Parity()
    for g, wn, ex in zip(got, want, exact):
        par.add(g[0], wn[0], ex[..., 0], fmt.max_value())
    print(par.check(), "sigma*255 at the middle:", folds[n // 2][1][0] * 255)
