"""NLMeans prefilters through the C ABI on the GPU, against the CPU oracle on the same seeded frames.

The bilateral prefilter (nlmeans/kernels/bilateral.rs) and the spatial-NLM pilot
(nlmeans/dispatch/mod.rs:598-620) build a reference ring the patch distances compare, while the
averaged values stay the input's (the `_ref` launches of nlmeans/kernels/fused.rs:532-900). The bar
is the NLMeans one: no sample more than 1 LSB from the oracle and >= 99.9% identical over the
non-tie samples (gpu_util.Parity)."""

import numpy as np
import pytest

from conftest import avd
from gpu_util import Parity, Runner, oracle_pass

pytestmark = pytest.mark.gpu


def clip(w, h, n, depth=8, chroma="gray", seed=0, sigma=10.0):
    from av_denoise_b200 import synth

    return synth.make_clip(w, h, n, depth=depth, chroma=chroma, sigma_luma=sigma, sigma_chroma=sigma * 0.6,
                           global_motion=2, sprites=1, sprite_size=24, seed=seed)


def fast(prefilter, d=0, a=2, s=2, strength=1.2):
    mode = avd.DenoisingMode.temporal(d) if d else avd.DenoisingMode.spacial()
    tuning = avd.NlmTuning(search_radius=a, patch_radius=s, strength=strength)
    return avd.NlmeansAlgorithm.fast(avd.NlmeansOptions(prefilter=prefilter, tuning=tuning, mode=mode))


def hq(prefilter, d, a, s, sigma, strength=None, confidence=False):
    mode = avd.DenoisingMode.temporal(d) if d else avd.DenoisingMode.spacial()
    tuning = avd.NlmTuning(search_radius=a, patch_radius=s, strength=strength)
    params = avd.HqParams(sigma_override=sigma, temporal_confidence=confidence)
    opts = avd.NlmeansOptions(prefilter=prefilter, tuning=tuning, mode=mode)
    return avd.NlmeansAlgorithm.hq_(avd.NlmeansHqOptions(nlm=opts, hq=params))


def check(oracle, got_planes, frames, fmt, d, a, s, strength, prefilter, chroma=False, hq_sigma=None,
          hq_confidence=False):
    want, exact = oracle_pass(oracle, frames, fmt, d, a, s, strength, chroma=chroma, exact=True, hq_sigma=hq_sigma,
                              hq_confidence=hq_confidence, prefilter=prefilter)
    par = Parity()
    for g, wn, ex in zip(got_planes, want, exact):
        for c in range(len(wn)):
            par.add(g[c], wn[c], ex[..., c], fmt.max_value())
    st = par.check()
    print(st)
    return st


BILATERAL = [avd.PrefilterMode.bilateral(1.0, 0.1), avd.PrefilterMode.bilateral(2.0, 0.05),
             avd.PrefilterMode.bilateral(0.3, 0.2)]


@pytest.mark.parametrize("w,h,d,a,s,strength,pf", [
    (120, 72, 0, 3, 2, 10.0, 0),
    (100, 66, 2, 4, 2, 8.0, 1),
    (96, 64, 1, 2, 3, 15.0, 2),
    (33, 17, 1, 2, 0, 20.0, 0),  # patch radius 0, ragged tiles
])
def test_bilateral_luma(oracle, w, h, d, a, s, strength, pf):
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 5, seed=300 + w + d)
    prefilter = BILATERAL[pf]
    spec = avd.EngineSpec.nlmeans(fast(prefilter, d, a, s, strength), None,
                                  avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    assert len(got) == len(frames)
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, a, s, strength, prefilter)


def test_bilateral_chroma_10bit(oracle):
    """Two interleaved channels: the range term sums both lanes (bilateral.rs:83-92)."""
    w, h = 96, 64
    fmt = avd.SampleFormat.u16(10)
    frames = clip(w, h, 3, depth=10, chroma="420", seed=311)
    prefilter = avd.PrefilterMode.bilateral(1.5, 0.08)
    spec = avd.EngineSpec.nlmeans(None, fast(prefilter, 1, 3, 2, 6.0),
                                  avd.Geometry(w, h, avd.ChromaLayout.YUV420, fmt, fmt))
    got = Runner(spec).run(frames)
    check(oracle, [[g[1], g[2]] for g in got], [[f[1], f[2]] for f in frames], fmt, 1, 3, 2, 6.0, prefilter,
          chroma=True)


def test_bilateral_largest_radius_on_a_small_frame(oracle):
    """sigma_s = 11 gives the largest radius, 22 (params.rs:78-84), over a frame smaller than the
    kernel: every tap past the edge reads the clamped border."""
    w, h = 20, 12
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 3, seed=313)
    prefilter = avd.PrefilterMode.bilateral(11.0, 0.3)
    spec = avd.EngineSpec.nlmeans(fast(prefilter, 1, 2, 1, 12.0), None,
                                  avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, 1, 2, 1, 12.0, prefilter)


@pytest.mark.parametrize("w,h,d,a,s,strength,scale", [
    (120, 72, 0, 3, 2, 10.0, 0.4),
    (100, 66, 2, 4, 2, 8.0, 1.0),
    (64, 40, 1, 5, 3, 15.0, 0.7),
    (3, 3, 1, 2, 1, 10.0, 0.4),  # minimum frame
])
def test_pilot_luma(oracle, w, h, d, a, s, strength, scale):
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 5, seed=320 + w + d)
    prefilter = avd.PrefilterMode.nlm_spatial(scale)
    spec = avd.EngineSpec.nlmeans(fast(prefilter, d, a, s, strength), None,
                                  avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    assert len(got) == len(frames)
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, a, s, strength, prefilter)


@pytest.mark.parametrize("d,a,s,sigma,confidence", [(1, 4, 2, 10.0 / 255, False), (2, 3, 2, 6.0 / 255, True),
                                                    (0, 5, 1, 14.0 / 255, False)])
def test_pilot_hq_pinned_sigma(oracle, d, a, s, sigma, confidence):
    """NLMeans-HQ with the pilot: the pilot subtracts the input's noise floor, the main pass none
    (nlmeans/denoiser/noise.rs:343-390); the confidence pass still scores the input."""
    w, h = 112, 72
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 4, seed=330 + d)
    prefilter = avd.PrefilterMode.nlm_spatial(0.4)
    spec = avd.EngineSpec.nlmeans(hq(prefilter, d, a, s, sigma, confidence=confidence), None,
                                  avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    strength = avd.hq_default_strength(1, d)
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, a, s, strength, prefilter, hq_sigma=sigma,
          hq_confidence=confidence)


def test_pilot_chroma_hq_and_bilateral_hq(oracle):
    w, h = 96, 64
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 3, chroma="420", seed=341)
    sigma = 6.0 / 255
    for prefilter in (avd.PrefilterMode.nlm_spatial(0.5), avd.PrefilterMode.bilateral(1.0, 0.06)):
        spec = avd.EngineSpec.nlmeans(None, hq(prefilter, 1, 3, 2, sigma, strength=0.8),
                                      avd.Geometry(w, h, avd.ChromaLayout.YUV420, fmt, fmt))
        got = Runner(spec).run(frames)
        check(oracle, [[g[1], g[2]] for g in got], [[f[1], f[2]] for f in frames], fmt, 1, 3, 2, 0.8, prefilter,
              chroma=True, hq_sigma=sigma)


@pytest.mark.parametrize("prefilter", [avd.PrefilterMode.bilateral(1.0, 0.1), avd.PrefilterMode.nlm_spatial(1.0)])
def test_uniform_frame_passes_through(prefilter):
    """prefilter.rs (`bilateral_uniform_image_passthrough`, `nlm_spatial_pilot_uniform_passthrough`):
    a flat frame stays flat."""
    w, h = 16, 16
    fmt = avd.SampleFormat.u8()
    frame = [np.full((h, w), 128, np.uint8)]
    spec = avd.EngineSpec.nlmeans(fast(prefilter, 0, 2, 2, 1.2), None,
                                  avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run([frame])
    assert np.array_equal(got[0][0], frame[0])


def test_prefilter_smooths_more_than_it_moves(oracle):
    """The pilot cleans the distances, so a noisy flat region ends up smoother than without it."""
    w, h = 64, 48
    fmt = avd.SampleFormat.u8()
    rng = np.random.default_rng(7)
    frames = [[np.clip(128 + rng.normal(0, 12, (h, w)), 0, 255).astype(np.uint8)] for _ in range(3)]
    rough = []
    for prefilter in (avd.PrefilterMode.none(), avd.PrefilterMode.nlm_spatial(1.0)):
        spec = avd.EngineSpec.nlmeans(fast(prefilter, 1, 3, 2, 6.0), None,
                                      avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
        got = Runner(spec).run(frames)
        rough.append(float(np.mean([np.abs(np.diff(g[0].astype(np.int32), axis=1)).mean() for g in got])))
    assert rough[1] < rough[0], rough
