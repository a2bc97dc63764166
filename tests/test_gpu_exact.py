"""The exact NLMeans kernel against the FP32 oracle, bit for bit on float outputs.

With a deterministic tuning every sample is computed by the exact kernel (nlm_exact.cu) in the
operation order of the reference's baseline as the oracle restates it (row-major patch sums,
separately rounded operations, the mirror's exponential), so even the float outputs equal the
oracle's exactly. These cases cover the exact kernel's compile-time patch radii (0..3) and its
generic loop (s = 5, 9), luma and chroma, pairs and the single pass, the noise offsets and tables of
NLMeans-HQ, temporal confidence, the bilateral and NLM-pilot prefilters, frames smaller than the
reach and the frame borders."""

import numpy as np
import pytest

from conftest import avd
from gpu_util import Runner, oracle_pass

pytestmark = pytest.mark.gpu

DET = avd.TuningConfig(deterministic=True)


def clip(w, h, n, chroma="gray", seed=0, depth=8):
    from av_denoise_b200 import synth

    return synth.make_clip(w, h, n, depth=depth, chroma=chroma, sigma_luma=10.0, sigma_chroma=6.0,
                           global_motion=2, sprites=1, sprite_size=24, seed=seed)


def float_planes(frames, depth, chroma):
    """Float planes holding code / max (chroma planes minus the f32 chroma bias), as f32 input."""
    m = float((1 << depth) - 1)
    if not chroma:
        return [[(f[0].astype(np.float32) / np.float32(m)).astype(np.float32)] for f in frames]
    return [[(p.astype(np.float32) / np.float32(m) - np.float32(0.5)).astype(np.float32) for p in f[1:]]
            for f in frames]


def fast(d, a, s, strength, prefilter=None):
    mode = avd.DenoisingMode.temporal(d) if d else avd.DenoisingMode.spacial()
    tuning = avd.NlmTuning(search_radius=a, patch_radius=s, strength=strength)
    kw = {"prefilter": prefilter} if prefilter is not None else {}
    return avd.NlmeansAlgorithm.fast(avd.NlmeansOptions(tuning=tuning, mode=mode, **kw))


def hq(d, a, s, sigma, confidence=False, prefilter=None):
    mode = avd.DenoisingMode.temporal(d) if d else avd.DenoisingMode.spacial()
    kw = {"prefilter": prefilter} if prefilter is not None else {}
    opts = avd.NlmeansOptions(tuning=avd.NlmTuning(search_radius=a, patch_radius=s), mode=mode, **kw)
    return avd.NlmeansAlgorithm.hq_(avd.NlmeansHqOptions(
        nlm=opts, hq=avd.HqParams(sigma_override=sigma, temporal_confidence=confidence)))


def run_exact(oracle, w, h, alg, chroma, d, a, s, strength, seed, **oracle_kw):
    f32 = avd.SampleFormat.f32()
    # chroma: a 4:2:0 clip of twice the size, so its chroma planes are w x h
    frames = clip(2 * w, 2 * h, 5, chroma="420", seed=seed) if chroma else clip(w, h, 5, seed=seed)
    planes = float_planes(frames, 8, chroma)
    if chroma:
        geo = avd.Geometry(2 * w, 2 * h, avd.ChromaLayout.YUV420, f32, f32)
        spec = avd.EngineSpec.nlmeans(None, alg, geo)
        lum = np.zeros((2 * h, 2 * w), np.float32)
        stream = [[lum] + p for p in planes]
    else:
        geo = avd.Geometry(w, h, avd.ChromaLayout.GRAY, f32, f32)
        spec = avd.EngineSpec.nlmeans(alg, None, geo)
        stream = planes
    got = Runner(spec, DET).run(stream)
    want = oracle_pass(oracle, planes, f32, d, a, s, strength, chroma=chroma, **oracle_kw)
    assert len(got) == len(want)
    bad = 0
    for g, wn in zip(got, want):
        gp = g[1:] if chroma else g
        for c in range(len(wn)):
            bad += int((gp[c].view(np.uint32) != wn[c].view(np.uint32)).sum())
    assert bad == 0, f"{bad} float samples differ"


@pytest.mark.parametrize("w,h,d,a,s,strength", [
    (80, 48, 2, 5, 2, 8.0),
    (80, 48, 1, 0, 2, 15.0),
    (64, 40, 0, 7, 3, 12.0),
    (50, 31, 1, 3, 1, 10.0),
    (40, 24, 1, 2, 0, 20.0),
    (48, 32, 1, 3, 5, 30.0),
    (40, 30, 0, 4, 9, 40.0),
    (6, 5, 1, 2, 1, 10.0),
])
def test_exact_luma_floats(oracle, w, h, d, a, s, strength):
    run_exact(oracle, w, h, fast(d, a, s, strength), False, d, a, s, strength, seed=w * h + d)


@pytest.mark.parametrize("d,a,s", [(0, 5, 2), (1, 3, 1), (1, 2, 4)])
def test_exact_chroma_floats(oracle, d, a, s):
    run_exact(oracle, 48, 32, fast(d, a, s, 5.0), True, d, a, s, 5.0, seed=11 + d)


@pytest.mark.parametrize("d,a,s,confidence", [(1, 4, 2, False), (2, 3, 2, True), (0, 5, 3, False)])
def test_exact_hq_floats(oracle, d, a, s, confidence):
    sigma = 10.0 / 255
    strength = avd.hq_default_strength(1, d)
    run_exact(oracle, 72, 48, hq(d, a, s, sigma, confidence), False, d, a, s, strength, seed=30 + d,
              hq_sigma=sigma, hq_confidence=confidence)


def test_exact_hq_chroma_floats(oracle):
    sigma = 6.0 / 255
    run_exact(oracle, 40, 28, hq(1, 3, 2, sigma), True, 1, 3, 2, avd.hq_default_strength(2, 1), seed=5,
              hq_sigma=sigma)


@pytest.mark.parametrize("kind", ["bilateral", "pilot"])
def test_exact_prefilters_floats(oracle, kind):
    pf = avd.PrefilterMode.bilateral(1.5, 0.1) if kind == "bilateral" else avd.PrefilterMode.nlm_spatial(1.5)
    run_exact(oracle, 64, 40, fast(1, 3, 2, 12.0, prefilter=pf), False, 1, 3, 2, 12.0, seed=9, prefilter=pf)
