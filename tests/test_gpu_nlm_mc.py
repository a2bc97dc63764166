"""NLMeans with motion compensation through the C ABI on the GPU, against the oracle's slot-by-slot
replay of the ring (nlmeans/dispatch/motion.rs:104-487, denoiser/stages.rs:62-209): each window's
neighbours are matched against the centre (Direct with its truemotion stage, or the Chained pair
walk refined), warped along their fields (motion/kernels/compensate.rs), and the temporal passes
compare the warped frames, with HQ temporal confidence taken from the window search.

The vectors are bit-exact by construction (tests/test_gpu_motion.py); the denoised samples meet
the NLMeans bar (at most 1 LSB apart, >= 99.9% identical outside rounding ties)."""

import pytest

from conftest import avd
from gpu_util import Parity, Runner, oracle_pass

pytestmark = pytest.mark.gpu


def clip(w, h, n, depth=8, chroma="gray", seed=0, sigma=8.0, motion=3):
    from av_denoise_b200 import synth

    return synth.make_clip(w, h, n, depth=depth, chroma=chroma, sigma_luma=sigma, sigma_chroma=sigma * 0.6,
                           global_motion=motion, sprites=1, sprite_size=24, seed=seed)


def search(est=avd.MotionEstimation.AUTO, blksize=16, overlap=8, radius=4, levels=2, refine=2):
    return avd.MotionSearch(blksize=blksize, overlap=overlap, search_radius=radius, max_search_escalation=radius,
                            pyramid_levels=levels, estimation=est, refine_radius=refine)


def options(d, a, s, strength, ms, prefilter=None):
    mode = avd.DenoisingMode.temporal(d) if d else avd.DenoisingMode.spacial()
    tuning = avd.NlmTuning(search_radius=a, patch_radius=s, strength=strength)
    return avd.NlmeansOptions(prefilter=prefilter or avd.PrefilterMode.none(),
                              motion_compensation=avd.MotionCompensationMode(ms), tuning=tuning, mode=mode)


def check(oracle, got_planes, frames, fmt, d, a, s, strength, ms, chroma=False, **kw):
    want, exact = oracle_pass(oracle, frames, fmt, d, a, s, strength, chroma=chroma, exact=True, motion=ms, **kw)
    par = Parity()
    assert len(got_planes) == len(want)
    for g, wn, ex in zip(got_planes, want, exact):
        for c in range(len(wn)):
            par.add(g[c], wn[c], ex[..., c], fmt.max_value())
    st = par.check()
    print(st)
    return st


@pytest.mark.parametrize("w,h,n,d,a,s,strength,ms", [
    (128, 80, 5, 1, 3, 2, 8.0, search()),
    (120, 72, 6, 2, 2, 2, 10.0, search()),
    (112, 64, 7, 3, 2, 1, 12.0, search()),  # Auto resolves to Chained
    (96, 64, 5, 2, 3, 2, 8.0, search(avd.MotionEstimation.CHAINED, refine=1)),
    (96, 64, 5, 3, 2, 2, 8.0, search(avd.MotionEstimation.DIRECT)),
    (100, 60, 4, 1, 2, 2, 8.0, search(blksize=8, overlap=4, radius=3, levels=1)),
    (136, 88, 4, 1, 2, 1, 8.0, search(blksize=32, overlap=16, radius=6, levels=3)),
    (48, 40, 2, 2, 2, 1, 10.0, search()),  # a stream shorter than the window
])
def test_fast_luma_motion_compensated(oracle, w, h, n, d, a, s, strength, ms):
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, n, seed=900 + w + d)
    alg = avd.NlmeansAlgorithm.fast(options(d, a, s, strength, ms))
    spec = avd.EngineSpec.nlmeans(alg, None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    assert len(got) == n
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, a, s, strength, ms)


@pytest.mark.parametrize("d,est", [(1, avd.MotionEstimation.AUTO), (2, avd.MotionEstimation.DIRECT),
                                   (3, avd.MotionEstimation.AUTO)])
def test_hq_pinned_sigma_with_confidence(oracle, d, est):
    """HQ: the window search scores every block against the floor at the pinned sigma and the
    temporal weights take their motion block's confidence (dispatch/mod.rs:175-200)."""
    w, h, sigma = 120, 80, 8.0 / 255
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 5, seed=950 + d)
    ms = search(est)
    params = avd.HqParams(sigma_override=sigma, temporal_confidence=True)
    alg = avd.NlmeansAlgorithm.hq_(avd.NlmeansHqOptions(nlm=options(d, 3, 2, None, ms), hq=params))
    spec = avd.EngineSpec.nlmeans(alg, None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, 3, 2, avd.hq_default_strength(1, d), ms,
          hq_sigma=sigma, hq_confidence=True)


@pytest.mark.parametrize("prefilter,est", [(avd.PrefilterMode.bilateral(1.0, 0.06), avd.MotionEstimation.DIRECT),
                                           (avd.PrefilterMode.nlm_spatial(0.5), avd.MotionEstimation.CHAINED)])
def test_prefilter_with_motion_compensation(oracle, prefilter, est):
    """The search matches on the reference's pyramid and the reference ring is warped along the
    same fields (stages.rs:62-108, dispatch/motion.rs:452-487)."""
    w, h, d = 112, 72, 2
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 5, seed=970)
    ms = search(est)
    alg = avd.NlmeansAlgorithm.fast(options(d, 3, 2, 8.0, ms, prefilter))
    spec = avd.EngineSpec.nlmeans(alg, None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, 3, 2, 8.0, ms, prefilter=prefilter)


def test_chroma_motion_compensated_10bit(oracle):
    """A chroma pass refines the luma guide's mapped vectors on lane 0 (U) and warps both
    interleaved lanes."""
    w, h = 128, 72
    fmt = avd.SampleFormat.u16(10)
    frames = clip(w, h, 4, depth=10, chroma="420", seed=981)
    ms = search()
    spec = avd.EngineSpec.nlmeans(None, avd.NlmeansAlgorithm.fast(options(1, 3, 2, 5.0, ms)),
                                  avd.Geometry(w, h, avd.ChromaLayout.YUV420, fmt, fmt))
    got = Runner(spec).run(frames)
    share = oracle.MotionShare((16, 9, 8, 16), (8, 5, 8, 16), 1, 1)
    f32 = [oracle.ingest([f[0]], fmt.kind, fmt.max_value(), 0.0) for f in frames]
    oracle.nlm_stream_mc(f32, 1, 3, 2, oracle.h2_inv_norm(5.0, 2), share_writes=share)
    check(oracle, [[g[1], g[2]] for g in got], [[f[1], f[2]] for f in frames], fmt, 1, 3, 2, 5.0, ms, chroma=True,
          share_reads=share)


@pytest.mark.parametrize("d,est,radius,ceiling,hq", [(2, avd.MotionEstimation.DIRECT, 2, 6, False),
                                                     (3, avd.MotionEstimation.AUTO, 2, 8, False),
                                                     (1, avd.MotionEstimation.DIRECT, 1, 4, True)])
def test_escalating_motion_compensation(oracle, d, est, radius, ceiling, hq):
    """A search whose max_search_escalation exceeds its radius (the slow presets): failing blocks
    search again up to the ceiling, and the truemotion stage runs a second pass over the blocks
    next to a changed one (motion/escalate.rs, truemotion/stage.rs:82-142)."""
    w, h = 128, 80
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 5, seed=1010 + d, motion=7)
    ms = avd.MotionSearch(blksize=16, overlap=8, search_radius=radius, max_search_escalation=ceiling,
                          pyramid_levels=2, estimation=est, refine_radius=2)
    if hq:
        sigma = 8.0 / 255
        params = avd.HqParams(sigma_override=sigma, temporal_confidence=True)
        alg = avd.NlmeansAlgorithm.hq_(avd.NlmeansHqOptions(nlm=options(d, 3, 2, None, ms), hq=params))
    else:
        alg = avd.NlmeansAlgorithm.fast(options(d, 3, 2, 8.0, ms))
    spec = avd.EngineSpec.nlmeans(alg, None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    if hq:
        check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, 3, 2, avd.hq_default_strength(1, d),
              ms, hq_sigma=sigma, hq_confidence=True)
    else:
        check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, 3, 2, 8.0, ms)


@pytest.mark.parametrize("layout,shifts,d,est", [("420", (1, 1), 2, avd.MotionEstimation.DIRECT),
                                                 ("422", (1, 0), 3, avd.MotionEstimation.AUTO)])
def test_chroma_refines_the_luma_motion(oracle, layout, shifts, d, est):
    """Motion compensation on both planes of one engine: the chroma pass takes the luma pass's
    window fields mapped onto its block grid and searches one pixel around them at one level
    (engine/spec.rs:350-365, nlmeans/dispatch/motion.rs:231-310)."""
    w, h = 112, 64
    fmt = avd.SampleFormat.u8()
    chroma_layout = avd.ChromaLayout.YUV420 if layout == "420" else avd.ChromaLayout.YUV422
    frames = clip(w, h, 5, chroma=layout, seed=990 + d)
    ms = search(est)
    luma = avd.NlmeansAlgorithm.fast(options(d, 3, 2, 8.0, ms))
    chroma = avd.NlmeansAlgorithm.fast(options(d, 3, 2, 5.0, ms))
    spec = avd.EngineSpec.nlmeans(luma, chroma, avd.Geometry(w, h, chroma_layout, fmt, fmt))
    got = Runner(spec).run(frames)
    cw, ch = w >> shifts[0], h >> shifts[1]
    share = oracle.MotionShare((-(-w // 8), -(-h // 8), 8, 16), (-(-cw // 8), -(-ch // 8), 8, 16), *shifts)
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, 3, 2, 8.0, ms, share_writes=share)
    check(oracle, [[g[1], g[2]] for g in got], [[f[1], f[2]] for f in frames], fmt, d, 3, 2, 5.0, ms, chroma=True,
          share_reads=share)


def test_chroma_only_engine_follows_a_luma_guide(oracle):
    """A chroma-only engine with motion compensation: luma passes through, and a luma guide pass
    with the chroma pass's settings searches the motion the chroma pass refines
    (engine/spec.rs:220-236)."""
    import numpy as np

    w, h, d = 112, 64, 2
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 5, chroma="420", seed=995)
    ms = search(avd.MotionEstimation.DIRECT)
    chroma = avd.NlmeansAlgorithm.fast(options(d, 3, 2, 5.0, ms))
    spec = avd.EngineSpec.nlmeans(None, chroma, avd.Geometry(w, h, avd.ChromaLayout.YUV420, fmt, fmt))
    got = Runner(spec).run(frames)
    for g, f in zip(got, frames):
        assert np.array_equal(g[0], f[0])
    share = oracle.MotionShare((-(-w // 8), -(-h // 8), 8, 16), (-(-(w // 2) // 8), -(-(h // 2) // 8), 8, 16), 1, 1)
    f32 = [oracle.ingest([f[0]], fmt.kind, fmt.max_value(), 0.0) for f in frames]
    oracle.nlm_stream_mc(f32, d, 3, 2, oracle.h2_inv_norm(5.0, 2), share_writes=share)
    check(oracle, [[g[1], g[2]] for g in got], [[f[1], f[2]] for f in frames], fmt, d, 3, 2, 5.0, ms, chroma=True,
          share_reads=share)
