"""The NL4D engine (pinned sigma; Direct and Chained motion) on the GPU through the C ABI against the
oracle's stream restatement: the same ring, pass schedule, motion search, pair fields and chains,
group filter and normalise.

Every stage is bit-exact between the two (the motion sums in the reference's order, the filter with
every multiply and add rounded as the restatement rounds them, integer aggregation, the same
normalise), so every output sample is identical."""

import numpy as np
import pytest

from conftest import avd
from gpu_util import Parity, Runner

pytestmark = pytest.mark.gpu

NL4D_TIE_BAND = 1e-4


def clip(w, h, n, depth=8, chroma="gray", seed=0, sigma=10.0):
    from av_denoise_b200 import synth

    return synth.make_clip(w, h, n, depth=depth, chroma=chroma, sigma_luma=sigma, sigma_chroma=sigma * 0.6,
                           global_motion=2, sprites=1, sprite_size=24, seed=seed)


def opts(d, sigma, **kw):
    return avd.Nl4dOptions(sigma=sigma, temporal_radius=d,
                           motion=avd.MotionSearch(estimation=avd.MotionEstimation.DIRECT), **kw)


def oracle_nl4d(oracle, frames, fmt, d, sigma, chroma=False, context=0, **kw):
    f32 = [oracle.ingest(p, fmt.kind, fmt.max_value(), 0.0) for p in frames]
    default_lambda = 3.234 if chroma else 4.158
    lam = kw.pop("lambda_ht", None) or default_lambda
    pooled = kw.pop("pooled_threshold", True)
    outs = oracle.nl4d_stream(f32, d, sigma, lambda_ht=lam, pool_ratio=(2.42 / default_lambda) if pooled else None,
                              context=context, **kw)
    return [oracle.egress(o, fmt.kind, fmt.max_value(), 0.0) for o in outs], outs


def check(oracle, got_planes, frames, fmt, d, sigma, chroma=False, context=0, **kw):
    want, exact = oracle_nl4d(oracle, frames, fmt, d, sigma, chroma=chroma, context=context, **kw)
    assert len(got_planes) == len(want)
    par = Parity()
    for g, wn, ex in zip(got_planes, want, exact):
        for c in range(len(wn)):
            par.add(g[c], wn[c], ex[..., c], fmt.max_value(), tie_band=NL4D_TIE_BAND)
    st = par.check(min_identical=1.0, min_raw=1.0)
    assert st["max_lsb"] == 0, st
    print(st)
    return st


@pytest.mark.parametrize("w,h,n,d,sigma,sr", [(96, 64, 7, 1, 10.0 / 255, 4), (80, 56, 6, 2, 14.0 / 255, 9),
                                              (72, 40, 9, 2, 6.0 / 255, 6)])
def test_nl4d_luma_matches_oracle(oracle, w, h, n, d, sigma, sr):
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, n, seed=w + d)
    spec = avd.EngineSpec.nl4d(opts(d, sigma, spatial_radius=sr), None,
                               avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, sigma, spatial_radius=sr)


def test_nl4d_plain_threshold_10bit(oracle):
    w, h, d, sigma = 64, 48, 1, 8.0 / 255
    fmt = avd.SampleFormat.u16(10)
    frames = clip(w, h, 5, depth=10, seed=5)
    o = opts(d, sigma, spatial_radius=5, pooled_threshold=False, lambda_ht=2.7, kaiser_beta=0.0, c_min=0.2)
    spec = avd.EngineSpec.nl4d(o, None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, sigma, spatial_radius=5,
          pooled_threshold=False, lambda_ht=2.7, kaiser_beta=0.0, c_min=0.2)


@pytest.mark.parametrize("d,est", [(1, avd.MotionEstimation.DIRECT), (3, avd.MotionEstimation.AUTO)])
def test_nl4d_chroma_with_luma_passthrough(oracle, d, est):
    """A chroma-only engine: luma passes through word for word, and a luma guide pass with the
    chroma pass's settings searches the motion the chroma pass refines (engine/spec.rs:220-236)."""
    w, h, sigma = 96, 64, 8.0 / 255
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 5, chroma="420", seed=9 + d)
    o = avd.Nl4dOptions(sigma=sigma, temporal_radius=d, spatial_radius=4, motion=avd.MotionSearch(estimation=est))
    spec = avd.EngineSpec.nl4d(None, o, avd.Geometry(w, h, avd.ChromaLayout.YUV420, fmt, fmt))
    got = Runner(spec).run(frames)
    for g, f in zip(got, frames):
        assert np.array_equal(g[0], f[0])
    share = oracle.MotionShare((12, 8, 8, 16), (6, 4, 8, 16), 1, 1)
    chained = d >= 3
    f32 = [oracle.ingest([f[0]], fmt.kind, fmt.max_value(), 0.0) for f in frames]
    oracle.nl4d_stream(f32, d, sigma, spatial_radius=4, chained=chained, share_writes=share)
    check(oracle, [[g[1], g[2]] for g in got], [[f[1], f[2]] for f in frames], fmt, d, sigma, chroma=True,
          spatial_radius=4, chained=chained, share_reads=share)


@pytest.mark.parametrize("n", [1, 2, 4])
def test_nl4d_short_stream(oracle, n):
    """A stream shorter than the ring is padded with its last frame at flush and every real frame
    is a pass centre (nl4d/denoiser.rs:544-596)."""
    w, h, d, sigma = 64, 40, 2, 10.0 / 255
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, n, seed=20 + n)
    spec = avd.EngineSpec.nl4d(opts(d, sigma, spatial_radius=3), None,
                               avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    assert len(got) == n
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, sigma, spatial_radius=3)


def test_nl4d_continuation_skips_head_passes(oracle):
    """Priming pushes mark a continuation: no head passes (nl4d/engine.rs:310-327)."""
    w, h, d, sigma = 64, 48, 1, 10.0 / 255
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 7, seed=31)
    spec = avd.EngineSpec.nl4d(opts(d, sigma, spatial_radius=3), None,
                               avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames, context=2)
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, sigma, context=2, spatial_radius=3)


def test_nl4d_default_options_build_on_every_layout():
    """The reference's default NL4D call (automatic sigma, noise map on) builds on gray frames and on
    frames with chroma, luma and chroma passes alike, as does search escalation."""
    fmt = avd.SampleFormat.u8()
    for layout in (avd.ChromaLayout.GRAY, avd.ChromaLayout.YUV420, avd.ChromaLayout.YUV444):
        g = avd.Geometry(64, 48, layout, fmt, fmt)
        chroma = None if layout == avd.ChromaLayout.GRAY else avd.Nl4dOptions(temporal_radius=1)
        avd.build_engine(avd.EngineSpec.nl4d(avd.Nl4dOptions(temporal_radius=1), chroma, g)).close()
    g420 = avd.Geometry(64, 48, avd.ChromaLayout.YUV420, fmt, fmt)
    avd.build_engine(avd.EngineSpec.nl4d(None, avd.Nl4dOptions(temporal_radius=1), g420)).close()
    escalating = avd.Nl4dOptions(sigma=0.03, temporal_radius=1, motion=avd.MotionSearch(max_search_escalation=8))
    avd.build_engine(avd.EngineSpec.nl4d(escalating, None, g420)).close()


@pytest.mark.parametrize("n,d,estimation,refine_radius,context", [
    (9, 3, avd.MotionEstimation.AUTO, 2, 0),      # Auto resolves to Chained { refine_radius: 2 } at d >= 3
    (7, 2, avd.MotionEstimation.CHAINED, 1, 0),
    (4, 3, avd.MotionEstimation.AUTO, 2, 0),      # shorter than the ring: duplicated frames' pairs are zero
    (8, 2, avd.MotionEstimation.CHAINED, 3, 2),   # continuation
    (8, 2, avd.MotionEstimation.CHAINED, 3, 0),
    (8, 2, avd.MotionEstimation.CHAINED, 2, 2),
])
def test_nl4d_chained_matches_oracle(oracle, n, d, estimation, refine_radius, context):
    """Chained estimation: pair fields between adjacent frames on every push, every neighbour's seed
    walked from the centre through them, then refined with confidence (motion/chain.rs,
    kernels/chain.rs, analyse.rs:273-316)."""
    w, h, sigma = 96, 64, 10.0 / 255
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, n, seed=40 + n + d)
    o = avd.Nl4dOptions(sigma=sigma, temporal_radius=d, spatial_radius=4,
                        motion=avd.MotionSearch(estimation=estimation, refine_radius=refine_radius))
    spec = avd.EngineSpec.nl4d(o, None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames, context=context)
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, sigma, context=context, spatial_radius=4,
          chained=True, refine_radius=refine_radius)


@pytest.mark.parametrize("layout,shifts,d,est", [("420", (1, 1), 1, avd.MotionEstimation.DIRECT),
                                                 ("422", (1, 0), 2, avd.MotionEstimation.DIRECT),
                                                 ("444", (0, 0), 3, avd.MotionEstimation.AUTO)])
def test_nl4d_chroma_refines_the_luma_motion(oracle, layout, shifts, d, est):
    """Luma and chroma in one engine: the chroma pass takes the luma pass's window fields mapped onto
    its block grid (the lower median of the covered luma blocks, divided by the subsampling) and
    searches one pixel around them at one level (engine/spec.rs:350-365,
    nlmeans/dispatch/motion.rs:231-310); every sample of both planes matches the oracle."""
    w, h, n, sigma = 96, 64, 6, 9.0 / 255
    fmt = avd.SampleFormat.u8()
    chroma_layout = {"420": avd.ChromaLayout.YUV420, "422": avd.ChromaLayout.YUV422,
                     "444": avd.ChromaLayout.YUV444}[layout]
    frames = clip(w, h, n, chroma=layout, seed=31 + d)
    o = avd.Nl4dOptions(sigma=sigma, temporal_radius=d, spatial_radius=5, motion=avd.MotionSearch(estimation=est))
    spec = avd.EngineSpec.nl4d(o, o, avd.Geometry(w, h, chroma_layout, fmt, fmt))
    got = Runner(spec).run(frames)
    cw, ch = w >> shifts[0], h >> shifts[1]
    step = 8
    share = oracle.MotionShare((-(-w // step), -(-h // step), step, 16), (-(-cw // step), -(-ch // step), step, 16),
                               shifts[0], shifts[1])
    chained = est == avd.MotionEstimation.AUTO and d >= 3
    common = dict(spatial_radius=5, chained=chained)
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, sigma, share_writes=share, **common)
    check(oracle, [[g[1], g[2]] for g in got], [[f[1], f[2]] for f in frames], fmt, d, sigma, chroma=True,
          share_reads=share, **common)


@pytest.mark.parametrize("d,chained", [(1, False), (3, True)])
def test_nl4d_escalating_motion_matches_oracle(oracle, d, chained):
    """NL4D under a search that escalates to 8 from radius 2 (the slow preset's ceiling): the
    window search, the pair searches and the chained refine widen their failing blocks, and the
    truemotion stage runs two passes."""
    w, h, sigma = 96, 64, 10.0 / 255
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 2 * d + 3, seed=1200 + d)
    est = avd.MotionEstimation.CHAINED if chained else avd.MotionEstimation.DIRECT
    ms = avd.MotionSearch(search_radius=2, max_search_escalation=8, estimation=est, refine_radius=2)
    o = avd.Nl4dOptions(sigma=sigma, temporal_radius=d, spatial_radius=4, motion=ms)
    spec = avd.EngineSpec.nl4d(o, None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, sigma, spatial_radius=4,
          search_radius=2, chained=chained, refine_radius=2, ceiling=8)
