"""NLMeans through the C ABI on the GPU, against the CPU oracle on the same seeded frames.

Bar (north star): at the source bit depth no sample more than 1 LSB from the oracle and >= 99.9% of
all samples identical (gpu_util.Parity); float outputs within 2e-5 absolute.
Passthrough planes are bit exact."""

import numpy as np
import pytest

from conftest import avd
from gpu_util import Parity, Runner, oracle_pass

pytestmark = pytest.mark.gpu


def nlm(d=0, a=2, s=2, strength=1.2, wref=None):
    mode = avd.DenoisingMode.temporal(d) if d else avd.DenoisingMode.spacial()
    tuning = avd.NlmTuning(search_radius=a, patch_radius=s, strength=strength, self_weight=wref)
    return avd.NlmeansAlgorithm.fast(avd.NlmeansOptions(tuning=tuning, mode=mode))


def clip(w, h, n, depth=8, chroma="gray", seed=0, sigma=10.0):
    from av_denoise_b200 import synth

    return synth.make_clip(w, h, n, depth=depth, chroma=chroma, sigma_luma=sigma, sigma_chroma=sigma * 0.6,
                           global_motion=2, sprites=1, sprite_size=24, seed=seed)


def fmt_for(depth):
    return avd.SampleFormat.u8() if depth == 8 else avd.SampleFormat.u16(depth)


def check_group(oracle, got_planes, frames, fmt, d, a, s, strength, chroma=False, wref=1.0,
                hq_sigma=None, hq_confidence=False, thsad_scale=1.0):
    """Compares one plane group of every emitted frame with the oracle; returns the stats."""
    want, exact = oracle_pass(oracle, frames, fmt, d, a, s, strength, wref=wref, chroma=chroma, exact=True,
                              hq_sigma=hq_sigma, hq_confidence=hq_confidence, thsad_scale=thsad_scale)
    par = Parity()
    for g, wn, ex in zip(got_planes, want, exact):
        for c in range(len(wn)):
            par.add(g[c], wn[c], ex[..., c], fmt.max_value())
    st = par.check()
    print(st)
    return st


@pytest.mark.parametrize(
    "w,h,depth,d,a,s,strength",
    [
        (160, 90, 8, 0, 7, 3, 12.0),  # the 640x360 spatial workload's parameters
        (140, 90, 8, 2, 5, 2, 8.0),  # the 1080p temporal luma parameters, odd sizes
        (128, 80, 10, 1, 4, 2, 30.0),
        (100, 74, 12, 0, 3, 1, 120.0),
        (65, 33, 8, 1, 2, 0, 20.0),  # patch radius 0
        # Search radius 0: the single pass is empty and the max weight is the larger pair weight,
        # so every sample with one dominant neighbour frame is a half-code tie (the FP32 oracle
        # agrees with FP64 on only ~98.7% of them); the exact finish decides them as the oracle does.
        (80, 48, 8, 1, 0, 2, 15.0),
        (96, 80, 8, 0, 4, 9, 40.0),  # patch radius above the reference's separable threshold
        (3, 3, 8, 1, 2, 1, 10.0),  # minimum frame: 45 samples
    ])
def test_luma_parity(oracle, w, h, depth, d, a, s, strength):
    fmt = fmt_for(depth)
    frames = clip(w, h, 5, depth=depth, seed=w * h + d)
    spec = avd.EngineSpec.nlmeans(nlm(d, a, s, strength), None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    assert len(got) == len(frames)
    check_group(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, a, s, strength)


def test_chroma_only_with_luma_passthrough(oracle):
    w, h = 144, 100
    frames = clip(w, h, 4, chroma="420", seed=3)
    fmt = avd.SampleFormat.u8()
    spec = avd.EngineSpec.nlmeans(None, nlm(0, 5, 2, 5.0), avd.Geometry(w, h, avd.ChromaLayout.YUV420, fmt, fmt))
    got = Runner(spec).run(frames)
    for i, g in enumerate(got):
        assert np.array_equal(g[0], frames[i][0])  # luma passes through word for word
    # Strength 5 on chroma: one neighbour often dominates, so half-code ties are common; the exact
    # finish recomputes them in the oracle's order.
    check_group(oracle, [[g[1], g[2]] for g in got], [[f[1], f[2]] for f in frames], fmt, 0, 5, 2, 5.0,
                chroma=True)


def test_luma_temporal_with_chroma_passthrough(oracle):
    w, h = 130, 74
    frames = clip(w, h, 6, chroma="420", seed=4)
    fmt = avd.SampleFormat.u8()
    spec = avd.EngineSpec.nlmeans(nlm(2, 5, 2, 8.0), None, avd.Geometry(w, h, avd.ChromaLayout.YUV420, fmt, fmt))
    got = Runner(spec).run(frames)
    assert len(got) == 6
    for i, g in enumerate(got):
        assert np.array_equal(g[1], frames[i][1]) and np.array_equal(g[2], frames[i][2])
    check_group(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, 2, 5, 2, 8.0)


@pytest.mark.parametrize("layout", [avd.ChromaLayout.YUV444, avd.ChromaLayout.YUV422])
def test_luma_and_chroma_10bit(oracle, layout):
    w, h = 96, 72
    name = {avd.ChromaLayout.YUV444: "444", avd.ChromaLayout.YUV422: "422"}[layout]
    frames = clip(w, h, 4, depth=10, chroma=name, seed=9)
    fmt = avd.SampleFormat.u16(10)
    spec = avd.EngineSpec.nlmeans(nlm(1, 3, 2, 20.0), nlm(1, 3, 1, 12.0), avd.Geometry(w, h, layout, fmt, fmt))
    got = Runner(spec).run(frames)
    check_group(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, 1, 3, 2, 20.0)
    check_group(oracle, [[g[1], g[2]] for g in got], [[f[1], f[2]] for f in frames], fmt, 1, 3, 1, 12.0,
                chroma=True)


def test_float_planes(oracle):
    w, h = 40, 30
    rng = np.random.default_rng(1)
    frames = [[rng.random((h, w), dtype=np.float32), (rng.random((h // 2, w // 2), dtype=np.float32) - 0.5),
               (rng.random((h // 2, w // 2), dtype=np.float32) - 0.5)] for _ in range(3)]
    fmt = avd.SampleFormat.f32()
    spec = avd.EngineSpec.nlmeans(nlm(1, 2, 1, 60.0), nlm(1, 2, 1, 60.0),
                                  avd.Geometry(w, h, avd.ChromaLayout.YUV420, fmt, fmt))
    got = Runner(spec).run(frames)
    want_y = oracle_pass(oracle, [[f[0]] for f in frames], fmt, 1, 2, 1, 60.0)
    want_c = oracle_pass(oracle, [[f[1], f[2]] for f in frames], fmt, 1, 2, 1, 60.0, chroma=True)
    for g, wy, wc in zip(got, want_y, want_c):
        np.testing.assert_allclose(g[0], wy[0], atol=2e-5, rtol=0)
        np.testing.assert_allclose(g[1], wc[0], atol=2e-5, rtol=0)
        np.testing.assert_allclose(g[2], wc[1], atol=2e-5, rtol=0)


def test_float_intermediates_against_fp64(oracle):
    """u8 in, f32 out: the kernel's float result against the FP64 oracle, max relative error."""
    w, h = 96, 64
    fin, fout = avd.SampleFormat.u8(), avd.SampleFormat.f32()
    frames = clip(w, h, 5, seed=31)
    spec = avd.EngineSpec.nlmeans(nlm(2, 5, 2, 8.0), None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fin, fout))
    got = Runner(spec).run(frames)
    f32 = [oracle.ingest([f[0]], 0, 255.0) for f in frames]
    exact = oracle.nlm_stream_repeat(f32, 2, 5, 2, oracle.h2_inv_norm(8.0, 2), fp64=True)
    rel = max(float(np.max(np.abs(g[0] - e[..., 0]) / np.maximum(np.abs(e[..., 0]), 1e-3)))
              for g, e in zip(got, exact))
    print("max relative error against FP64:", rel)
    assert rel < 1e-5


def test_self_weight_zero_and_uniform_frame(oracle):
    w, h = 20, 20
    fmt = avd.SampleFormat.u8()
    frames = [[np.full((h, w), 77, np.uint8)] for _ in range(2)]
    spec = avd.EngineSpec.nlmeans(nlm(0, 3, 2, 1.2, wref=0.0), None,
                                  avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    for g in got:
        assert (g[0] == 77).all()


def test_stream_shorter_than_window(oracle):
    # d = 8 with two frames: both repeat edges fill the window (ring.rs:106-146).
    w, h = 48, 40
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 2, seed=21)
    spec = avd.EngineSpec.nlmeans(nlm(8, 2, 1, 10.0), None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    assert len(got) == 2
    check_group(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, 8, 2, 1, 10.0)


def test_engine_errors_and_poison():
    import torch

    w, h = 16, 16
    fmt = avd.SampleFormat.u8()
    spec = avd.EngineSpec.nlmeans(nlm(1, 2, 1, 10.0), None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    r = Runner(spec)
    e = r.engine
    frames = clip(w, h, 4, seed=5)
    _, p0 = r.planes_for(frames[0], fmt)
    _, p1 = r.planes_for(frames[1], fmt)
    with pytest.raises(avd.NothingToEmit):
        e.emit_into(r.out_planes())
    assert e.push(p0) == 0
    assert e.push(p1) == 1
    with pytest.raises(avd.OutputsPending):
        e.push(p1)
    e.emit_into(r.out_planes())
    with pytest.raises(avd.ContextAfterPush):
        e.push_context(p0)
    with pytest.raises(avd.PlaneMismatch):
        e.push([avd.DevicePlane(p0[0].ptr, p0[0].bytes, w + 1, h)])
    with pytest.raises(avd.PlaneMismatch):
        e.push([avd.DevicePlane(p0[0].ptr, 8, w, h)])
    with pytest.raises(avd.PlaneMismatch):
        e.push([p0[0], p0[0]])
    with pytest.raises(avd.GpuError):
        e.fail_for_test()
    with pytest.raises(avd.NeedsReset):
        e.push(p0)
    e.reset()
    assert e.push(p0) == 0
    assert e.finish() == 1
    r.emit()
    with pytest.raises(avd.NothingToEmit):
        e.emit_into(r.out_planes())
    assert e.max_held_frames() == 1
    span = e.window_span()
    assert (span.behind, span.ahead, span.edges) == (1, 1, "repeat")
    torch.cuda.synchronize()


def test_push_context_reseeds_mid_clip(oracle):
    # engine/mod.rs:74-81: context frames fill the window so a stream can start mid-clip. A stream
    # that starts at frame 2 with frame 1 as context reproduces the full stream's output for every
    # frame whose window does not reach back past frame 1.
    w, h = 30, 22
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 8, seed=8)
    spec = avd.EngineSpec.nlmeans(nlm(1, 2, 1, 10.0), None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    full = Runner(spec).run(frames)
    part = Runner(spec).run(frames[1:], context=1)
    assert len(part) == 7  # the context frame is emitted too
    for i in range(2, 8):
        assert np.array_equal(part[i - 1][0], full[i][0])


def test_device_timing():
    w, h = 64, 48
    fmt = avd.SampleFormat.u8()
    spec = avd.EngineSpec.nlmeans(nlm(1, 3, 2, 10.0), None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    r = Runner(spec)
    r.engine.sample_device_time(1)
    r.run(clip(w, h, 4, seed=2))
    t = r.engine.timing()
    assert t.luma is not None and t.luma.frames == 4 and t.luma.device_time > 0
    assert t.chroma is None


def test_full_1080p_crops_match_oracle(oracle):
    """Full-size frames (1920x1080 4:2:0, luma d=2, a=5, s=2): the oracle on interior and corner
    crops with a margin of a+s reproduces the GPU output inside each crop."""
    from av_denoise_b200 import synth

    frames = synth.temporal_1080p_clip(frames=5)
    fmt = avd.SampleFormat.u8()
    spec = avd.EngineSpec.nlmeans(nlm(2, 5, 2, 8.0), None, avd.Geometry(1920, 1080, avd.ChromaLayout.YUV420, fmt, fmt))
    got = Runner(spec).run(frames)
    m = 7
    par = Parity()
    for (cx, cy) in [(0, 0), (900, 500), (1920 - 96, 1080 - 96), (1600, 37)]:
        x0, y0 = max(cx - m, 0), max(cy - m, 0)
        x1, y1 = min(cx + 96 + m, 1920), min(cy + 96 + m, 1080)
        crop = [[f[0][y0:y1, x0:x1]] for f in frames]
        want, exact = oracle_pass(oracle, crop, fmt, 2, 5, 2, 8.0, exact=True)
        ix0 = 0 if x0 == 0 else m
        iy0 = 0 if y0 == 0 else m
        ix1 = (x1 - x0) if x1 == 1920 else (x1 - x0 - m)
        iy1 = (y1 - y0) if y1 == 1080 else (y1 - y0 - m)
        for i in range(5):
            g = got[i][0][y0:y1, x0:x1]
            par.add(g[iy0:iy1, ix0:ix1], want[i][0][iy0:iy1, ix0:ix1], exact[i][iy0:iy1, ix0:ix1, 0], 255.0)
    print(par.check())


def hq(d, a, s, sigma, strength=None, confidence=False, thsad_scale=1.0):
    mode = avd.DenoisingMode.temporal(d) if d else avd.DenoisingMode.spacial()
    tuning = avd.NlmTuning(search_radius=a, patch_radius=s, strength=strength)
    params = avd.HqParams(sigma_override=sigma, temporal_confidence=confidence, thsad_scale=thsad_scale)
    return avd.NlmeansAlgorithm.hq_(avd.NlmeansHqOptions(nlm=avd.NlmeansOptions(tuning=tuning, mode=mode), hq=params))


@pytest.mark.parametrize("d,a,s,sigma", [(1, 4, 2, 10.0 / 255), (0, 5, 3, 6.0 / 255), (2, 3, 1, 14.0 / 255)])
def test_hq_pinned_sigma_luma(oracle, d, a, s, sigma):
    """NLMeans-HQ with sigma_override: strength = hq_default_strength * sigma * 255 and the noise
    floor subtracted from every distance (flat spatial table at rho = 0)."""
    w, h = 120, 72
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 4, seed=40 + d)
    spec = avd.EngineSpec.nlmeans(hq(d, a, s, sigma), None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    strength = avd.hq_default_strength(1, d)
    # The noise floor clamps many distances to 0, so many weights are exactly 1 and many outputs
    # exact means of integer codes: ~10% of samples are half-code ties here, all of them recomputed
    # by the exact finish.
    check_group(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, a, s, strength, hq_sigma=sigma)


def test_hq_pinned_sigma_chroma_10bit(oracle):
    w, h = 96, 64
    fmt = avd.SampleFormat.u16(10)
    frames = clip(w, h, 3, depth=10, chroma="420", seed=44)
    sigma = 5.0 / 255
    spec = avd.EngineSpec.nlmeans(None, hq(0, 4, 2, sigma, strength=0.9),
                                  avd.Geometry(w, h, avd.ChromaLayout.YUV420, fmt, fmt))
    got = Runner(spec).run(frames)
    check_group(oracle, [[g[1], g[2]] for g in got], [[f[1], f[2]] for f in frames], fmt, 0, 4, 2, 0.9, chroma=True,
                hq_sigma=sigma)


@pytest.mark.parametrize("d,a,s,sigma,thsad_scale", [(1, 4, 2, 10.0 / 255, 1.0), (2, 3, 2, 6.0 / 255, 0.5),
                                                     (3, 2, 1, 14.0 / 255, 2.0)])
def test_hq_temporal_confidence_luma(oracle, d, a, s, sigma, thsad_scale):
    """NLMeans-HQ with temporal confidence: each neighbour's 16x16 blocks (step 8) are scored where
    they stand and every temporal weight is scaled by its block's confidence
    (nlmeans/dispatch/motion.rs:554-613, kernels/fused.rs:317-324)."""
    w, h = 136, 80
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 5, seed=60 + d)
    spec = avd.EngineSpec.nlmeans(hq(d, a, s, sigma, confidence=True, thsad_scale=thsad_scale), None,
                                  avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    strength = avd.hq_default_strength(1, d)
    check_group(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, a, s, strength, hq_sigma=sigma,
                hq_confidence=True, thsad_scale=thsad_scale)


def test_hq_temporal_confidence_chroma(oracle):
    """Chroma scores lane 0 (U) of the interleaved ring (stages.rs:110-130)."""
    w, h = 112, 64
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 4, chroma="420", seed=71)
    sigma = 8.0 / 255
    spec = avd.EngineSpec.nlmeans(None, hq(1, 3, 2, sigma, strength=0.8, confidence=True),
                                  avd.Geometry(w, h, avd.ChromaLayout.YUV420, fmt, fmt))
    got = Runner(spec).run(frames)
    check_group(oracle, [[g[1], g[2]] for g in got], [[f[1], f[2]] for f in frames], fmt, 1, 3, 2, 0.8, chroma=True,
                hq_sigma=sigma, hq_confidence=True)


def test_exp_mirror_matches_oracle_bit_for_bit(lib, oracle):
    """The exponential of the exact finish and the bilateral prefilter (exp_mirror.cuh) equals the
    oracle's restatement bit for bit over the weights' whole range (a fused multiply-add rounds
    once on both sides)."""
    import torch

    x = np.concatenate([np.linspace(-90.0, 0.0, 3_000_001, dtype=np.float32),
                        -np.geomspace(1e-9, 1.0, 200_001).astype(np.float32),
                        np.linspace(0.0, 88.0, 100_001, dtype=np.float32),
                        np.array([0.0, -0.0, -87.0, -87.00001, np.nan], np.float32)])
    dx = torch.from_numpy(x).cuda()
    dy = torch.empty_like(dx)
    assert lib.avd_exp_mirror(dx.data_ptr(), dy.data_ptr(), x.size, None) == 0
    torch.cuda.synchronize()
    got = dy.cpu().numpy()
    want = oracle.exp_mirror(x)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_one_engine_runs_chroma_beside_luma():
    """One engine cleaning luma and chroma runs each push's chroma pass on a second stream beside the
    luma pass (it reads nothing the luma pass writes): every output plane equals, bit for bit, what a
    luma-only engine and a chroma-only engine give over the same 9 frames of 4:2:0 u8."""
    w, h = 256, 144
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 9, chroma="420", seed=41)
    geo = avd.Geometry(w, h, avd.ChromaLayout.YUV420, fmt, fmt)
    both = Runner(avd.EngineSpec.nlmeans(nlm(1, 5, 2, 8.0), nlm(1, 5, 2, 5.0), geo)).run(frames)
    luma = Runner(avd.EngineSpec.nlmeans(nlm(1, 5, 2, 8.0), None, geo)).run(frames)
    chroma = Runner(avd.EngineSpec.nlmeans(None, nlm(1, 5, 2, 5.0), geo)).run(frames)
    assert len(both) == len(luma) == len(chroma) == 9
    for b, l, c in zip(both, luma, chroma):
        assert np.array_equal(b[0], l[0])
        assert np.array_equal(b[1], c[1]) and np.array_equal(b[2], c[2])
