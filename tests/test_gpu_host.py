"""The host denoiser (av-denoise/src/host/mod.rs:111-420) on the GPU: frames pushed as wire bytes
come back identical to the same clip pushed through the device engine, and meet the NLMeans parity
bar against the oracle directly; the queue, plane-check, poison and reset rules behave as the
reference's host tests expect (host/tests)."""

import numpy as np
import pytest

from conftest import avd
from gpu_util import Parity, Runner, oracle_pass

pytestmark = pytest.mark.gpu


def clip(w, h, n, depth=8, chroma="gray", seed=0):
    from av_denoise_b200 import synth

    return synth.make_clip(w, h, n, depth=depth, chroma=chroma, sigma_luma=10.0, sigma_chroma=6.0,
                           global_motion=2, sprites=1, sprite_size=24, seed=seed)


def wire(frame, fmt):
    dt = {0: np.uint8, 1: "<u2", 2: "<f4"}[fmt.kind]
    return [np.ascontiguousarray(p.astype(dt)).tobytes() for p in frame]


def unwire(planes, fmt, dims):
    dt = {0: np.uint8, 1: "<u2", 2: "<f4"}[fmt.kind]
    return [np.frombuffer(b, dtype=dt).reshape(h, w) for b, (w, h) in zip(planes, dims)]


def nlm_spec(w, h, d=2, chroma=avd.ChromaLayout.GRAY, fmt=None):
    fmt = fmt or avd.SampleFormat.u8()
    tuning = avd.NlmTuning(search_radius=3, patch_radius=2, strength=8.0)
    alg = avd.NlmeansAlgorithm.fast(avd.NlmeansOptions(tuning=tuning, mode=avd.DenoisingMode.temporal(d)))
    chroma_alg = alg if chroma != avd.ChromaLayout.GRAY else None
    return avd.EngineSpec.nlmeans(alg, chroma_alg, avd.Geometry(w, h, chroma, fmt, fmt))


def nl4d_spec(w, h, d=2):
    fmt = avd.SampleFormat.u8()
    o = avd.Nl4dOptions(sigma=10.0 / 255, temporal_radius=d, spatial_radius=5,
                        motion=avd.MotionSearch(estimation=avd.MotionEstimation.DIRECT))
    return avd.EngineSpec.nl4d(o, None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))


def run_host(den, frames, fmt, dims, priming=0):
    """Pushes every frame, collecting as the queue fills (the usage of mod.rs:80-104)."""
    out = []
    for i, f in enumerate(frames):
        planes = wire(f, fmt)
        if i < priming:
            den.push_priming(planes)
            continue
        try:
            den.push(planes)
        except avd.QueueFull:
            out.append(den.recv())
            den.push(planes)
        got = den.recv()
        if got is not None:
            out.append(got)
    den.flush(out.append)
    return [unwire(p, fmt, dims) for p in out]


def assert_same(host_out, engine_out):
    assert len(host_out) == len(engine_out)
    for hf, ef in zip(host_out, engine_out):
        for hp, ep in zip(hf, ef):
            np.testing.assert_array_equal(hp, ep)


@pytest.mark.parametrize("w,h,depth,chroma", [(96, 64, 8, avd.ChromaLayout.GRAY),
                                              (67, 45, 10, avd.ChromaLayout.YUV420),
                                              (33, 20, 8, avd.ChromaLayout.YUV422)])
def test_host_nlm_matches_engine(w, h, depth, chroma):
    fmt = avd.SampleFormat.u8() if depth == 8 else avd.SampleFormat.u16(depth)
    name = {avd.ChromaLayout.GRAY: "gray", avd.ChromaLayout.YUV420: "420", avd.ChromaLayout.YUV422: "422"}[chroma]
    frames = clip(w, h, 7, depth=depth, chroma=name, seed=w)
    spec = nlm_spec(w, h, chroma=chroma, fmt=fmt)
    want = Runner(spec).run(frames)
    g = spec.geometry
    dims = [g.plane_dims(i) for i in range(g.plane_count())]
    with avd.HostDenoiser(spec) as den:
        assert den.plane_lengths == [len(b) for b in wire(frames[0], fmt)]
        got = run_host(den, frames, fmt, dims)
    assert_same(got, want)


@pytest.mark.parametrize("w,h,depth", [(96, 64, 8), (67, 45, 10)])
def test_host_nlm_matches_oracle(oracle, w, h, depth):
    """Wire bytes in, wire bytes out, against the oracle on the same clip: every sample of both
    plane groups identical (raw), none off by more than 1 LSB."""
    fmt = avd.SampleFormat.u8() if depth == 8 else avd.SampleFormat.u16(depth)
    frames = clip(w, h, 7, depth=depth, chroma="420", seed=w + depth)
    spec = nlm_spec(w, h, chroma=avd.ChromaLayout.YUV420, fmt=fmt)
    g = spec.geometry
    dims = [g.plane_dims(i) for i in range(g.plane_count())]
    with avd.HostDenoiser(spec) as den:
        got = run_host(den, frames, fmt, dims)
    want_y = oracle_pass(oracle, [[f[0]] for f in frames], fmt, 2, 3, 2, 8.0)
    want_uv = oracle_pass(oracle, [[f[1], f[2]] for f in frames], fmt, 2, 3, 2, 8.0, chroma=True)
    assert len(got) == len(want_y) == len(frames)
    par = Parity()
    for k in range(len(frames)):
        par.add(got[k][0], want_y[k][0], None, fmt.max_value())
        for c in range(2):
            par.add(got[k][1 + c], want_uv[k][c], None, fmt.max_value())
    st = par.stats()
    assert st["max_lsb"] <= 1 and st["identical"] >= 0.999, st


def test_host_nl4d_priming_matches_engine():
    w, h = 80, 48
    frames = clip(w, h, 8, seed=3)
    spec = nl4d_spec(w, h)
    want = Runner(spec).run(frames, context=2)
    with avd.HostDenoiser(spec) as den:
        got = run_host(den, frames, spec.geometry.input, [(w, h)], priming=2)
    assert_same(got, want)


def test_host_queue_full_and_plane_checks():
    w, h = 64, 32
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 8, seed=9)
    spec = nlm_spec(w, h, d=1)
    want = Runner(spec).run(frames)
    with avd.HostDenoiser(spec) as den:
        assert den.recv() is None
        with pytest.raises(avd.PlaneMismatch):
            den.push([wire(frames[0], fmt)[0][:-1]])
        with pytest.raises(avd.PlaneMismatch):
            den.push(wire(frames[0], fmt) * 2)
        out, i = [], 0
        # Push without collecting until the queue is full; it stays usable (not poisoned).
        while True:
            try:
                den.push(wire(frames[i], fmt))
                i += 1
            except avd.QueueFull:
                break
        assert i == avd.MAX_PENDING + 1  # d = 1: the first frame readies nothing
        with pytest.raises(avd.ContextAfterPush):
            den.push_priming(wire(frames[i], fmt))
        while (got := den.recv()) is not None:
            out.append(got)
        for f in frames[i:]:
            den.push(wire(f, fmt))
            while (got := den.recv()) is not None:
                out.append(got)
        den.flush(out.append)
    assert_same([unwire(p, fmt, [(w, h)]) for p in out], want)


def test_host_poison_and_reset_stream():
    w, h = 48, 40
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 6, seed=4)
    spec = nlm_spec(w, h, d=2)
    want = Runner(spec).run(frames)
    with avd.HostDenoiser(spec) as den:
        den.push(wire(frames[0], fmt))
        den.poison_for_test()
        with pytest.raises(avd.Poisoned):
            den.push(wire(frames[1], fmt))
        with pytest.raises(avd.Poisoned):
            den.recv()
        with pytest.raises(avd.Poisoned):
            den.flush(lambda p: None)
        den.reset_stream()
        first = run_host(den, frames, fmt, [(w, h)])
        # After a flush the denoiser takes a fresh stream with the same result.
        second = run_host(den, frames, fmt, [(w, h)])
    assert_same(first, want)
    assert_same(second, want)


def test_host_flush_sink_error_propagates():
    w, h = 40, 24
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 4, seed=1)
    with avd.HostDenoiser(nlm_spec(w, h, d=1)) as den:
        for f in frames:
            den.push(wire(f, fmt))
            den.recv()

        def sink(_planes):
            raise KeyError("sink")

        with pytest.raises(KeyError):
            den.flush(sink)


def test_host_timing_counts_frames():
    w, h = 64, 48
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, 6, seed=2)
    with avd.HostDenoiser(nlm_spec(w, h, d=1)) as den:
        den.sample_device_time(1)
        run_host(den, frames, fmt, [(w, h)])
        t = den.timing()
    assert t.frames == len(frames)
    assert t.blocked >= 0 and t.submit > 0
    assert t.luma is not None and t.luma > 0
    assert t.chroma is None
