"""NL4D with the automatic noise estimate (luma, no sigma) on the GPU through the C ABI against the
oracle's stream restatement: the 8-frame look-ahead searches each frame against the one before it,
reads the noise along that motion (the first frame again along the motion to the second), and every
pass folds the window around its centre frame into the sigma, weight scale and motion SAD floor it
filters with (nlmeans/denoiser/lookahead.rs, nl4d/denoiser.rs, noise/*). With the noise map on (the
default) the readings carry the luma noise curve and each pass scales its luma threshold by the
folded curve at the reference patch's mean luma (collab/kernels/fused/mod.rs:617-660).

Every stage is bit-exact, so every output sample is identical to the oracle's."""

import numpy as np
import pytest

from conftest import avd
from gpu_util import Runner
from test_gpu_nl4d import check, clip

pytestmark = pytest.mark.gpu


def auto_noise(oracle, frames, fmt, d, *, blksize=16, overlap=8, search_radius=4, levels=2, sigma_scale=1.0,
               noise_map=False):
    """The per-pass (sigma, weight scale, SAD floor, curve) of the measured front, by centre frame;
    the curve is None unless the noise map is on and the fold's curve flag is set."""
    f32 = [oracle.ingest(p, fmt.kind, fmt.max_value(), 0.0) for p in frames]
    h, w, c = f32[0].shape
    readings, totals = oracle.noise_readings_mc(f32, c, w, h, blksize=blksize, overlap=overlap,
                                                search_radius=search_radius, levels=levels, luma_fields=noise_map)
    f = np.float32
    area, unit = f(81.0), f(1.2) * f(1.0) * f(255.0)
    settings = oracle.fold_words(w, h, sigma_scale=sigma_scale, curve_applies=noise_map,
                                 g_max=float(oracle.dct_noise_profile(0.0).max()),
                                 h2_per_inverse_variance=float(f(65025.0) / (f(3.0) * unit * unit * area)),
                                 h2_fixed=float(f(65025.0) / (f(3.0) * f(1.2) * f(1.2) * area)),
                                 offset_per_variance=float(f(2.0) * f(3.0) * f(1.0) * area),
                                 sad_per_sigma=oracle.sad_noise_floor(blksize, 1.0))
    folds = oracle.fold_stream(readings, totals, settings, c, 0, d)
    derived = [fd[1] for fd in folds]
    curves = [fd[0][16:32].copy() if fd[1][3] != 0 else None for fd in folds]
    return (lambda frame: (float(derived[frame][0]), float(derived[frame][2]), float(derived[frame][4]),
                           curves[frame])), derived, curves


@pytest.mark.parametrize("w,h,n,d,estimation,context", [
    (96, 64, 12, 2, avd.MotionEstimation.DIRECT, 0),
    (96, 64, 14, 3, avd.MotionEstimation.AUTO, 0),    # Chained at d >= 3
    (80, 48, 5, 2, avd.MotionEstimation.DIRECT, 0),   # shorter than the look-ahead
    (72, 56, 11, 1, avd.MotionEstimation.DIRECT, 2),  # continuation
    (88, 40, 20, 2, avd.MotionEstimation.CHAINED, 0),  # the history wraps
])
def test_nl4d_auto_sigma_matches_oracle(oracle, w, h, n, d, estimation, context):
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, n, seed=w + n + d, sigma=9.0)
    o = avd.Nl4dOptions(sigma=None, noise_map=False, temporal_radius=d, spatial_radius=4,
                        motion=avd.MotionSearch(estimation=estimation))
    spec = avd.EngineSpec.nl4d(o, None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    assert spec.max_held_frames() == 2 * d + 8
    got = Runner(spec).run(frames, context=context)
    noise, derived, _ = auto_noise(oracle, [[f[0]] for f in frames], fmt, d)
    chained = estimation == avd.MotionEstimation.CHAINED or (estimation == avd.MotionEstimation.AUTO and d >= 3)
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, 0.0, context=context, spatial_radius=4,
          chained=chained, noise=noise)
    # Along the motion the estimate finds the synthetic 9-code noise.
    sig = derived[n // 2][0] * 255
    assert 6.5 < sig < 11.0, sig


def test_nl4d_auto_10bit_sigma_scale(oracle):
    w, h, n, d = 96, 64, 10, 1
    fmt = avd.SampleFormat.u16(10)
    frames = clip(w, h, n, depth=10, seed=77, sigma=12.0)
    o = avd.Nl4dOptions(sigma=None, noise_map=False, sigma_scale=1.2, temporal_radius=d, spatial_radius=3,
                        pooled_threshold=False, lambda_ht=2.7)
    spec = avd.EngineSpec.nl4d(o, None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    noise, _, _ = auto_noise(oracle, [[f[0]] for f in frames], fmt, d, sigma_scale=1.2)
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, 0.0, spatial_radius=3, noise=noise,
          pooled_threshold=False, lambda_ht=2.7)


def graded_clip(w, h, n, seed):
    """A luma clip panning 2 pixels a frame over a smooth horizontal ramp whose grain grows with
    brightness (3 to 6 codes), so the reading finds a rising noise curve."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w + 4 * n].astype(np.float32)
    ramp = 0.06 + 0.88 * x / (w + 4 * n)
    frames = []
    for i in range(n):
        base = ramp[:, 2 * i:2 * i + w]
        grain = rng.normal(0, 1, base.shape) * (3.0 + 3.0 * base) / 255.0
        frames.append([np.clip(np.rint((base + grain) * 255), 0, 255).astype(np.uint8)])
    return frames


@pytest.mark.parametrize("w,h,n,d,estimation", [
    (384, 224, 12, 2, avd.MotionEstimation.DIRECT),
    (352, 208, 14, 3, avd.MotionEstimation.AUTO),
    (384, 224, 6, 1, avd.MotionEstimation.DIRECT),   # shorter than the look-ahead
])
def test_nl4d_auto_noise_map_matches_oracle(oracle, w, h, n, d, estimation):
    """The default NL4D call on gray frames (automatic sigma, noise map on): identical samples."""
    fmt = avd.SampleFormat.u8()
    frames = graded_clip(w, h, n, seed=w + n)
    o = avd.Nl4dOptions(sigma=None, temporal_radius=d, spatial_radius=4,
                        motion=avd.MotionSearch(estimation=estimation))
    assert o.noise_map
    spec = avd.EngineSpec.nl4d(o, None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    noise, _, curves = auto_noise(oracle, [f for f in frames], fmt, d, noise_map=True)
    chained = estimation == avd.MotionEstimation.AUTO and d >= 3
    check(oracle, [[g[0]] for g in got], frames, fmt, d, 0.0, spatial_radius=4, chained=chained, noise=noise)
    # The brighter side of the ramp carries more grain: every pass's folded curve rises.
    assert all(c is not None for c in curves), "a pass folded no curve"
    assert all(c[12] > 1.3 * c[2] for c in curves)


def pack_plane(codes):
    """A u8 plane as the engine's word-packed layout."""
    flat = np.asarray(codes, np.uint8).reshape(-1)
    return np.concatenate([flat, np.zeros((-len(flat)) % 4, np.uint8)]).view(np.uint32)


def colour_noise(oracle, clip_frames, fmt, d, luma, *, blksize=16, overlap=8, search_radius=4, levels=2):
    """The measured front of a luma (`luma`) or chroma NL4D pass over a 4:2:0 u8 clip with its colour
    grain gains: per centre frame (sigma, weight scale, SAD floor, curve, colour), as the engine
    pools each reading into its frame's cell sums and fits the window at each fold
    (noise/colour.rs:733-827, nl4d/collab_pass.rs:71-75)."""
    planes = [f[0:1] if luma else f[1:3] for f in clip_frames]
    f32 = [oracle.ingest(p, fmt.kind, fmt.max_value(), 0.0) for p in planes]
    h, w, c = f32[0].shape
    H, W = clip_frames[0][0].shape
    means = [oracle.colour_means(pack_plane(f[0]), pack_plane(f[1]), pack_plane(f[2]), W, H, 1, 1, 4, False, 1.0, 0.0)
             for f in clip_frames]
    grid = [m[0] if luma else m[1] for m in means]
    records = []
    # A chroma pass refines the luma pass's motion and fits no camera models of its own.
    readings, totals = oracle.noise_readings_mc(f32, c, w, h, blksize=blksize, overlap=overlap,
                                                search_radius=search_radius, levels=levels, luma_fields=luma,
                                                records_out=records, camera_model=luma)
    f = np.float32
    area, unit = f(81.0), f(1.2) * f(1.0) * f(255.0)
    settings = oracle.fold_words(w, h, curve_applies=luma, g_max=float(oracle.dct_noise_profile(0.0).max()),
                                 h2_per_inverse_variance=float(f(65025.0) / (f(3.0) * unit * unit * area)),
                                 h2_fixed=float(f(65025.0) / (f(3.0) * f(1.2) * f(1.2) * area)),
                                 offset_per_variance=float(f(2.0) * (f(3.0) if luma else f(1.5)) * f(1.0) * area),
                                 sad_per_sigma=oracle.sad_noise_floor(blksize, 1.0))
    folds = oracle.fold_stream(readings, totals, settings, c, 0, d)
    cap = 2 * 8 + 1 + d
    cells = [oracle.colour_accumulate(r, g, w, h, c, luma, 255.0) for r, g in zip(records, grid)]
    ring = np.zeros((cap, len(cells[0])), np.int32)
    out = []
    for centre in range(len(clip_frames)):
        first, last = oracle.noise_window(centre, len(clip_frames) - 1)
        for fr in range(first, last + 1):
            ring[fr % cap] = cells[fr]
        window = oracle.colour_window(ring, cap, first, last)
        state, derived = folds[centre][0], folds[centre][1]
        _, gains, _ = oracle.colour_fit(window, c, luma, state[16:32], bool(derived[3]))
        curve = state[16:32].copy() if derived[3] != 0 else None
        sigma = float(derived[0]) if c == 1 else (float(derived[0]), float(derived[1]))
        out.append((sigma, float(derived[2]), float(derived[4]), curve, (gains, grid[centre], 255.0)))
    return (lambda frame: out[frame]), out


def colour_clip(w, h, n, seed):
    """A 4:2:0 u8 clip panning 2 pixels a frame over coloured bands whose luma grain grows with
    warmth (Cr above Cb) and brightness, Cb grain with Cb and Cr grain as Cr falls, so the colour
    gains move away from 1."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w + 4 * n].astype(np.float32)
    luma = 40 + 170 * x / (w + 4 * n)
    cb = 128 + 45 * np.sin(y / 23.0)
    cr = 128 + 45 * np.cos(x / 31.0 + y / 47.0)
    frames = []
    for i in range(n):
        sl = slice(2 * i, 2 * i + w)
        lb, cbb, crb = luma[:, sl], cb[:, sl], cr[:, sl]
        warm = np.clip((crb - cbb) / 40.0, 0, None)
        grain = (2.0 + lb / 80.0) * (1.0 + warm)
        yp = np.clip(np.rint(lb + rng.normal(0, 1, lb.shape) * grain), 0, 255).astype(np.uint8)
        cb2, cr2 = cbb[::2, ::2], crb[::2, ::2]
        ugrain = 1.0 + 2.5 * np.clip((cb2 - 128) / 45.0, 0, None)
        vgrain = 1.0 + 2.5 * np.clip((128 - cr2) / 45.0, 0, None)
        up = np.clip(np.rint(cb2 + rng.normal(0, 1, cb2.shape) * ugrain), 0, 255).astype(np.uint8)
        vp = np.clip(np.rint(cr2 + rng.normal(0, 1, cr2.shape) * vgrain), 0, 255).astype(np.uint8)
        frames.append([yp, up, vp])
    return frames


@pytest.mark.parametrize("w,h,n,d", [(256, 192, 10, 2), (224, 160, 6, 1)])
def test_nl4d_auto_noise_map_with_colour_gains_matches_oracle(oracle, w, h, n, d):
    """The default NL4D call on 4:2:0 frames (automatic sigma, noise map on): the luma pass scales
    its threshold by the noise curve and the colour grain gains; identical samples."""
    fmt = avd.SampleFormat.u8()
    frames = colour_clip(w, h, n, seed=w + n)
    o = avd.Nl4dOptions(sigma=None, temporal_radius=d, spatial_radius=4,
                        motion=avd.MotionSearch(estimation=avd.MotionEstimation.DIRECT))
    spec = avd.EngineSpec.nl4d(o, None, avd.Geometry(w, h, avd.ChromaLayout.YUV420, fmt, fmt))
    got = Runner(spec).run(frames)
    noise, per_pass = colour_noise(oracle, frames, fmt, d, True)
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, 0.0, spatial_radius=4, noise=noise)
    for g, src in zip(got, frames):
        assert np.array_equal(g[1], src[1]) and np.array_equal(g[2], src[2])
    # The gains moved off 1 somewhere once the window held enough blocks.
    assert any(np.abs(p[4][0]).max() > 0.01 for p in per_pass)


@pytest.mark.parametrize("d", [1, 2])
def test_nl4d_chroma_auto_sigma_with_colour_gains_matches_oracle(oracle, d):
    """A chroma-only engine with the automatic estimate: the luma guide measures its own noise for
    its motion search, and the chroma pass measures both chroma channels, pools them into colour
    cells on the chroma grid and scales each channel's threshold by its gain; identical samples."""
    w, h, n = 192, 128, 8
    fmt = avd.SampleFormat.u8()
    frames = colour_clip(w, h, n, seed=77 + d)
    o = avd.Nl4dOptions(sigma=None, temporal_radius=d, spatial_radius=4,
                        motion=avd.MotionSearch(estimation=avd.MotionEstimation.DIRECT))
    spec = avd.EngineSpec.nl4d(None, o, avd.Geometry(w, h, avd.ChromaLayout.YUV420, fmt, fmt))
    got = Runner(spec).run(frames)
    for g, f in zip(got, frames):
        assert np.array_equal(g[0], f[0])
    share = oracle.MotionShare((w // 8, h // 8, 8, 16), (w // 16, h // 16, 8, 16), 1, 1)
    guide_noise, _, _ = auto_noise(oracle, [[f[0]] for f in frames], fmt, d)
    f32 = [oracle.ingest([f[0]], fmt.kind, fmt.max_value(), 0.0) for f in frames]
    oracle.nl4d_stream(f32, d, 0.0, spatial_radius=4, share_writes=share, noise=guide_noise)
    noise, per_pass = colour_noise(oracle, frames, fmt, d, False)
    check(oracle, [[g[1], g[2]] for g in got], [[f[1], f[2]] for f in frames], fmt, d, 0.0, chroma=True,
          spatial_radius=4, share_reads=share, noise=noise)
    assert all(p[0][0] > 0 and p[0][1] > 0 for p in per_pass)
    assert any(np.abs(p[4][0]).max() > 0.01 for p in per_pass)
