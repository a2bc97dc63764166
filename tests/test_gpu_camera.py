"""The camera model on the GPU through the C ABI, bit for bit against the oracle: the fit on the
fields the reference's fit tests use (with SADs, contrast stats and priors), the composition of pair
models into window predictions, the block means and the high pass, and the block search and the
truemotion stage with the model's second window and their SAD outputs, on frames rendered through a
pan that reaches past the search window."""

import ctypes as C

import numpy as np
import pytest

import test_oracle_camera_model as tc
from camera_cases import render
from motion_cases import moving_window

pytestmark = pytest.mark.gpu


def stream():
    import torch

    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def dev(a, dtype=None):
    import torch

    t = torch.from_numpy(np.ascontiguousarray(a).reshape(-1).copy())
    return (t if dtype is None else t.to(dtype)).cuda()


def host(t):
    import torch

    torch.cuda.synchronize()
    return t.cpu().numpy()


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def gpu_fit(lib, field, *, sad=None, has_contrast=False, older_to_newer=True, prior=None, w=tc.W, h=tc.H,
            blksize=tc.BLK, overlap=tc.OVL):
    import torch

    from av_denoise_b200 import _abi

    ring = np.zeros(2 * 5, np.float32)
    if prior is not None:
        ring[:4] = np.asarray(prior, np.float32)
        ring[4] = 1.0
    step = blksize - overlap
    blocks = max(-(-w // step), 1) * max(-(-h // step), 1)
    f, r = dev(np.asarray(field, np.int32)), dev(ring)
    s = dev(np.asarray(sad, np.float32)) if sad is not None else None
    scratch = torch.full((lib.avd_model_fit_scratch_floats(blocks),), -7.0, device="cuda")
    p = _abi.AvdModelFit()
    p.field, p.sad = f.data_ptr(), s.data_ptr() if s is not None else 0
    p.has_contrast, p.means_offset, p.older_to_newer = int(has_contrast), blocks, int(older_to_newer)
    p.width, p.height, p.blksize, p.overlap = w, h, blksize, overlap
    p.prior, p.models, p.slot, p.scratch = (0 if prior is not None else -1), r.data_ptr(), 1, scratch.data_ptr()
    assert lib.avd_model_fit(C.byref(p), stream()) == 0, lib.avd_last_error().decode()
    return host(r), host(scratch)[:8]


def fit_cases():
    row, col = tc.rows_cols()
    cases = {}
    cam = tc.similarity(2.5, 1.01, 6.0, -4.0)
    cases["roll_zoom_shift"] = dict(field=tc.camera_field(cam))
    cases["backward"] = dict(field=tc.camera_field(tc.inverse(tc.similarity(-1.5, 0.99, -8.0, 3.0))),
                             older_to_newer=False)
    cases["group"] = dict(field=tc.with_group(tc.similarity(1.5, 1.0, 5.0, 2.0)))
    cases["zero"] = dict(field=np.zeros((tc.BLOCKS, 2), np.int32))
    cases["nonsense"] = dict(field=tc.random_field(5))
    f = tc.camera_field(tc.similarity(0.0, 1.0, 5.0, 1.0))
    bar = round(tc.BX * 0.12)
    f[(col < bar) | (col >= tc.BX - bar)] = 0
    cases["pillarbox"] = dict(field=f)
    f, in_layer = tc.layer_between_bands()
    black = (1.0, 1.24, np.float32(18.0) / np.float32(255.0))
    cases["bars_with_stats"] = dict(field=f, sad=tc.stats_sad(lambda r: tc.DETAILED if in_layer(r) else black),
                                    has_contrast=True)
    f = tc.camera_field(tc.similarity(1.0, 1.0, 9.0, -3.0))
    rng = np.random.default_rng(33)
    grain = (tc.oracle.thsad(16, 1.0) * (3.0 + 2.0 * rng.random(tc.BLOCKS))).astype(np.float32)
    f[col >= 60] = (10, -8)
    cases["grain_sads"] = dict(field=f, sad=np.where(col >= 60, 3.0 * grain, grain).astype(np.float32))
    f = tc.camera_field(tc.similarity(1.0, 1.0, 9.0, -3.0))
    f[col >= 48] = (10, -8)
    cases["valid_prior"] = dict(field=f, prior=tc.similarity(1.1, 1.0, 8.5, -3.0))
    cases["stale_prior"] = dict(field=tc.with_group(tc.similarity(-1.0, 1.0, -3.0, 2.0)),
                                prior=tc.similarity(4.0, 1.0, 30.0, 0.0))
    return cases


CASES = fit_cases()


@pytest.mark.parametrize("name", list(CASES))
def test_model_fit_matches_oracle(lib, oracle, name):
    kw = CASES[name]
    got, state = gpu_fit(lib, **kw)
    ring = np.zeros(10, np.float32)
    if kw.get("prior") is not None:
        ring[:4] = np.asarray(kw["prior"], np.float32)
        ring[4] = 1.0
    want, want_state = oracle.model_fit(kw["field"], tc.W, tc.H, tc.BLK, tc.OVL, sad=kw.get("sad"),
                                        has_contrast=kw.get("has_contrast", False),
                                        older_to_newer=kw.get("older_to_newer", True), models=ring, slot=1,
                                        prior=0 if kw.get("prior") is not None else None)
    assert np.array_equal(bits(got), bits(want)), (got, want)
    # State words 0..6: the mean SAD, the reference model and the scale limit (word 7 is unused).
    assert np.array_equal(bits(state[:7]), bits(want_state[:7])), (state, want_state)


def test_model_fit_on_odd_grids(lib, oracle):
    """Grids whose last blocks reach past the frame and whose count is not a multiple of 256."""
    for (w, h, blk, ovl) in [(333, 191, 8, 4), (250, 130, 32, 16), (97, 61, 16, 0)]:
        step = blk - ovl
        bx, by = -(-w // step), -(-h // step)
        col, row = np.arange(bx * by) % bx, np.arange(bx * by) // bx
        field = np.stack([np.full(bx * by, 3), np.where(row > by // 2, -2, -1)], 1).astype(np.int32)
        field[(col % 7) == 3] = (-5, 4)
        rng = np.random.default_rng(w)
        sad = rng.random(3 * bx * by).astype(np.float32)
        got, state = gpu_fit(lib, field, sad=sad, has_contrast=True, w=w, h=h, blksize=blk, overlap=ovl)
        want, want_state = oracle.model_fit(field, w, h, blk, ovl, sad=sad, has_contrast=True,
                                            models=np.zeros(10, np.float32), slot=1)
        assert np.array_equal(bits(got), bits(want)) and np.array_equal(bits(state[:7]), bits(want_state[:7])), (w, h)


def test_compose_matches_oracle(lib, oracle):
    import torch

    rng = np.random.default_rng(3)
    depth = 9
    ring = np.zeros(depth * 5, np.float32)
    for s in range(depth):
        a, b, tx, ty = tc.similarity(rng.uniform(-3, 3), rng.uniform(0.95, 1.05), rng.uniform(-20, 20),
                                     rng.uniform(-20, 20))
        ring[s * 5:s * 5 + 5] = (a, b, tx, ty, 0.0 if s == 4 else 1.0)
    for frames, centre in [([10, 11, 12, 13, 14], 2), ([3, 3, 3, 4, 5], 1), ([20, 21, 22, 23, 24, 25, 26], 3),
                           ([7, 8, 9, 9, 9], 2)]:
        nb = len(frames) - 1
        gaps = oracle.compose_gaps(frames, centre, nb, lambda f: f % depth)
        want = oracle.compose_models(ring, gaps, nb, nb, centre)
        out = torch.full((nb * 6,), -1.0, device="cuda")
        g = dev(gaps.view(np.int32))
        assert lib.avd_compose_models(dev(ring).data_ptr(), g.data_ptr(), out.data_ptr(), nb, nb, centre, stream()) == 0
        assert np.array_equal(bits(host(out)), bits(want)), frames


@pytest.mark.parametrize("w,h,blk,ovl", [(160, 90, 16, 8), (123, 77, 8, 4), (64, 40, 32, 16)])
def test_block_means_and_high_pass_match_oracle(lib, oracle, w, h, blk, ovl):
    import torch

    plane = render((1.0, 0.0, 3.3, -1.2), w, h)
    step = blk - ovl
    nb = max(-(-w // step), 1) * max(-(-h // step), 1)
    means = torch.full((nb,), -1.0, device="cuda")
    p = dev(plane)
    assert lib.avd_block_means(p.data_ptr(), means.data_ptr(), w, h, blk, ovl, stream()) == 0
    assert np.array_equal(bits(host(means)), bits(oracle.block_means(plane, w, h, blk, step)))
    rows, out = torch.zeros(w * h, device="cuda"), torch.zeros(w * h, device="cuda")
    assert lib.avd_high_pass(p.data_ptr(), rows.data_ptr(), out.data_ptr(), w, h, 8, stream()) == 0
    assert np.array_equal(bits(host(out)), bits(oracle.high_pass(plane, w, h)))


# ---- the search and truemotion stage with the model's window ----------------------------------------

def panned_ring(w, h, frames, velocity, seed=0):
    """Frames of the texture panned `velocity` px per frame, with a little grain."""
    rng = np.random.default_rng(seed)
    out = [render((1.0, 0.0, velocity[0] * f, velocity[1] * f), w, h) + rng.normal(0, 0.01, (h, w)).astype(np.float32)
           for f in range(frames)]
    return np.stack(out).astype(np.float32)


def predictions_for(neighbours, velocity, centre, slots, jitter=0.0):
    """The prediction of each neighbour slot s of a pan: (1, 0, 0, 1, v * (s - centre))."""
    p = np.zeros((len(slots), 6), np.float32)
    for i, s in enumerate(slots):
        p[i] = (1.0, -0.0, 0.0, 1.0, velocity[0] * (s - centre) + jitter, velocity[1] * (s - centre) - jitter)
    return p


def gpu_search(lib, pyr, w, h, frames, centre, slots, *, blksize, overlap, radius, levels, predictions, floor,
               thsad, ceiling=0, esc_reads_floor=False, coarse_radius=0, factor=1, seeds=None, keep=False):
    import torch

    from av_denoise_b200 import _abi

    step = blksize - overlap
    bx, by = max(-(-w // step), 1), max(-(-h // step), 1)
    n = len(slots)
    slots_t = torch.tensor(np.asarray(slots, np.int32), device="cuda")
    mv = torch.zeros(n * bx * by * 2, dtype=torch.int32, device="cuda") if seeds is None else dev(seeds)
    sad = torch.full((2 * n * bx * by,), -1.0, device="cuda")
    noise = torch.tensor([floor], dtype=torch.float32, device="cuda")
    pr = dev(predictions) if predictions is not None else None
    kept = torch.zeros_like(mv) if keep else None
    p = _abi.AvdMotionPass()
    p.pyramid, p.neighbour_slots, p.mv_field, p.noise = pyr.data_ptr(), slots_t.data_ptr(), mv.data_ptr(), noise.data_ptr()
    p.width, p.height, p.frame_count, p.centre_slot, p.neighbours = w, h, frames, centre, n
    p.blksize, p.overlap, p.search_radius, p.levels = blksize, overlap, radius, levels
    p.mv_stride, p.conf_stride, p.sad_floor_word, p.thsad = bx * by * 2, bx * by, 0, thsad
    p.seeded = int(seeds is not None)
    p.keep_seeds = kept.data_ptr() if keep else 0
    p.predictions = pr.data_ptr() if pr is not None else 0
    p.sad, p.coarse_radius, p.coarse_block_factor = sad.data_ptr(), coarse_radius, factor
    if ceiling:
        state = torch.zeros(lib.avd_escalation_state_floats(n, bx * by), dtype=torch.float32, device="cuda")
        p.escalation, p.ceiling, p.esc_reads_floor = state.data_ptr(), ceiling, int(esc_reads_floor)
    assert lib.avd_motion_search(C.byref(p), stream()) == 0, lib.avd_last_error().decode()
    return host(mv).reshape(n, bx * by, 2), host(sad), (host(kept) if keep else None)


SEARCH_CASES = [
    # w, h, frames, levels, blksize, overlap, radius, velocity, ceiling, coarse_radius, factor
    (192, 128, 3, 2, 16, 8, 4, (14, -6), 0, 0, 1),
    (192, 128, 5, 1, 16, 8, 3, (11, 4), 0, 0, 1),
    (160, 96, 3, 2, 8, 4, 2, (9, 9), 0, 0, 1),
    (200, 120, 3, 2, 32, 16, 4, (-17, 5), 0, 0, 1),
    (150, 90, 3, 2, 12, 6, 3, (13, -2), 0, 0, 1),       # the generic kernels
    (192, 128, 3, 2, 16, 8, 2, (12, 7), 6, 0, 1),       # escalation with the coarse level widened
    (240, 136, 3, 3, 16, 8, 4, (30, -3), 0, 12, 2),     # the deep acquisition search
    (240, 136, 3, 3, 8, 4, 4, (26, 2), 0, 12, 2),       # its generic coarse kernel (4 x 4 coarse blocks)
    (192, 128, 3, 1, 16, 8, 0, (7, 0), 0, 0, 1),        # radius 0, one level
]


@pytest.mark.parametrize("case", SEARCH_CASES, ids=lambda c: "_".join(map(str, c[:7])) + f"_c{c[8]}_r{c[9]}")
@pytest.mark.parametrize("floor", [0.0, 40.0])
def test_search_with_the_model_window_matches_oracle(lib, oracle, case, floor):
    import torch

    w, h, frames, levels, blksize, overlap, radius, vel, ceiling, crad, factor = case
    ring = panned_ring(w, h, frames, vel, seed=w + radius)
    o_pyr = oracle.motion_pyramid(ring.reshape(-1), 1, w, h, levels)
    centre = frames // 2
    slots = [s for s in range(frames) if s != centre]
    pred = predictions_for(len(slots), vel, centre, slots, jitter=0.3)
    th = oracle.thsad(blksize, 1.0)
    step = blksize - overlap
    n, blocks = len(slots), max(-(-w // step), 1) * max(-(-h // step), 1)
    want_sad = np.full(2 * n * blocks, -1.0, np.float32)
    want, _ = oracle.motion_search(o_pyr, w, h, frames, centre, slots, blksize=blksize, overlap=overlap,
                                   search_radius=radius, levels=levels, sad_floor=floor, thsad=th, ceiling=ceiling,
                                   predictions=pred, sad_out=want_sad, coarse_radius=crad or None,
                                   coarse_block_factor=factor)
    got, sad, _ = gpu_search(lib, torch.from_numpy(o_pyr).cuda(), w, h, frames, centre, slots, blksize=blksize,
                             overlap=overlap, radius=radius, levels=levels, predictions=pred, floor=floor, thsad=th,
                             ceiling=ceiling, coarse_radius=crad, factor=factor)
    assert np.array_equal(got, want), np.argwhere(got != want)[:5]
    assert np.array_equal(bits(sad), bits(want_sad))
    # The premise: the pan lies past the window, and the model's window found it (a floor of 40
    # biases most blocks back to the first window).
    if floor == 0.0:
        assert np.mean(np.all(got[0] == np.asarray(vel) * (slots[0] - centre), axis=1)) > 0.5


def test_truemotion_with_the_model_candidate_matches_oracle(lib, oracle):
    import torch

    from av_denoise_b200 import _abi

    w, h, frames, blksize, overlap = 192, 128, 3, 16, 8
    vel = (13, -5)
    ring = panned_ring(w, h, frames, vel, seed=9)
    o_pyr = oracle.motion_pyramid(ring.reshape(-1), 1, w, h, 2)
    centre, slots = 1, [0, 2]
    pred = predictions_for(2, vel, centre, slots)
    step = blksize - overlap
    bx, by = -(-w // step), -(-h // step)
    rng = np.random.default_rng(1)
    mv_in = rng.integers(-4, 5, (2, bx * by, 2)).astype(np.int32)
    th = oracle.thsad(blksize, 1.0)
    want_sad = np.full(2 * bx * by, -1.0, np.float32)
    want, _ = oracle.truemotion_pass(o_pyr, w, h, frames, centre, slots, mv_in, None, blksize=blksize,
                                     overlap=overlap, field_lambda=1.0, thsad=th, sad_floor=0.0, reads_floor=False,
                                     predictions=pred, sad_out=want_sad)
    pyr = torch.from_numpy(o_pyr).cuda()
    slots_t = torch.tensor(slots, dtype=torch.int32, device="cuda")
    mi, mo = dev(mv_in), torch.zeros(2 * bx * by * 2, dtype=torch.int32, device="cuda")
    sad = torch.full((2 * bx * by,), -1.0, device="cuda")
    noise = torch.zeros(1, device="cuda")
    pr = dev(pred)
    t = _abi.AvdTruemotionPass()
    t.pyramid, t.neighbour_slots, t.mv_in, t.mv_out, t.noise = (pyr.data_ptr(), slots_t.data_ptr(), mi.data_ptr(),
                                                                 mo.data_ptr(), noise.data_ptr())
    t.width, t.height, t.frame_count, t.centre_slot, t.neighbours = w, h, frames, centre, 2
    t.blksize, t.overlap, t.mv_stride, t.conf_stride, t.sad_field, t.reads_floor = blksize, overlap, bx * by * 2, bx * by, 0, 0
    t.field_lambda, t.thsad, t.predictions, t.sad = 1.0, th, pr.data_ptr(), sad.data_ptr()
    assert lib.avd_truemotion_pass(C.byref(t), stream()) == 0, lib.avd_last_error().decode()
    assert np.array_equal(host(mo).reshape(2, -1, 2), want)
    assert np.array_equal(bits(host(sad)), bits(want_sad))
    assert np.mean(np.all(want[1] == np.asarray(vel), axis=1)) > 0.5, "premise: the model's point wins"


def test_search_without_a_model_is_unchanged(lib, oracle):
    """No predictions: the SAD outputs come with the plain search, whose vectors the older tests pin."""
    import torch

    w, h, frames = 160, 96, 5
    ring = moving_window(w, h, frames, seed=3)
    o_pyr = oracle.motion_pyramid(ring, 1, w, h, 2)
    slots = [0, 1, 3, 4]
    want_sad = np.zeros(2 * 4 * 20 * 12, np.float32)
    want, _ = oracle.motion_search(o_pyr, w, h, frames, 2, slots, blksize=16, overlap=8, search_radius=4, levels=2,
                                   sad_floor=0.5, thsad=oracle.thsad(16, 1.0), ceiling=8, sad_out=want_sad)
    got, sad, _ = gpu_search(lib, torch.from_numpy(o_pyr).cuda(), w, h, frames, 2, slots, blksize=16, overlap=8,
                             radius=4, levels=2, predictions=None, floor=0.5, thsad=oracle.thsad(16, 1.0), ceiling=8)
    assert np.array_equal(got, want)
    assert np.array_equal(bits(sad), bits(want_sad))


# ---- the engine's producer ----------------------------------------------------------------------------

def pan_clip(w, h, n, velocity, seed):
    rng = np.random.default_rng(seed)
    out = []
    for f in range(n):
        v = render((1.0, 0.0, velocity[0] * f, velocity[1] * f), w, h) * 200.0 + 20.0
        out.append([np.clip(np.round(v + rng.normal(0, 3.0, (h, w))), 0, 255).astype(np.uint8)])
    return out


@pytest.mark.parametrize("d,estimation,velocity", [(1, "DIRECT", (21, -4)), (2, "CHAINED", (-18, 6))])
def test_engine_fits_the_oracle_camera_models(oracle, d, estimation, velocity):
    """An NLMeans engine with motion compensation fits one model per pushed frame pair, bit for bit
    the oracle's producer fed the same normalised luma, and recovers the pan."""
    from conftest import avd
    from gpu_util import Runner
    from test_gpu_nlm_mc import options, search

    w, h, n = 256, 144, 6
    fmt = avd.SampleFormat.u8()
    frames = pan_clip(w, h, n, velocity, seed=d)
    ms = search(getattr(avd.MotionEstimation, estimation))
    spec = avd.EngineSpec.nlmeans(avd.NlmeansAlgorithm.fast(options(d, 2, 1, 8.0, ms)), None,
                                  avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    r = Runner(spec)
    pm = oracle.PairModels(w, h)
    keep = []
    for i, frame in enumerate(frames):
        bufs, planes = r.planes_for(frame, fmt)
        keep.append(bufs)
        for _ in range(r.engine.push(planes)):
            r.emit()
        pm.push(oracle.ingest([frame[0]], fmt.kind, fmt.max_value())[..., 0], i)
        ring = r.engine.camera_models()
        assert ring is not None and ring.shape[0] == r.engine.max_held_frames() + 2 * d + 1 + 2
        got = ring[i % ring.shape[0]]
        assert np.array_equal(bits(got), bits(pm.model(i))), (i, got, pm.model(i))
        if i > 0:
            assert got[4] == 1.0 and abs(got[2] - velocity[0]) < 0.5 and abs(got[3] - velocity[1]) < 0.5, got


def _moved_share(oracle, frames, fmt, d, ms, **kw):
    """How many output samples the camera model moves: the oracle with and without it."""
    f32 = [oracle.ingest(p, fmt.kind, fmt.max_value(), 0.0) for p in frames]
    with_model = oracle.nlm_stream_mc(f32, d, 2, 1, oracle.h2_inv_norm(8.0, 1), blksize=ms.blksize,
                                      overlap=ms.overlap, search_radius=ms.search_radius, levels=ms.pyramid_levels,
                                      thsad_scale=1.0, **kw)
    without = oracle.nlm_stream_mc(f32, d, 2, 1, oracle.h2_inv_norm(8.0, 1), blksize=ms.blksize,
                                   overlap=ms.overlap, search_radius=ms.search_radius, levels=ms.pyramid_levels,
                                   thsad_scale=1.0, camera_model=False, **kw)
    return float(np.mean([np.mean(a != b) for a, b in zip(with_model, without)]))


@pytest.mark.parametrize("d,estimation", [(2, "DIRECT"), (3, "CHAINED")])
def test_nlm_fast_pan_past_the_search_matches_oracle(oracle, d, estimation):
    """A pan of 14 px per frame, past the 4 + 4 * 2 reach of the unseeded search: the camera model's
    window finds it, and the engine matches the oracle that replays the same models."""
    from conftest import avd
    from gpu_util import Runner
    from test_gpu_nlm_mc import check, options, search

    w, h, n = 192, 112, 7
    fmt = avd.SampleFormat.u8()
    frames = pan_clip(w, h, n, (14, -3), seed=40 + d)
    ms = search(getattr(avd.MotionEstimation, estimation))
    spec = avd.EngineSpec.nlmeans(avd.NlmeansAlgorithm.fast(options(d, 2, 1, 8.0, ms)), None,
                                  avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    check(oracle, got, frames, fmt, d, 2, 1, 8.0, ms)
    assert _moved_share(oracle, frames, fmt, d, ms, chained=estimation == "CHAINED") > 0.01, \
        "premise: the camera model changes the output"


def test_nl4d_fast_pan_past_the_search_matches_oracle(oracle):
    from conftest import avd
    from gpu_util import Runner
    from test_gpu_nl4d import check, opts

    w, h, n, d = 160, 96, 6, 2
    fmt = avd.SampleFormat.u8()
    frames = pan_clip(w, h, n, (-13, 4), seed=5)
    spec = avd.EngineSpec.nl4d(opts(d, 6.0 / 255, spatial_radius=4), None,
                               avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    check(oracle, got, frames, fmt, d, 6.0 / 255, spatial_radius=4)
