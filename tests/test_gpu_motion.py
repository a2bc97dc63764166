"""The block-matching motion search on the GPU through the C ABI against the CPU oracle: pyramid
values, vectors and confidences bit for bit (every SAD is a sequential f32 sum in the reference's
order, and the confidence one correctly rounded division)."""

import ctypes as C

import numpy as np
import pytest

from motion_cases import moving_window

pytestmark = pytest.mark.gpu

CASES = [
    # width, height, frames, levels, blksize, overlap, radius, channels, confidence
    (160, 96, 5, 2, 16, 8, 4, 1, True),
    (123, 77, 3, 3, 16, 8, 6, 2, True),
    (64, 48, 3, 1, 8, 4, 2, 1, False),
    (200, 120, 5, 2, 32, 16, 8, 1, True),
    (96, 64, 5, 1, 16, 8, 0, 1, True),
    (33, 17, 3, 2, 8, 0, 3, 1, True),
]


def gpu_search(lib, ring, w, h, frames, levels, blksize, overlap, radius, channels, confidence, centre, slots,
               sad_floor, thsad, ceiling=0, esc_reads_floor=False):
    import torch

    from av_denoise_b200 import _abi

    dev = torch.from_numpy(ring.reshape(-1)).cuda()
    pyr = torch.zeros(lib.avd_motion_pyramid_floats(w, h, frames, levels), dtype=torch.float32, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for s in range(frames):
        assert lib.avd_motion_pyramid_build(dev.data_ptr(), channels, w, h, frames, s, levels, pyr.data_ptr(), s,
                                            stream) == 0
    step = blksize - overlap
    bx, by = max(-(-w // step), 1), max(-(-h // step), 1)
    n = len(slots)
    slots_t = torch.tensor(np.asarray(slots, np.int32), device="cuda")
    mv = torch.zeros(n * bx * by * 2, dtype=torch.int32, device="cuda")
    conf = torch.zeros(n * bx * by, dtype=torch.float32, device="cuda")
    noise = torch.tensor([sad_floor], dtype=torch.float32, device="cuda")
    p = _abi.AvdMotionPass()
    p.pyramid, p.neighbour_slots, p.mv_field = pyr.data_ptr(), slots_t.data_ptr(), mv.data_ptr()
    p.confidence = conf.data_ptr() if confidence else 0
    p.noise = noise.data_ptr()
    p.width, p.height, p.frame_count, p.centre_slot, p.neighbours = w, h, frames, centre, n
    p.blksize, p.overlap, p.search_radius, p.levels = blksize, overlap, radius, levels
    p.mv_stride, p.conf_stride, p.sad_floor_word, p.thsad = bx * by * 2, bx * by, 0, thsad
    if ceiling:
        state = torch.zeros(lib.avd_escalation_state_floats(n, bx * by), dtype=torch.float32, device="cuda")
        p.escalation, p.ceiling, p.esc_reads_floor = state.data_ptr(), ceiling, int(esc_reads_floor)
    st = lib.avd_motion_search(C.byref(p), stream)
    assert st == 0, lib.avd_last_error().decode()
    torch.cuda.synchronize()
    return pyr.cpu().numpy(), mv.cpu().numpy().reshape(n, bx * by, 2), conf.cpu().numpy().reshape(n, bx * by)


@pytest.mark.parametrize("case", CASES, ids=lambda c: "x".join(map(str, c[:7])))
def test_motion_search_matches_oracle_bit_for_bit(lib, oracle, case):
    w, h, frames, levels, blksize, overlap, radius, channels, confidence = case
    ring = moving_window(w, h, frames, seed=w * 7 + h, channels=channels)
    centre = frames // 2
    slots = [s for s in range(frames) if s != centre][::-1]
    floor = oracle.sad_noise_floor(blksize, 0.02)
    th = oracle.thsad(blksize, 1.0)
    pyr, mv, conf = gpu_search(lib, ring, w, h, frames, levels, blksize, overlap, radius, channels, confidence,
                               centre, slots, floor, th)
    o_pyr = oracle.motion_pyramid(ring, channels, w, h, levels)
    assert np.array_equal(pyr.view(np.uint32), o_pyr.view(np.uint32))
    o_mv, o_conf = oracle.motion_search(o_pyr, w, h, frames, centre, slots, blksize=blksize, overlap=overlap,
                                        search_radius=radius, levels=levels, confidence=confidence,
                                        sad_floor=floor, thsad=th)
    assert np.array_equal(mv, o_mv), np.argwhere(mv != o_mv)[:5]
    if confidence:
        assert np.array_equal(conf.view(np.uint32), o_conf.view(np.uint32))
        assert 0.0 <= conf.min() and conf.max() <= 1.0


def test_seeded_refine_matches_oracle(lib, oracle):
    """The seeded search of the chained refine: no coarse pass, the window centred on each block's
    seed (motion/analyse.rs:273-316), bit for bit."""
    import torch

    from av_denoise_b200 import _abi

    w, h, frames, levels, blksize, overlap, radius = 120, 80, 3, 2, 16, 8, 2
    ring = moving_window(w, h, frames, seed=77)
    o_pyr = oracle.motion_pyramid(ring, 1, w, h, levels)
    step = blksize - overlap
    bx, by = -(-w // step), -(-h // step)
    rng = np.random.default_rng(5)
    seeds = rng.integers(-6, 7, (2, bx * by, 2)).astype(np.int32)
    floor, th = oracle.sad_noise_floor(blksize, 0.02), oracle.thsad(blksize, 1.0)
    o_mv, o_conf = oracle.motion_search(o_pyr, w, h, frames, 1, [0, 2], blksize=blksize, overlap=overlap,
                                        search_radius=radius, levels=levels, confidence=True, sad_floor=floor,
                                        thsad=th, seeds=seeds)
    pyr = torch.from_numpy(o_pyr).cuda()
    slots = torch.tensor([0, 2], dtype=torch.int32, device="cuda")
    mv = torch.from_numpy(seeds.reshape(-1).copy()).cuda()
    conf = torch.zeros(2 * bx * by, device="cuda")
    noise = torch.tensor([floor], device="cuda")
    p = _abi.AvdMotionPass()
    p.pyramid, p.neighbour_slots, p.mv_field, p.confidence, p.noise = (pyr.data_ptr(), slots.data_ptr(),
                                                                         mv.data_ptr(), conf.data_ptr(),
                                                                         noise.data_ptr())
    p.width, p.height, p.frame_count, p.centre_slot, p.neighbours = w, h, frames, 1, 2
    p.blksize, p.overlap, p.search_radius, p.levels = blksize, overlap, radius, levels
    p.mv_stride, p.conf_stride, p.sad_floor_word, p.thsad, p.seeded = bx * by * 2, bx * by, 0, th, 1
    assert lib.avd_motion_search(C.byref(p), C.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0
    torch.cuda.synchronize()
    assert np.array_equal(mv.cpu().numpy().reshape(2, -1, 2), o_mv)
    assert np.array_equal(conf.cpu().numpy().view(np.uint32), o_conf.reshape(-1).view(np.uint32))


@pytest.mark.parametrize("w,h,d,centre,head_mod", [(96, 64, 2, 2, 0), (96, 64, 2, 0, 3), (96, 64, 2, 4, 1),
                                                   (61, 37, 3, 5, 2), (61, 37, 3, 1, 5)])
def test_chain_compose_matches_oracle(lib, oracle, w, h, d, centre, head_mod):
    """The chained seeds: every neighbour's walk through the pair ring (motion/kernels/chain.rs), with
    pair vectors large enough to leave the frame."""
    import torch

    blksize, overlap = 16, 8
    step = blksize - overlap
    bx, by = -(-w // step), -(-h // step)
    rng = np.random.default_rng(w + d + centre)
    pairs = {i: (rng.integers(-9, 10, (bx * by, 2)).astype(np.int32),
                 rng.integers(-9, 10, (bx * by, 2)).astype(np.int32)) for i in range(2 * d)}
    stride = bx * by * 2 + 6
    ring = np.zeros((2 * d, 2, stride), np.int32)
    for i in range(2 * d):
        ring[i, 0, :bx * by * 2] = pairs[i][0].reshape(-1)
        ring[i, 1, :bx * by * 2] = pairs[i][1].reshape(-1)
    dev = torch.from_numpy(ring.reshape(-1)).cuda()
    mv = torch.zeros(2 * d * stride, dtype=torch.int32, device="cuda")
    st = lib.avd_chain_compose(dev.data_ptr(), mv.data_ptr(), stride, centre, d, head_mod, stride, w, h, blksize,
                               overlap, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, lib.avd_last_error().decode()
    torch.cuda.synchronize()
    got = mv.cpu().numpy().reshape(2 * d, stride)[:, :bx * by * 2].reshape(2 * d, bx * by, 2)
    want = oracle.chain_compose(pairs, centre, d, head_mod, step, w, h, bx, by)
    assert np.array_equal(got, want), np.argwhere(got != want)[:5]


TM_CASES = [
    # width, height, frames, levels, blksize, overlap, radius, field_lambda, reads_floor, sigma
    (160, 96, 5, 2, 16, 8, 4, 1.0, True, 0.02),
    (123, 77, 3, 3, 16, 8, 6, 1.0, False, 0.0),
    (200, 120, 3, 2, 32, 16, 8, 2.5, True, 0.05),
    (64, 48, 3, 1, 8, 4, 2, 0.5, True, 0.01),  # one level: no seed candidates
    (33, 17, 3, 2, 8, 0, 3, 1.0, True, 0.03),
    (16, 8, 3, 2, 16, 8, 2, 1.0, True, 0.02),  # a grid of 2 x 1 blocks
]


@pytest.mark.parametrize("case", TM_CASES, ids=lambda c: "x".join(map(str, c[:8])))
def test_search_then_truemotion_matches_oracle_bit_for_bit(lib, oracle, case):
    """The search with its truemotion stage (motion/analyse.rs:175-312): the coarse field kept as the
    seed candidates, then one pass over the fine field; vectors and confidences bit for bit."""
    import torch

    from av_denoise_b200 import _abi

    w, h, frames, levels, blksize, overlap, radius, lam, reads_floor, sigma = case
    ring = moving_window(w, h, frames, seed=w * 3 + h, channels=1)
    rng = np.random.default_rng(w)
    ring = (ring + rng.normal(0, sigma, ring.shape)).astype(np.float32) if sigma else ring
    centre = frames // 2
    slots = [s for s in range(frames) if s != centre][::-1]
    floor = oracle.sad_noise_floor(blksize, sigma)
    th = oracle.thsad(blksize, 1.0)
    o_pyr = oracle.motion_pyramid(ring, 1, w, h, levels)
    o_mv, o_conf = oracle.motion_search(o_pyr, w, h, frames, centre, slots, blksize=blksize, overlap=overlap,
                                        search_radius=radius, levels=levels, confidence=True, sad_floor=floor,
                                        thsad=th, field_lambda=lam, reads_floor=reads_floor)
    plain, _ = oracle.motion_search(o_pyr, w, h, frames, centre, slots, blksize=blksize, overlap=overlap,
                                    search_radius=radius, levels=levels, sad_floor=floor, thsad=th)
    step = blksize - overlap
    bx, by = max(-(-w // step), 1), max(-(-h // step), 1)
    n = len(slots)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    pyr = torch.from_numpy(o_pyr).cuda()
    slots_t = torch.tensor(np.asarray(slots, np.int32), device="cuda")
    mv = torch.zeros(n * bx * by * 2, dtype=torch.int32, device="cuda")
    seeds = torch.zeros_like(mv)
    out = torch.full_like(mv, 12345)
    conf = torch.zeros(n * bx * by, dtype=torch.float32, device="cuda")
    noise = torch.tensor([floor], dtype=torch.float32, device="cuda")
    p = _abi.AvdMotionPass()
    p.pyramid, p.neighbour_slots, p.mv_field, p.confidence, p.noise = (pyr.data_ptr(), slots_t.data_ptr(),
                                                                         mv.data_ptr(), 0, noise.data_ptr())
    p.width, p.height, p.frame_count, p.centre_slot, p.neighbours = w, h, frames, centre, n
    p.blksize, p.overlap, p.search_radius, p.levels = blksize, overlap, radius, levels
    p.mv_stride, p.conf_stride, p.sad_floor_word, p.thsad = bx * by * 2, bx * by, 0, th
    p.keep_seeds = seeds.data_ptr() if levels > 1 else 0
    assert lib.avd_motion_search(C.byref(p), stream) == 0, lib.avd_last_error().decode()
    t = _abi.AvdTruemotionPass()
    t.pyramid, t.neighbour_slots, t.mv_in = pyr.data_ptr(), slots_t.data_ptr(), mv.data_ptr()
    t.seeds = seeds.data_ptr() if levels > 1 else 0
    t.mv_out, t.confidence, t.noise = out.data_ptr(), conf.data_ptr(), noise.data_ptr()
    t.width, t.height, t.frame_count, t.centre_slot, t.neighbours = w, h, frames, centre, n
    t.blksize, t.overlap, t.mv_stride, t.conf_stride = blksize, overlap, bx * by * 2, bx * by
    t.sad_field, t.reads_floor, t.field_lambda, t.thsad = 0, int(reads_floor), lam, th
    assert lib.avd_truemotion_pass(C.byref(t), stream) == 0, lib.avd_last_error().decode()
    torch.cuda.synchronize()
    assert np.array_equal(mv.cpu().numpy().reshape(n, -1, 2), plain)
    got = out.cpu().numpy().reshape(n, -1, 2)
    assert np.array_equal(got, o_mv), np.argwhere(got != o_mv)[:5]
    assert np.array_equal(conf.cpu().numpy().view(np.uint32), o_conf.reshape(-1).view(np.uint32))
    print("blocks the stage changed:", int((got != plain).any(axis=2).sum()), "of", n * bx * by)


def test_truemotion_rejects_bad_passes(lib):
    from av_denoise_b200 import _abi

    t = _abi.AvdTruemotionPass()
    assert lib.avd_truemotion_pass(C.byref(t), None) != 0  # null buffers
    t.pyramid = t.neighbour_slots = t.noise = 256
    t.mv_in = t.mv_out = 512
    t.width, t.height, t.frame_count, t.neighbours, t.blksize, t.overlap = 64, 48, 3, 2, 16, 8
    t.mv_stride, t.conf_stride, t.field_lambda = 2 * 48, 48, 1.0
    assert lib.avd_truemotion_pass(C.byref(t), None) != 0  # mv_out is mv_in
    t.mv_out = 1024
    t.field_lambda = 0.0
    assert lib.avd_truemotion_pass(C.byref(t), None) != 0  # lambda 0 runs no stage
    t.field_lambda, t.mv_stride = 1.0, 10
    assert lib.avd_truemotion_pass(C.byref(t), None) != 0  # stride below the blocks


ESC_CASES = [
    # width, height, frames, levels, blksize, overlap, radius, ceiling, reads floor, sad-floor sigma
    (160, 96, 5, 1, 16, 8, 2, 6, False, 0.02),
    (160, 96, 5, 2, 16, 8, 2, 8, False, 0.02),
    (123, 77, 3, 3, 16, 8, 3, 8, True, 0.02),
    (96, 64, 3, 2, 8, 4, 1, 5, True, 0.0),
    (200, 120, 5, 2, 32, 16, 4, 8, False, 0.05),
    (40, 24, 3, 1, 16, 8, 0, 3, False, 0.02),
    # blksizes outside 8/16/32: the generic fine kernel, then the recorded centres and tracking
    (120, 80, 3, 2, 12, 6, 2, 6, False, 0.02),
    (64, 48, 3, 1, 4, 2, 1, 4, True, 0.02),
]


@pytest.mark.parametrize("case", ESC_CASES, ids=lambda c: "x".join(map(str, c[:8])))
def test_escalating_search_matches_oracle_bit_for_bit(lib, oracle, case):
    """motion/escalate.rs: the first pass's SADs and edge bars, the floor (read or measured), the
    failure flags and the wider search (coarse level included) give the oracle's vectors and
    confidences bit for bit."""
    w, h, frames, levels, blksize, overlap, radius, ceiling, reads, sig = case
    ring = moving_window(w, h, frames, seed=w * 11 + h, channels=1)
    centre = frames // 2
    slots = [s for s in range(frames) if s != centre]
    floor = oracle.sad_noise_floor(blksize, sig)
    th = oracle.thsad(blksize, 1.0)
    _, mv, conf = gpu_search(lib, ring, w, h, frames, levels, blksize, overlap, radius, 1, True, centre, slots,
                             floor, th, ceiling=ceiling, esc_reads_floor=reads)
    o_pyr = oracle.motion_pyramid(ring, 1, w, h, levels)
    o_mv, o_conf = oracle.motion_search(o_pyr, w, h, frames, centre, slots, blksize=blksize, overlap=overlap,
                                        search_radius=radius, levels=levels, confidence=True, sad_floor=floor,
                                        thsad=th, ceiling=ceiling, esc_reads_floor=reads)
    plain, _ = oracle.motion_search(o_pyr, w, h, frames, centre, slots, blksize=blksize, overlap=overlap,
                                    search_radius=radius, levels=levels, confidence=True, sad_floor=floor, thsad=th)
    print("blocks escalated to a new vector:", int(np.any(o_mv != plain, axis=-1).sum()), "of", o_mv.shape[0] * o_mv.shape[1])
    assert np.array_equal(mv, o_mv), np.argwhere(mv != o_mv)[:5]
    assert np.array_equal(conf.view(np.uint32), o_conf.view(np.uint32))
